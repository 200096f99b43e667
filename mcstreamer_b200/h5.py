"""A small HDF5 reader and writer for the files MCStreamer exchanges (numpy only).

MCStreamer writes its grid fields with HDF5.jl (`h5export`, MCStreamer/src/plot.jl:210-238)
and reads its initial densities from HDF5 files (`loadinit`, MCStreamer/src/initdens.jl:
23-55).  This image has no HDF5 library, so this module implements the part of the HDF5
file format (the HDF Group's "HDF5 File Format Specification", version 3) those files use.

Writer: superblock version 0, version-1 object headers, groups as symbol tables (a v1 group
B-tree, symbol-table nodes and a local heap for the names), contiguous datasets of fixed-point
and IEEE floating-point numbers (little-endian), scalar or n-dimensional, and attributes.
These are the structures every HDF5 library version reads.

Reader: superblock versions 0-3; object headers of version 1 and 2 with continuation blocks;
groups as symbol tables or as compact link messages; datasets with compact, contiguous or
chunked (v1 B-tree index) storage, the deflate, shuffle and Fletcher-32 filters; fixed-point
and floating-point types of either byte order; attributes.  Dense link storage (fractal
heaps), variable-length and compound types are not read.

Julia arrays are column-major and HDF5.jl stores an M x N array as an N x M dataset whose
bytes are the array's column-major bytes.  `write(..., julia=True)` stores a numpy array the
same way and `read(..., julia=True)` returns it with the Julia shape.
"""
from __future__ import annotations

import struct
import zlib
from typing import Dict, List, Optional, Tuple, Union

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K, INTERNAL_K = 4, 16          # the library's defaults for group nodes

Scalar = Union[int, float, np.integer, np.floating]


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


# -----------------------------------------------------------------------------------------
# Datatype and dataspace messages
# -----------------------------------------------------------------------------------------
def _datatype_message(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    if dt.byteorder == ">":
        raise ValueError("big-endian arrays are written after conversion to little-endian")
    if dt.kind == "f":
        if dt.itemsize == 8:
            sign, eloc, esize, msize, bias = 63, 52, 11, 52, 1023
        elif dt.itemsize == 4:
            sign, eloc, esize, msize, bias = 31, 23, 8, 23, 127
        else:
            raise TypeError(f"unsupported float size {dt.itemsize}")
        head = struct.pack("<B3BI", (1 << 4) | 1, 0x20, sign, 0, dt.itemsize)
        props = struct.pack("<HHBBBBI", 0, 8 * dt.itemsize, eloc, esize, 0, msize, bias)
        return head + props
    if dt.kind in "iub":
        signed = 0x08 if dt.kind == "i" else 0
        head = struct.pack("<B3BI", (1 << 4) | 0, signed, 0, 0, dt.itemsize)
        return head + struct.pack("<HH", 0, 8 * dt.itemsize)
    raise TypeError(f"unsupported dtype {dt}")


def _dataspace_message(shape: Tuple[int, ...]) -> bytes:
    out = struct.pack("<BBBB4x", 1, len(shape), 0, 0)
    for d in shape:
        out += struct.pack("<Q", d)
    return out


# -----------------------------------------------------------------------------------------
# Writer
# -----------------------------------------------------------------------------------------
class _Node:
    def __init__(self):
        self.attrs: Dict[str, np.ndarray] = {}


class _Group(_Node):
    def __init__(self):
        super().__init__()
        self.children: Dict[str, _Node] = {}


class _Dataset(_Node):
    def __init__(self, data: np.ndarray, shape: Tuple[int, ...]):
        super().__init__()
        self.data, self.shape = data, shape


def _as_array(value, julia: bool) -> Tuple[np.ndarray, Tuple[int, ...]]:
    a = np.asarray(value)
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    if a.dtype.kind not in "iuf":
        raise TypeError(f"unsupported value type {a.dtype}")
    a = a.astype(a.dtype.newbyteorder("<"), copy=False)
    if a.ndim == 0:
        return a.reshape(1), ()
    if julia:
        return np.ascontiguousarray(a.ravel(order="F")), tuple(reversed(a.shape))
    return np.ascontiguousarray(a), tuple(a.shape)


class Writer:
    """Builds the object tree in memory and writes the file on close()."""

    def __init__(self, path: str):
        self.path = path
        self.root = _Group()

    def _parent(self, path: str, create: bool = True) -> Tuple[_Group, str]:
        parts = [p for p in path.split("/") if p]
        if not parts:
            raise ValueError("empty path")
        g = self.root
        for p in parts[:-1]:
            nxt = g.children.get(p)
            if nxt is None:
                if not create:
                    raise KeyError(path)
                nxt = g.children[p] = _Group()
            if not isinstance(nxt, _Group):
                raise ValueError(f"{p} is not a group")
            g = nxt
        return g, parts[-1]

    def create_group(self, path: str) -> None:
        g, name = self._parent(path)
        if name in g.children:
            raise ValueError(f"{path} exists")
        g.children[name] = _Group()

    def write(self, path: str, value, julia: bool = True) -> None:
        g, name = self._parent(path)
        if name in g.children:
            raise ValueError(f"{path} exists")
        data, shape = _as_array(value, julia)
        g.children[name] = _Dataset(data, shape)

    def write_attr(self, path: str, name: str, value, julia: bool = True) -> None:
        node: _Node = self.root
        for p in [p for p in path.split("/") if p]:
            node = node.children[p]   # type: ignore[attr-defined]
        node.attrs[name] = _as_array(value, julia)   # type: ignore[assignment]

    # -- layout ------------------------------------------------------------------------
    def close(self) -> None:
        buf = bytearray(96)          # the superblock, filled last
        objects: List[Tuple[int, bytes]] = []
        cursor = [96]

        def alloc(n: int) -> int:
            a = cursor[0]
            cursor[0] += n + (-n % 8)
            return a

        def attr_messages(node: _Node) -> List[Tuple[int, bytes]]:
            out = []
            for name, (data, shape) in node.attrs.items():
                nm = name.encode() + b"\0"
                dtm, dsm = _datatype_message(data.dtype), _dataspace_message(shape)
                body = struct.pack("<BBHHH", 1, 0, len(nm), len(dtm), len(dsm))
                body += _pad8(nm) + _pad8(dtm) + _pad8(dsm) + data.tobytes()
                out.append((0x000C, body))
            return out

        def header(messages: List[Tuple[int, bytes]]) -> bytes:
            blob = b""
            for mtype, body in messages:
                body = _pad8(body)
                blob += struct.pack("<HHB3x", mtype, len(body), 0) + body
            return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(blob)) + blob

        def place_dataset(d: _Dataset) -> int:
            raw = d.data.tobytes()
            data_addr = alloc(len(raw)) if raw else UNDEF
            msgs = [(0x0001, _dataspace_message(d.shape)), (0x0003, _datatype_message(d.data.dtype)),
                    (0x0005, struct.pack("<BBBB", 2, 2, 2, 0)),
                    (0x0008, struct.pack("<BBQQ", 3, 1, data_addr, len(raw)))]
            msgs += attr_messages(d)
            hdr = header(msgs)
            addr = alloc(len(hdr))
            if raw:
                objects.append((data_addr, raw))
            objects.append((addr, hdr))
            return addr

        def place_group(g: _Group) -> Tuple[int, int, int]:
            names = sorted(g.children, key=lambda s: s.encode())
            child = {n: place(g.children[n]) for n in names}
            # local heap: "" at offset 0, then every name, each padded to 8 bytes
            seg = bytearray(8)
            offs = {}
            for n in names:
                offs[n] = len(seg)
                seg += _pad8(n.encode() + b"\0")
            seg_addr = alloc(len(seg))
            # no free block: the library's end-of-free-list value, 1
            heap = b"HEAP" + struct.pack("<B3xQQQ", 0, len(seg), 1, seg_addr)
            heap_addr = alloc(len(heap))
            objects.append((seg_addr, bytes(seg)))
            objects.append((heap_addr, heap))
            # symbol-table nodes of up to 2K entries, in name order
            per = 2 * LEAF_K
            chunks = [names[i:i + per] for i in range(0, len(names), per)] or [[]]
            if len(chunks) > 2 * INTERNAL_K:
                raise ValueError("group too large for one B-tree node")
            snods = []
            for ch in chunks:
                body = b"SNOD" + struct.pack("<BBH", 1, 0, len(ch))
                for n in ch:
                    c_addr, c_btree, c_heap = child[n]
                    if c_btree is not None:
                        body += struct.pack("<QQII QQ", offs[n], c_addr, 1, 0, c_btree, c_heap)
                    else:
                        body += struct.pack("<QQII16x", offs[n], c_addr, 0, 0)
                body += b"\0" * (8 + 40 * per - len(body))
                a = alloc(len(body))
                objects.append((a, body))
                snods.append((a, ch))
            # one leaf B-tree node over them: key 0 is "", key i the last name of child i-1
            bt = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(snods) if names else 0, UNDEF, UNDEF)
            bt += struct.pack("<Q", 0)
            for a, ch in snods:
                if not names:
                    break
                bt += struct.pack("<QQ", a, offs[ch[-1]])
            bt += b"\0" * (24 + 8 * (2 * INTERNAL_K) + 8 * (2 * INTERNAL_K + 1) - len(bt))
            bt_addr = alloc(len(bt))
            objects.append((bt_addr, bt))
            msgs = [(0x0011, struct.pack("<QQ", bt_addr, heap_addr))] + attr_messages(g)
            hdr = header(msgs)
            addr = alloc(len(hdr))
            objects.append((addr, hdr))
            return addr, bt_addr, heap_addr

        def place(node: _Node):
            if isinstance(node, _Group):
                return place_group(node)
            return place_dataset(node), None, None   # type: ignore[arg-type]

        root_addr, root_bt, root_heap = place_group(self.root)
        eof = cursor[0]
        sb = SIGNATURE + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0)
        sb += struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII QQ", 0, root_addr, 1, 0, root_bt, root_heap)
        assert len(sb) == 96
        buf[:96] = sb
        out = bytearray(eof)
        out[:96] = buf
        for a, b in objects:
            out[a:a + len(b)] = b
        with open(self.path, "wb") as f:
            f.write(out)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if exc[0] is None:
            self.close()


# -----------------------------------------------------------------------------------------
# Reader
# -----------------------------------------------------------------------------------------
def _parse_datatype(b: bytes, o: int = 0) -> np.dtype:
    cv, f0, f1, f2, size = struct.unpack_from("<BBBBI", b, o)
    cls = cv & 0x0F
    order = ">" if f0 & 1 else "<"
    if cls == 0:
        return np.dtype(f"{order}{'i' if f0 & 0x08 else 'u'}{size}")
    if cls == 1:
        if size not in (4, 8):
            raise TypeError(f"unsupported float size {size}")
        return np.dtype(f"{order}f{size}")
    raise TypeError(f"unsupported HDF5 datatype class {cls}")


def _parse_dataspace(b: bytes, o: int = 0) -> Tuple[int, ...]:
    ver, ndims, flags = struct.unpack_from("<BBB", b, o)
    if ver == 1:
        p = o + 8
    elif ver == 2:
        if b[o + 3] == 2:         # null dataspace
            return (0,)
        p = o + 4
    else:
        raise ValueError(f"dataspace version {ver}")
    return tuple(struct.unpack_from(f"<{ndims}Q", b, p)) if ndims else ()


class Reader:
    """Read datasets, groups and attributes: `r["group1/electron_density"]`,
    `r.attrs("group1")`, `r.keys("grid")`."""

    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.b = f.read()
        b = self.b
        base = b.find(SIGNATURE)
        if base != 0:
            raise ValueError("not an HDF5 file (no signature at offset 0)")
        ver = b[8]
        if ver in (0, 1):
            self.so, self.sl = b[13], b[14]
            if (self.so, self.sl) != (8, 8):
                raise ValueError("only 8-byte offsets and lengths are supported")
            p = 24 + (4 if ver == 1 else 0) + 32
            self.root = struct.unpack_from("<Q", b, p + 8)[0]
        elif ver in (2, 3):
            self.so, self.sl = b[9], b[10]
            if (self.so, self.sl) != (8, 8):
                raise ValueError("only 8-byte offsets and lengths are supported")
            self.root = struct.unpack_from("<Q", b, 12 + 24)[0]
        else:
            raise ValueError(f"superblock version {ver}")

    # -- object headers ----------------------------------------------------------------
    def _messages(self, addr: int) -> List[Tuple[int, bytes]]:
        b = self.b
        out: List[Tuple[int, bytes]] = []
        if b[addr:addr + 4] == b"OHDR":
            flags = b[addr + 5]
            p = addr + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            sz = 1 << (flags & 3)
            size = int.from_bytes(b[p:p + sz], "little")
            p += sz
            blocks = [(p, p + size)]
            while blocks:
                s, e = blocks.pop(0)
                q = s
                while q + 4 <= e:        # a gap shorter than a message prefix ends the block
                    mtype, msize, _ = struct.unpack_from("<BHB", b, q)
                    q += 4 + (2 if flags & 0x04 else 0)
                    body = b[q:q + msize]
                    q += msize
                    if mtype == 0x10:
                        caddr, clen = struct.unpack_from("<QQ", body, 0)
                        blocks.append((caddr + 4, caddr + clen - 4))   # "OCHK" ... checksum
                    elif mtype:
                        out.append((mtype, body))
            return out
        if b[addr] != 1:
            raise ValueError(f"object header version {b[addr]} at {addr}")
        nmsg, _, size = struct.unpack_from("<HII", b, addr + 2)
        blocks = [(addr + 16, addr + 16 + size)]
        count = 0
        while blocks and count < nmsg:
            s, e = blocks.pop(0)
            q = s
            while q + 8 <= e and count < nmsg:
                mtype, msize, mflags = struct.unpack_from("<HHB", b, q)
                body = b[q + 8:q + 8 + msize]
                q += 8 + msize
                count += 1
                if mtype == 0x10:
                    caddr, clen = struct.unpack_from("<QQ", body, 0)
                    blocks.append((caddr, caddr + clen))
                else:
                    out.append((mtype, body))
        return out

    # -- groups ------------------------------------------------------------------------
    def _heap_string(self, heap: int, off: int) -> str:
        seg = struct.unpack_from("<Q", self.b, heap + 24)[0]
        end = self.b.index(b"\0", seg + off)
        return self.b[seg + off:end].decode()

    def _btree_group(self, addr: int, heap: int, out: Dict[str, int]) -> None:
        b = self.b
        if b[addr:addr + 4] != b"TREE":
            raise ValueError("bad group B-tree node")
        level = b[addr + 5]
        used = struct.unpack_from("<H", b, addr + 6)[0]
        p = addr + 24 + 8
        for _ in range(used):
            child = struct.unpack_from("<Q", b, p)[0]
            p += 16
            if level > 0:
                self._btree_group(child, heap, out)
            else:
                if b[child:child + 4] != b"SNOD":
                    raise ValueError("bad symbol-table node")
                n = struct.unpack_from("<H", b, child + 6)[0]
                for k in range(n):
                    e = child + 8 + 40 * k
                    name_off, obj = struct.unpack_from("<QQ", b, e)
                    out[self._heap_string(heap, name_off)] = obj

    def _links(self, addr: int) -> Dict[str, int]:
        links: Dict[str, int] = {}
        for mtype, body in self._messages(addr):
            if mtype == 0x11:
                bt, heap = struct.unpack_from("<QQ", body, 0)
                self._btree_group(bt, heap, links)
            elif mtype == 0x06:
                flags = body[1]
                p = 2
                ltype = 0
                if flags & 0x08:
                    ltype = body[p]
                    p += 1
                if flags & 0x04:
                    p += 8
                if flags & 0x10:
                    p += 1
                lsz = 1 << (flags & 3)
                nlen = int.from_bytes(body[p:p + lsz], "little")
                p += lsz
                name = body[p:p + nlen].decode()
                p += nlen
                if ltype == 0:
                    links[name] = struct.unpack_from("<Q", body, p)[0]
            elif mtype == 0x02:
                fheap = struct.unpack_from("<Q", body, 2 + (8 if body[1] & 1 else 0))[0]
                if fheap != UNDEF:
                    raise NotImplementedError("dense link storage (fractal heap) is not read")
        return links

    def _resolve(self, path: str) -> int:
        addr = self.root
        for part in [p for p in path.split("/") if p]:
            links = self._links(addr)
            if part not in links:
                raise KeyError(path)
            addr = links[part]
        return addr

    def keys(self, path: str = "/") -> List[str]:
        return sorted(self._links(self._resolve(path)))

    def is_group(self, path: str) -> bool:
        return any(t in (0x11, 0x06, 0x02) for t, _ in self._messages(self._resolve(path)))

    # -- attributes --------------------------------------------------------------------
    def attrs(self, path: str = "/", julia: bool = True) -> Dict[str, np.ndarray]:
        out = {}
        for mtype, body in self._messages(self._resolve(path)):
            if mtype != 0x0C:
                continue
            ver = body[0]
            nlen, dtlen, dslen = struct.unpack_from("<HHH", body, 2)
            p = 8 if ver in (1, 2) else 9
            pad = (lambda n: n + (-n % 8)) if ver == 1 else (lambda n: n)
            name = body[p:p + nlen].split(b"\0")[0].decode()
            p += pad(nlen)
            dt = _parse_datatype(body, p)
            p += pad(dtlen)
            shape = _parse_dataspace(body, p)
            p += pad(dslen)
            n = int(np.prod(shape)) if shape else 1
            a = np.frombuffer(body, dtype=dt, count=n, offset=p).astype(dt.newbyteorder("="))
            out[name] = self._shape(a, shape, julia)
        return out

    # -- datasets ----------------------------------------------------------------------
    @staticmethod
    def _shape(a: np.ndarray, shape: Tuple[int, ...], julia: bool):
        if not shape:
            return a[0]
        if julia:
            return a.reshape(tuple(reversed(shape)), order="F")
        return a.reshape(shape)

    def read(self, path: str, julia: bool = True):
        msgs = self._messages(self._resolve(path))
        shape: Optional[Tuple[int, ...]] = None
        dt: Optional[np.dtype] = None
        layout: Optional[bytes] = None
        filters: List[Tuple[int, Tuple[int, ...]]] = []
        for mtype, body in msgs:
            if mtype == 0x01:
                shape = _parse_dataspace(body)
            elif mtype == 0x03:
                dt = _parse_datatype(body)
            elif mtype == 0x08:
                layout = body
            elif mtype == 0x0B:
                filters = self._filters(body)
        if shape is None or dt is None or layout is None:
            raise ValueError(f"{path} is not a dataset")
        n = int(np.prod(shape)) if shape else 1
        raw = self._raw(layout, shape, dt, filters, n)
        a = np.frombuffer(raw, dtype=dt, count=n).astype(dt.newbyteorder("="))
        return self._shape(a, shape, julia)

    __getitem__ = read

    @staticmethod
    def _filters(body: bytes) -> List[Tuple[int, Tuple[int, ...]]]:
        ver, nf = body[0], body[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(nf):
            fid, = struct.unpack_from("<H", body, p)
            if ver == 1 or fid >= 256:
                nlen = struct.unpack_from("<H", body, p + 2)[0]
                flags, nval = struct.unpack_from("<HH", body, p + 4)
                p += 8
                p += nlen + ((-nlen % 8) if ver == 1 else 0)
            else:
                flags, nval = struct.unpack_from("<HH", body, p + 2)
                p += 6
            vals = struct.unpack_from(f"<{nval}I", body, p)
            p += 4 * nval
            if ver == 1 and nval % 2:
                p += 4
            out.append((fid, vals))
        return out

    @staticmethod
    def _unfilter(chunk: bytes, filters, mask: int, itemsize: int) -> bytes:
        for k in range(len(filters) - 1, -1, -1):
            if mask & (1 << k):
                continue
            fid, _ = filters[k]
            if fid == 1:
                chunk = zlib.decompress(chunk)
            elif fid == 2:
                a = np.frombuffer(chunk, dtype=np.uint8)
                n = len(a) // itemsize
                chunk = a[:n * itemsize].reshape(itemsize, n).T.tobytes() + a[n * itemsize:].tobytes()
            elif fid == 3:
                chunk = chunk[:-4]
            else:
                raise NotImplementedError(f"HDF5 filter {fid}")
        return chunk

    def _raw(self, layout: bytes, shape, dt: np.dtype, filters, n: int) -> bytes:
        b = self.b
        ver, cls = layout[0], layout[1]
        if ver not in (3, 4):
            raise NotImplementedError(f"data layout version {ver}")
        nbytes = n * dt.itemsize
        if cls == 0:
            size = struct.unpack_from("<H", layout, 2)[0]
            return layout[4:4 + size]
        if cls == 1:
            addr, size = struct.unpack_from("<QQ", layout, 2)
            if addr == UNDEF:
                return b"\0" * nbytes
            return b[addr:addr + size]
        if cls == 2 and ver == 3:
            rank = layout[2]
            btree = struct.unpack_from("<Q", layout, 3)[0]
            cdims = struct.unpack_from(f"<{rank}I", layout, 11)   # last one is the element size
            cshape = tuple(cdims[:-1])
            full = np.zeros(shape if shape else (1,), dtype=dt)
            if btree != UNDEF:
                for offs, addr, size, mask in self._chunks(btree, rank):
                    raw = self._unfilter(b[addr:addr + size], filters, mask, dt.itemsize)
                    blk = np.frombuffer(raw, dtype=dt, count=int(np.prod(cshape))).reshape(cshape)
                    sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cshape, shape))
                    full[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]
            return full.tobytes()
        raise NotImplementedError(f"data layout class {cls} (version {ver})")

    def _chunks(self, addr: int, rank: int):
        b = self.b
        if b[addr:addr + 4] != b"TREE":
            raise ValueError("bad chunk B-tree node")
        level = b[addr + 5]
        used = struct.unpack_from("<H", b, addr + 6)[0]
        ksize = 8 + 8 * rank
        p = addr + 24
        for _ in range(used):
            size, mask = struct.unpack_from("<II", b, p)
            offs = struct.unpack_from(f"<{rank}Q", b, p + 8)
            child = struct.unpack_from("<Q", b, p + ksize)[0]
            p += ksize + 8
            if level > 0:
                yield from self._chunks(child, rank)
            else:
                yield offs[:-1], child, size, mask
