"""The HDF5 subset of mcstreamer_b200.h5: writer/reader round trips in the layout HDF5.jl uses
(h5export, MCStreamer/src/plot.jl:210-238), the on-disk structures checked byte by byte
against the file-format specification, and a file built here from the specification with
the structures the writer does not emit (superblock 2, version-2 object headers, link
messages, chunked storage with the shuffle and deflate filters), as other HDF5 writers
produce them.  No HDF5 library exists in this image to cross-check with."""
import struct
import zlib

import numpy as np
import pytest

from mcstreamer_b200 import h5

UNDEF = 0xFFFFFFFFFFFFFFFF


def test_round_trip_groups_datasets_attributes(tmp_path):
    p = tmp_path / "a.h5"
    rng = np.random.default_rng(1)
    a = np.asfortranarray(rng.normal(size=(5, 7)))
    ints = rng.integers(-2 ** 40, 2 ** 40, size=(4, 3))
    with h5.Writer(str(p)) as w:
        w.create_group("grid")
        w.write("grid/R", 0.015)
        w.write("grid/M", np.int64(1536))
        w.write("grid/rc", np.linspace(0, 1, 11))
        w.write("u", a)
        w.write("p", ints)
        w.write("f32", np.arange(6, dtype=np.float32).reshape(2, 3))
        for k in range(21):                       # three symbol-table nodes in one group
            w.write(f"many/d{k:02d}", np.full(2, k, np.int32))
        w.write_attr("many", "x.delta", 0.25)
        w.write_attr("u", "units", np.array([1, 2, 3], np.int16))
    r = h5.Reader(str(p))
    assert r.keys("/") == ["f32", "grid", "many", "p", "u"]
    assert r.keys("grid") == ["M", "R", "rc"]
    assert r["grid/R"] == 0.015 and r["grid/M"] == 1536
    np.testing.assert_array_equal(r["grid/rc"], np.linspace(0, 1, 11))
    np.testing.assert_array_equal(r["u"], a)
    np.testing.assert_array_equal(r["p"], ints)
    assert r["p"].dtype == np.int64 and r["f32"].dtype == np.float32
    np.testing.assert_array_equal(r["f32"], np.arange(6, dtype=np.float32).reshape(2, 3))
    assert r.keys("many") == [f"d{k:02d}" for k in range(21)]
    np.testing.assert_array_equal(r["many/d17"], [17, 17])
    assert r.attrs("many")["x.delta"] == 0.25
    np.testing.assert_array_equal(r.attrs("u")["units"], [1, 2, 3])
    assert r.is_group("grid") and not r.is_group("u")
    with pytest.raises(KeyError):
        r["nope"]


def test_julia_layout_is_the_transposed_dataset(tmp_path):
    """HDF5.jl stores a Julia M x N matrix as an N x M dataset of its column-major bytes."""
    p = tmp_path / "j.h5"
    a = np.asfortranarray(np.arange(12.0).reshape(3, 4))
    with h5.Writer(str(p)) as w:
        w.write("a", a)
        w.write("c", a, julia=False)
    r = h5.Reader(str(p))
    np.testing.assert_array_equal(r.read("a", julia=False), a.T)      # dataset dims (4, 3)
    np.testing.assert_array_equal(r.read("a"), a)
    np.testing.assert_array_equal(r.read("c", julia=False), a)


def test_on_disk_structures(tmp_path):
    """Superblock version 0 and the structures it points to, field by field."""
    p = tmp_path / "s.h5"
    with h5.Writer(str(p)) as w:
        w.write("x", np.array([1.5, 2.5]))
    b = p.read_bytes()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])        # versions 0, 8-byte offsets/lengths
    leaf_k, internal_k, flags = struct.unpack_from("<HHI", b, 16)
    assert (leaf_k, internal_k, flags) == (4, 16, 0)
    base, freespace, eof, driver = struct.unpack_from("<QQQQ", b, 24)
    assert base == 0 and freespace == UNDEF and driver == UNDEF and eof == len(b)
    name_off, root, cache = struct.unpack_from("<QQI", b, 56)
    btree, heap = struct.unpack_from("<QQ", b, 80)
    assert name_off == 0 and cache == 1
    assert b[btree:btree + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    assert b[root] == 1                                       # object header version 1
    nmsg, refc, size = struct.unpack_from("<HII", b, root + 2)
    mtype, msize = struct.unpack_from("<HH", b, root + 16)
    assert (nmsg, refc, mtype, msize) == (1, 1, 0x11, 16)     # one symbol-table message
    assert struct.unpack_from("<QQ", b, root + 24) == (btree, heap)
    node_type, level, used = struct.unpack_from("<BBH", b, btree + 4)
    assert (node_type, level, used) == (0, 0, 1)
    snod = struct.unpack_from("<Q", b, btree + 32)[0]
    assert b[snod:snod + 4] == b"SNOD" and struct.unpack_from("<BBH", b, snod + 4) == (1, 0, 1)
    seg = struct.unpack_from("<Q", b, heap + 24)[0]
    assert b[seg + 8:seg + 10] == b"x\0"                       # "" at 0, then "x"


# -- a file with the structures the writer does not emit, built from the specification --
def _msg2(mtype, body):
    return struct.pack("<BHB", mtype, len(body), 0) + body


def _ohdr(messages):
    blob = b"".join(_msg2(t, b) for t, b in messages)
    return b"OHDR" + struct.pack("<BB", 2, 0x02) + struct.pack("<I", len(blob)) + blob + b"\0\0\0\0"


def _v2_file(data, chunk):
    """Superblock 2; root group with a link message; a float64 dataset in chunks, shuffled
    and deflated, indexed by a version-1 B-tree."""
    rows, cols = data.shape
    cr, cc = chunk
    out = bytearray(48)
    chunks = []
    for i0 in range(0, rows, cr):
        for j0 in range(0, cols, cc):
            blk = np.zeros((cr, cc))
            part = data[i0:i0 + cr, j0:j0 + cc]
            blk[:part.shape[0], :part.shape[1]] = part
            raw = blk.astype("<f8").tobytes()
            shuf = np.frombuffer(raw, np.uint8).reshape(-1, 8).T.tobytes()
            comp = zlib.compress(shuf, 4)
            chunks.append(((i0, j0), len(out), len(comp)))
            out += comp
    tree = len(out)
    node = b"TREE" + struct.pack("<BBHQQ", 1, 0, len(chunks), UNDEF, UNDEF)
    for (i0, j0), addr, size in chunks:
        node += struct.pack("<IIQQQ", size, 0, i0, j0, 0) + struct.pack("<Q", addr)
    node += struct.pack("<IIQQQ", 0, 0, rows, cols, 0)
    out += node
    dspace = struct.pack("<BBBB", 2, 2, 0, 1) + struct.pack("<QQ", rows, cols)
    dtype = struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    layout = struct.pack("<BBB", 3, 2, 3) + struct.pack("<Q", tree) + struct.pack("<III", cr, cc, 8)
    pipeline = struct.pack("<BB", 2, 2) + struct.pack("<HHHI", 2, 0, 1, 8) + struct.pack("<HHHI", 1, 0, 1, 4)
    dset = len(out)
    out += _ohdr([(0x01, dspace), (0x03, dtype), (0x08, layout), (0x0B, pipeline)])
    name = b"density"
    link = struct.pack("<BB", 1, 0x00) + struct.pack("<B", len(name)) + name + struct.pack("<Q", dset)
    linfo = struct.pack("<BB", 0, 0) + struct.pack("<QQ", UNDEF, UNDEF)
    root = len(out)
    out += _ohdr([(0x02, linfo), (0x06, link)])
    out[:12] = b"\x89HDF\r\n\x1a\n" + bytes([2, 8, 8, 0])
    out[12:44] = struct.pack("<QQQQ", 0, UNDEF, len(out), root)
    return bytes(out)


def test_reads_version2_headers_links_and_filtered_chunks(tmp_path):
    p = tmp_path / "v2.h5"
    data = np.random.default_rng(3).normal(size=(5, 7))
    p.write_bytes(_v2_file(data, (3, 4)))
    r = h5.Reader(str(p))
    assert r.keys("/") == ["density"]
    np.testing.assert_array_equal(r.read("density", julia=False), data)
    np.testing.assert_array_equal(r.read("density"), data.T)


def test_loaders_read_the_reference_layouts(tmp_path):
    """AMLoader and AfivoLoader (initdens.jl:23-55) on files in those layouts."""
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200.initdens import AfivoLoader, AMLoader

    M, N = 6, 9
    rng = np.random.default_rng(2)
    ne = np.asfortranarray(10 ** rng.uniform(15, 19, (M, N)))
    mp, mm = np.asfortranarray(1.1 * ne), np.asfortranarray(0.05 * ne)
    r = (np.arange(M) + 0.5) * 1e-5
    z = (np.arange(N) + 0.5) * 2e-5
    for name, arrs in (("ne.h5", {"e": ne}), ("q.h5", {"e": ne, "M_plus": mp, "M_min": mm})):
        with h5.Writer(str(tmp_path / name)) as w:
            for k, v in arrs.items():
                w.write(k, v)
            w.write("r", r)
            w.write("z", z)
    ne2, q2, dr, dz = AfivoLoader(str(tmp_path / "ne.h5"), str(tmp_path / "q.h5")).load()
    np.testing.assert_array_equal(ne2, ne)
    np.testing.assert_array_equal(q2, co.elementary_charge * (mp - mm - ne))
    assert dr == pytest.approx(1e-5) and dz == pytest.approx(2e-5)
    q = np.asfortranarray(rng.normal(size=(M, N)))
    with h5.Writer(str(tmp_path / "am.h5")) as w:
        w.write("group1/electron_density", ne)
        w.write("group1/charge_density", q)
        w.write_attr("group1", "x.delta", 1e-5)
        w.write_attr("group1", "y.delta", 2e-5)
    ne3, q3, dr3, dz3 = AMLoader(str(tmp_path / "am.h5"), str(tmp_path / "am.h5")).load()
    np.testing.assert_array_equal(ne3, ne)
    np.testing.assert_array_equal(q3, q)
    assert (dr3, dz3) == (1e-5, 2e-5)


def test_edge_values(tmp_path):
    """Empty datasets, booleans (stored as uint8), integer scalars, a group with no links."""
    p = tmp_path / "e.h5"
    with h5.Writer(str(p)) as w:
        w.write("empty", np.zeros(0))
        w.write("flags", np.array([True, False, True]))
        w.write("n", 7)
        w.write("neg", np.int64(-3))
        w.create_group("nothing")
    r = h5.Reader(str(p))
    assert r["empty"].shape == (0,)
    np.testing.assert_array_equal(r["flags"], [1, 0, 1])
    assert r["n"] == 7 and r["neg"] == -3
    assert r.keys("nothing") == []
    with pytest.raises(ValueError):
        with h5.Writer(str(tmp_path / "dup.h5")) as w:
            w.write("a", 1.0)
            w.write("a", 2.0)
    with pytest.raises(ValueError):
        h5.Reader(str(p)).read("nothing")                # a group is not a dataset
    (tmp_path / "bad.h5").write_bytes(b"not an hdf5 file at all")
    with pytest.raises(ValueError):
        h5.Reader(str(tmp_path / "bad.h5"))


def test_reads_a_header_continued_in_another_block(tmp_path):
    """A version-1 object header whose dataset messages sit in a continuation block
    (message 0x10: address and length of the next block), as libraries write when a
    header outgrows its first chunk."""
    p = tmp_path / "c.h5"
    with h5.Writer(str(p)) as w:
        w.write("d", np.arange(5.0))
    b = bytearray(p.read_bytes())
    # find the dataset's header: the symbol-table node's only entry
    btree = struct.unpack_from("<Q", b, 80)[0]
    snod = struct.unpack_from("<Q", b, btree + 32)[0]
    hdr = struct.unpack_from("<Q", b, snod + 8 + 8)[0]
    nmsg, _, size = struct.unpack_from("<HII", b, hdr + 2)
    msgs = bytes(b[hdr + 16:hdr + 16 + size])
    # move every message to a block at the end of the file and leave a continuation behind
    cont_addr = len(b)
    b += msgs
    cont = struct.pack("<HHB3x", 0x10, 16, 0) + struct.pack("<QQ", cont_addr, len(msgs))
    b[hdr + 16:hdr + 16 + len(cont)] = cont
    b[hdr + 16 + len(cont):hdr + 16 + size] = b"\0" * (size - len(cont))   # a NIL message's worth
    struct.pack_into("<H", b, hdr + 2, nmsg + 1)
    struct.pack_into("<I", b, hdr + 8, len(cont))
    struct.pack_into("<Q", b, 40, len(b))          # end-of-file address
    p.write_bytes(bytes(b))
    np.testing.assert_array_equal(h5.Reader(str(p))["d"], np.arange(5.0))


def test_h5export_layout_and_fields(tmp_path, monkeypatch):
    """h5export (plot.jl:210-238) from stand-ins of the device objects: the grid scalars and
    coordinates, each array's slice (cells [1:M, 1:N], er [1:M+1, 1:N], ez [1:M, 1:N+1]) and
    q0 = (qfixed + qpart - ne) e, read back with the Julia shapes."""
    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200 import fieldsio

    M, N = 4, 6
    rng = np.random.default_rng(7)
    dens = {L.Q_FIXED: rng.random((M + 2, N + 2)), L.Q_PART: -rng.random((M + 2, N + 2))}
    qfd = rng.random((M + 2, N + 2))
    ne = rng.random((M + 4, N + 4))
    er, ez = rng.random((M + 3, N + 3)), rng.random((M + 3, N + 3))

    class Grid:
        R, L, M, N = 1e-3, 2e-3, 4, 6
        read_density = staticmethod(lambda which: dens[which])
        read_qfixed_density = staticmethod(lambda: qfd)

    class Solver:
        q = rng.random((M + 2, N + 2))
        u = rng.random((M + 2, N + 2))

    class Fl:
        download = staticmethod(lambda: (ne, None, None))

    monkeypatch.setattr(fieldsio, "read_faces", lambda g: (er, ez))
    p = tmp_path / "f.h5"
    fieldsio.h5export(str(p), Grid, Solver, Fl, p=np.arange(M * N).reshape(M, N))
    f = fieldsio.load_fields(str(p))
    g = f["grid"]
    assert (g["R"], g["L"], g["M"], g["N"]) == (1e-3, 2e-3, M, N)
    np.testing.assert_allclose(g["rc"], (np.arange(M) + 0.5) * 1e-3 / M, rtol=1e-15)
    assert g["zf"].shape == (N + 1,)
    qf = dens[L.Q_FIXED] + qfd
    np.testing.assert_array_equal(f["qfixed"], qf[1:M + 1, 1:N + 1])
    np.testing.assert_array_equal(f["q0"], ((qf + dens[L.Q_PART])[1:M + 1, 1:N + 1] - ne[2:M + 2, 2:N + 2])
                                  * co.elementary_charge)
    np.testing.assert_array_equal(f["u"], Solver.u[1:M + 1, 1:N + 1])
    np.testing.assert_array_equal(f["er"], er[1:M + 2, 1:N + 1])
    np.testing.assert_array_equal(f["ez"], ez[1:M + 1, 1:N + 2])
    np.testing.assert_array_equal(f["p"], np.arange(M * N).reshape(M, N))
    assert (f["wtotal"] == 0).all() and f["p"].dtype == np.int64
    r = h5.Reader(str(p))
    assert r.read("er", julia=False).shape == (N, M + 1)        # HDF5.jl's dataset dims
