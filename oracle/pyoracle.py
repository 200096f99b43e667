"""ctypes wrapper of liboracle.so -- TEST INFRASTRUCTURE (the checker, never the product)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB, build

pd = C.POINTER(C.c_double)
pi64 = C.POINTER(C.c_int64)
pu8 = C.POINTER(C.c_uint8)
pi32 = C.POINTER(C.c_int)

NULL, ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, IONIZATION_UNIFORM, PHOTOEMISSION = 0, 1, 2, 3, 4, 5, 6
TAG_ADVANCE, TAG_SWARM_RESAMPLE, TAG_CELL_RESAMPLE, TAG_INIT, TAG_COLLISIONS, TAG_PHOTON = 0, 1, 2, 3, 4, 5


class Table(C.Structure):
    _fields_ = [("nrows", C.c_int), ("neps", C.c_int), ("e0", C.c_double), ("de", C.c_double),
                ("emax", C.c_double), ("rate", pd), ("kind", pi32), ("param", pd), ("maxrate", C.c_double),
                ("pe_lmin", pd), ("pe_lmax", pd), ("pe_mult", C.c_double), ("pe_pw", C.c_double)]


class Photons(C.Structure):
    _fields_ = [("x", pd), ("v", pd), ("nu", pd), ("w", pd), ("s", pd), ("active", pu8), ("n", C.c_int64),
                ("cap", C.c_int64), ("seed", C.c_uint64), ("step", C.c_uint32), ("numax", C.c_double)]


class Pop(C.Structure):
    _fields_ = [("x", pd), ("v", pd), ("w", pd), ("s", pd), ("active", pu8), ("n", C.c_int64),
                ("cap", C.c_int64), ("seed", C.c_uint64), ("step", C.c_uint32)]


class Field(C.Structure):
    _fields_ = [("type", C.c_int), ("e", C.c_double * 3), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("h", C.c_double), ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
                ("enodes", pd), ("R", C.c_double), ("L", C.c_double), ("M", C.c_int), ("N", C.c_int),
                ("er", pd), ("ez", pd)]


class Tracker(C.Structure):
    _fields_ = [("type", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("h", C.c_double),
                ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("qnodes", pi64),
                ("R", C.c_double), ("L", C.c_double), ("M", C.c_int), ("N", C.c_int), ("qcyl", pd)]


_L = None


def lib():
    global _L
    if _L is None:
        build()
        L = C.CDLL(str(LIB))
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_uniform.restype = C.c_double
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_advance.argtypes = [C.POINTER(Pop), C.POINTER(Table), C.POINTER(Field), C.c_double,
                                  C.POINTER(Tracker), C.c_int, C.c_int]
        L.orc_collisions.argtypes = [C.POINTER(Pop), C.POINTER(Table), C.c_double, C.POINTER(Tracker), C.c_int,
                                     C.c_int]
        L.orc_advance_injected.argtypes = [C.POINTER(Pop), C.POINTER(Table), C.POINTER(Field), C.c_double,
                                           C.POINTER(Tracker), C.c_int, C.c_int, pd, pi64, pi64, C.c_int64]
        L.orc_efield.argtypes = [C.POINTER(Field), pd, pd]
        L.orc_yoshida.argtypes = [C.POINTER(Field), pd, pd, C.c_double]
        L.orc_indweight.argtypes = [C.POINTER(Table), C.c_double, pi64, pd]
        L.orc_repack.argtypes = [C.POINTER(Pop)]
        L.orc_swarm_resample.argtypes = [C.POINTER(Pop), C.c_int64, C.c_double]
        L.orc_moments.argtypes = [C.POINTER(Pop), C.POINTER(Table), pd]
        L.orc_cell_key.restype = C.c_int64
        L.orc_cell_key.argtypes = [C.POINTER(Field), pd]
        L.orc_sort_cells.argtypes = [C.POINTER(Pop), C.POINTER(Field)]
        L.orc_resample_cells.argtypes = [C.POINTER(Pop), C.POINTER(Field), C.c_int, C.c_int, C.c_uint32]
        L.orc_deposit.argtypes = [C.POINTER(Pop), C.POINTER(Tracker), C.c_double, C.c_int]
        L.orc_advance_mixed.argtypes = [C.POINTER(Pop), C.POINTER(Photons), C.POINTER(Table), C.POINTER(Field),
                                        C.c_double, C.POINTER(Tracker), C.c_int, C.c_int]
        L.orc_photon_advance.argtypes = [C.POINTER(Photons), C.POINTER(Pop), C.c_double, C.POINTER(Tracker), C.c_int]
        L.orc_photons_repack.argtypes = [C.POINTER(Photons)]
        _L = L
    return _L


def philox(ctr, key):
    U4 = C.c_uint32 * 4
    U2 = C.c_uint32 * 2
    out = U4()
    lib().orc_philox4x32_10(U4(*ctr), U2(*key), out)
    return list(out)


def uniform(seed, c0, c1, tag, k):
    return lib().orc_uniform(seed, c0, c1, tag, k)


class OracleTable:
    """Keeps numpy buffers alive behind an orc_table."""

    def __init__(self, rate_em: np.ndarray, kinds: np.ndarray, params: np.ndarray, e0: float, emax: float,
                 maxrate: float, pe=None):
        self.rate = np.ascontiguousarray(rate_em, dtype=np.float64)
        self.kinds = np.ascontiguousarray(kinds, dtype=np.int32)
        self.params = np.ascontiguousarray(params, dtype=np.float64)
        neps, nrows = self.rate.shape
        self.s = Table(nrows, neps, e0, (emax - e0) / (neps - 1), emax, self.rate.ctypes.data_as(pd),
                       self.kinds.ctypes.data_as(pi32), self.params.ctypes.data_as(pd), maxrate)
        if pe is not None:   # (lmin per row, lmax per row, photon_multiplier, photon_weight)
            self.pe_lmin = np.ascontiguousarray(pe[0], dtype=np.float64)
            self.pe_lmax = np.ascontiguousarray(pe[1], dtype=np.float64)
            self.s.pe_lmin = self.pe_lmin.ctypes.data_as(pd)
            self.s.pe_lmax = self.pe_lmax.ctypes.data_as(pd)
            self.s.pe_mult, self.s.pe_pw = float(pe[2]), float(pe[3])

    @classmethod
    def from_lxcat(cls, t):
        pe = None
        if getattr(t, "has_photoemission", False):
            pe = (t.pe_lmin, t.pe_lmax, t.photon_multiplier, t.photon_weight)
        return cls(t.rate_energy_major(), t.kinds, t.params, t.energy.e0, t.energy.emax, t.maxrate, pe)


class OraclePop:
    """Host population with capacity, Julia layout."""

    def __init__(self, x, v, w, s, active, cap=None, seed=0, step=0):
        n = len(w)
        cap = cap or n
        self.x = np.zeros((cap, 3)); self.x[:n] = x
        self.v = np.zeros((cap, 3)); self.v[:n] = v
        self.w = np.zeros(cap); self.w[:n] = w
        self.s = np.zeros(cap); self.s[:n] = s
        self.active = np.zeros(cap, np.uint8); self.active[:n] = active
        self.p = Pop(self.x.ctypes.data_as(pd), self.v.ctypes.data_as(pd), self.w.ctypes.data_as(pd),
                     self.s.ctypes.data_as(pd), self.active.ctypes.data_as(pu8), n, cap, seed, step)

    @property
    def n(self):
        return self.p.n

    def arrays(self):
        n = self.p.n
        return self.x[:n].copy(), self.v[:n].copy(), self.w[:n].copy(), self.s[:n].copy(), self.active[:n].copy()


class OraclePhotons:
    """Host photon population (PhotonState, JuMC/src/photon.jl:11-18) with capacity."""

    def __init__(self, cap, numax, seed=0, step=0, x=None, v=None, nu=None, w=None, s=None, active=None):
        n = 0 if w is None else len(w)
        self.x = np.zeros((cap, 3)); self.v = np.zeros((cap, 3))
        self.nu = np.zeros(cap); self.w = np.zeros(cap); self.s = np.zeros(cap)
        self.active = np.zeros(cap, np.uint8)
        if n:
            self.x[:n] = x; self.v[:n] = v; self.nu[:n] = nu; self.w[:n] = w; self.s[:n] = s
            self.active[:n] = active
        self.p = Photons(self.x.ctypes.data_as(pd), self.v.ctypes.data_as(pd), self.nu.ctypes.data_as(pd),
                         self.w.ctypes.data_as(pd), self.s.ctypes.data_as(pd), self.active.ctypes.data_as(pu8),
                         n, cap, seed, step, numax)

    @property
    def n(self):
        return self.p.n

    def arrays(self):
        n = self.p.n
        return (self.x[:n].copy(), self.v[:n].copy(), self.nu[:n].copy(), self.w[:n].copy(), self.s[:n].copy(),
                self.active[:n].copy())


def advance_mixed(pop, photons, table, field, dt, tracker=None, threads=None, clamp=False):
    """advance!(mpopl, efield, dt, tracker) over electrons and photons."""
    return lib().orc_advance_mixed(C.byref(pop.p), C.byref(photons.p), C.byref(table.s), C.byref(field), dt,
                                   C.byref(tracker) if tracker is not None else None, threads or nthreads(),
                                   int(clamp))


def photons_repack(photons):
    return lib().orc_photons_repack(C.byref(photons.p))


def photon_advance(photons, pop, dt, tracker=None, threads=None):
    return lib().orc_photon_advance(C.byref(photons.p), C.byref(pop.p), dt,
                                    C.byref(tracker) if tracker is not None else None, threads or nthreads())


def field_uniform(ex=0.0, ey=0.0, ez=0.0):
    f = Field()
    f.type = 0
    f.e[0], f.e[1], f.e[2] = ex, ey, ez
    return f


def field_cart3d(nx, ny, nz, h, origin, enodes):
    f = Field()
    f.type = 1
    f.nx, f.ny, f.nz, f.h = nx, ny, nz, h
    f.x0, f.y0, f.z0 = origin
    f._keep = np.ascontiguousarray(enodes, dtype=np.float64)
    f.enodes = f._keep.ctypes.data_as(pd)
    return f


def field_cyl(R, L_, M, N, er, ez):
    f = Field()
    f.type = 2
    f.R, f.L, f.M, f.N = R, L_, M, N
    f._er = np.ascontiguousarray(er, dtype=np.float64)
    f._ez = np.ascontiguousarray(ez, dtype=np.float64)
    f.er = f._er.ctypes.data_as(pd)
    f.ez = f._ez.ctypes.data_as(pd)
    return f


def tracker_cart3d(nx, ny, nz, h, origin):
    t = Tracker()
    t.type = 1
    t.nx, t.ny, t.nz, t.h = nx, ny, nz, h
    t.x0, t.y0, t.z0 = origin
    t._q = np.zeros((nx + 1) * (ny + 1) * (nz + 1), dtype=np.int64)
    t.qnodes = t._q.ctypes.data_as(pi64)
    return t


def tracker_cyl(R, L_, M, N):
    t = Tracker()
    t.type = 2
    t.R, t.L, t.M, t.N = R, L_, M, N
    t._q = np.zeros((M + 2) * (N + 2), dtype=np.float64)
    t.qcyl = t._q.ctypes.data_as(pd)
    return t


def nthreads():
    return int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))


def advance(pop: OraclePop, table: OracleTable, field, dt, tracker=None, threads=None, clamp=False):
    return lib().orc_advance(C.byref(pop.p), C.byref(table.s), C.byref(field), dt,
                             C.byref(tracker) if tracker is not None else None, threads or nthreads(), int(clamp))


def advance_injected(pop: OraclePop, table: OracleTable, field, dt, per_slot, tracker=None, threads=None,
                     clamp=False):
    """advance! with each slot's draws taken from per_slot[i] in the reference's serial order."""
    lens = np.array([len(a) for a in per_slot], dtype=np.int64)
    end = np.cumsum(lens).astype(np.int64)
    pos = (end - lens).astype(np.int64)
    u = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in per_slot]) if len(lens) else
                             np.zeros(1))
    return lib().orc_advance_injected(C.byref(pop.p), C.byref(table.s), C.byref(field), dt,
                                      C.byref(tracker) if tracker is not None else None, threads or nthreads(),
                                      int(clamp), u.ctypes.data_as(pd), pos.ctypes.data_as(pi64),
                                      end.ctypes.data_as(pi64), len(lens))


def collisions(pop, table, dt, tracker=None, threads=None, clamp=False):
    return lib().orc_collisions(C.byref(pop.p), C.byref(table.s), dt,
                                C.byref(tracker) if tracker is not None else None, threads or nthreads(), int(clamp))


def repack(pop):
    return lib().orc_repack(C.byref(pop.p))


def swarm_resample(pop, n0, tol=0.1):
    return lib().orc_swarm_resample(C.byref(pop.p), n0, tol)


def moments(pop, table=None):
    nrows = table.s.nrows if table is not None else 0
    out = np.zeros(18 + nrows)
    lib().orc_moments(C.byref(pop.p), C.byref(table.s) if table is not None else None, out.ctypes.data_as(pd))
    return out


def sort_cells(pop, grid_field):
    return lib().orc_sort_cells(C.byref(pop.p), C.byref(grid_field))


def resample_cells(pop, grid_field, ntarget, nmax, call):
    return lib().orc_resample_cells(C.byref(pop.p), C.byref(grid_field), ntarget, nmax, call)


def deposit(pop, tracker, val, quantize_f32=False):
    lib().orc_deposit(C.byref(pop.p), C.byref(tracker), val, int(quantize_f32))
    return tracker._q


def efield(field, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    e = np.zeros(3)
    lib().orc_efield(C.byref(field), x.ctypes.data_as(pd), e.ctypes.data_as(pd))
    return e


def swarm_run(pop: OraclePop, table: OracleTable, field, dt: float, nt: int, n0: int, tol: float = 0.1,
              repack_every: int = 1, threads=None):
    """The oracle's Swarm.swarm time loop (Swarm/src/Swarm.jl:124-142): per step advance!, the
    sums of the active electrons (the first 12 moments: count, sum w, x, x^2, v, energy), then
    Swarm.resample!(n0, tol) and repack!; returns the (nt, 12) per-step sums and the moments
    (with the rate sums of `table`) of the final population."""
    nrows = table.s.nrows
    mom = np.zeros((nt, 12))
    buf = np.zeros(18 + nrows)
    for i in range(nt):
        st = advance(pop, table, field, dt, threads=threads)
        if st:
            raise RuntimeError(f"oracle advance! status {st}")
        mom[i] = moments(pop)[:12]
        if n0 > 0:
            swarm_resample(pop, n0, tol)
        if repack_every > 0 and (i + 1) % repack_every == 0:
            repack(pop)
    buf[:] = moments(pop, table)
    return mom, buf
