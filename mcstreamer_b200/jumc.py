"""Python mirror of JuMC's particle API over the C ABI.

Names follow the reference (JuMC/src): Julia's mutating `f!` becomes `f`.  A Population
lives on the GPU; `advance` is advance!(mpopl, efield, dt, tracker)
(mixed_population.jl:24), `collisions` is collisions! (:61), `repack` is repack!
(population.jl:191).  Every call goes through libmcs_b200.so; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from . import constants as co
from .lxcat import LXCatTable


class Context:
    """One CUDA device + stream (mcs_ctx)."""

    _default: dict[int, "Context"] = {}

    def __init__(self, device: int = 0, clamp_energy: bool = False):
        self.lib = L.lib()
        h = C.c_void_p()
        L.check(self.lib.mcs_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        if clamp_energy:
            self.set_flags(L.FLAG_CLAMP_ENERGY)

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = cls(device)
        return cls._default[device]

    def set_flags(self, flags: int) -> None:
        L.check(self.lib.mcs_ctx_set_flags(self.h, flags), self.h)

    def set_stream(self, stream_ptr: int) -> None:
        L.check(self.lib.mcs_ctx_set_stream(self.h, C.c_void_p(stream_ptr)), self.h)

    def sync(self) -> None:
        L.check(self.lib.mcs_sync(self.h), self.h)

    def check(self, code: int) -> None:
        L.check(code, self.h)

    def close(self) -> None:
        if self.h:
            self.lib.mcs_ctx_destroy(self.h)
            self.h = None


class CollisionTable:
    """CollisionTable (collisions.jl:9-22) resident on the device."""

    def __init__(self, table: LXCatTable, ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        self.table = table
        self.proc = table.proc
        self.maxrate = table.maxrate
        rate = table.rate_energy_major()
        kinds = table.kinds
        params = table.params
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_table_create(
            self.ctx.h, rate.shape[1], rate.shape[0], table.energy.e0, table.energy.emax, L.dptr(rate),
            L.i32ptr(kinds), L.dptr(params), table.maxrate, C.byref(h)))
        self.h = h
        if getattr(table, "has_photoemission", False):
            lmin = np.ascontiguousarray(table.pe_lmin)
            lmax = np.ascontiguousarray(table.pe_lmax)
            self.ctx.check(self.ctx.lib.mcs_table_set_photoemission(self.h, L.dptr(lmin), L.dptr(lmax),
                                                                   table.photon_multiplier, table.photon_weight))

    def __len__(self) -> int:
        return len(self.proc)

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_table_destroy(self.h)
            self.h = None


class FixedField:
    """FixedField (Swarm/src/Swarm.jl:28-32): E = (0, 0, ez)."""

    def __init__(self, ez: float, ctx: Optional[Context] = None, ex: float = 0.0, ey: float = 0.0):
        self.ctx = ctx or Context.default()
        self.ez = ez
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_field_uniform(self.ctx.h, ex, ey, ez, C.byref(h)))
        self.h = h

    def __call__(self, x):
        return np.array([0.0, 0.0, self.ez])

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_field_destroy(self.h)
            self.h = None


@dataclass
class ParticleArrays:
    """Host copy of a population in the Julia StructArray layout."""

    x: np.ndarray       # (n, 3) float64
    v: np.ndarray       # (n, 3) float64
    w: np.ndarray       # (n,) float64
    s: np.ndarray       # (n,) float64
    active: np.ndarray  # (n,) uint8

    @property
    def n(self) -> int:
        return len(self.w)

    @staticmethod
    def empty(n: int) -> "ParticleArrays":
        return ParticleArrays(np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n), np.zeros(n, np.uint8))

    def copy(self) -> "ParticleArrays":
        return ParticleArrays(self.x.copy(), self.v.copy(), self.w.copy(), self.s.copy(), self.active.copy())

    def energy(self) -> np.ndarray:
        return 0.5 * co.electron_mass * (self.v ** 2).sum(axis=1)


class Population:
    """Population (JuMC/src/population.jl:4-36) on the device.

    precision: "fp64" (parity mode) or "fp32" (FP32 push/sampling, FP64 time and sums).
    mesh: a grid created with Grid3D to store positions as (cell, in-cell offset).
    """

    def __init__(self, max_particles: int, particles: Optional[ParticleArrays], collisions: CollisionTable,
                 precision: str = "fp64", seed: int = 0, step: int = 0, mesh=None, ctx: Optional[Context] = None):
        self.ctx = ctx or collisions.ctx
        self.collisions = collisions
        self.capacity = int(max_particles)
        self.precision = precision
        prec = L.FP32 if precision == "fp32" else L.FP64
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_pop_create(self.ctx.h, self.capacity, prec,
                                                   mesh.h_ if mesh is not None else None, C.byref(h)))
        self.h = h
        self.mesh = mesh
        self.set_seed(seed, step)
        if particles is not None:
            self.upload(particles)

    # ---- state transfer ----
    def set_seed(self, seed: int, step: int = 0) -> None:
        self.ctx.check(self.ctx.lib.mcs_pop_set_seed(self.h, C.c_uint64(seed), step))

    @property
    def step(self) -> int:
        s = C.c_uint32()
        self.ctx.check(self.ctx.lib.mcs_pop_get_step(self.h, C.byref(s)))
        return s.value

    def set_uniforms(self, per_slot: Optional[Sequence[Sequence[float]]]) -> None:
        """Feed the following steps' draws from given values instead of the Philox streams
        (mcs_set_uniform_source): per_slot[i] are slot i's uniforms in the order the
        reference's serial run draws them (rand() in util.jl:5,8,17, collisions.jl:166).
        None returns to the streams."""
        lib = self.ctx.lib
        if per_slot is None:
            self.ctx.check(lib.mcs_set_uniform_source(self.h, L.UNIFORMS_PHILOX, None, None, 0))
            return
        lens = np.array([len(a) for a in per_slot], dtype=np.int64)
        offsets = np.zeros(len(lens) + 1, dtype=np.int64)
        np.cumsum(lens, out=offsets[1:])
        u = np.concatenate([np.asarray(a, dtype=np.float64) for a in per_slot]) if len(lens) else np.zeros(0)
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.ctx.check(lib.mcs_set_uniform_source(self.h, L.UNIFORMS_INJECTED, L.dptr(u), L.i64ptr(offsets),
                                                  len(lens)))

    def init_maxwellian(self, n: int, mean_ev: float = 1.0) -> None:
        """n swarm electrons drawn on the device (origin, weight 1, isotropic Maxwellian)."""
        self.ctx.check(self.ctx.lib.mcs_pop_init_maxwellian(self.h, int(n), float(mean_ev)))

    def init_cloud(self, n: int, centre, sigma: float, energy_ev: float, wmin: float, wmax: float) -> None:
        """n electrons of a Gaussian cloud drawn on the device (mcs_pop_init_cloud); unsorted."""
        cx, cy, cz = map(float, centre)
        self.ctx.check(self.ctx.lib.mcs_pop_init_cloud(self.h, int(n), cx, cy, cz, float(sigma), float(energy_ev),
                                                       float(wmin), float(wmax)))

    def upload(self, p: ParticleArrays) -> None:
        x = np.ascontiguousarray(p.x, dtype=np.float64)
        v = np.ascontiguousarray(p.v, dtype=np.float64)
        w = np.ascontiguousarray(p.w, dtype=np.float64)
        s = np.ascontiguousarray(p.s, dtype=np.float64)
        a = np.ascontiguousarray(p.active, dtype=np.uint8)
        self.ctx.check(self.ctx.lib.mcs_pop_upload(self.h, L.dptr(x), L.dptr(v), L.dptr(w), L.dptr(s), L.u8ptr(a),
                                                   len(w)))

    def download(self) -> ParticleArrays:
        n = self.nparticles()
        out = ParticleArrays.empty(n)
        nn = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_pop_download(self.h, L.dptr(out.x), L.dptr(out.v), L.dptr(out.w),
                                                     L.dptr(out.s), L.u8ptr(out.active), n, C.byref(nn)))
        return out

    # ---- population.jl accessors ----
    @property
    def n(self) -> int:
        return self.nparticles()

    def nparticles(self) -> int:
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_pop_nparticles(self.h, C.byref(n)))
        return n.value

    def moments(self, table: Optional[CollisionTable] = None) -> np.ndarray:
        nrows = len(table) if table is not None else 0
        out = np.zeros(L.MOMENTS_BASE + nrows)
        self.ctx.check(self.ctx.lib.mcs_moments(self.h, table.h if table is not None else None, L.dptr(out),
                                                len(out)))
        return out

    def nactives(self) -> int:
        return int(self.moments()[L.M_COUNT])

    actives = nactives

    def weight(self) -> float:
        return float(self.moments()[L.M_W])

    def meanenergy(self) -> float:
        m = self.moments()
        return float(m[L.M_WE] / m[L.M_W])

    def maxenergy(self) -> float:
        return float(self.moments()[L.M_EMAX])

    def spread(self):
        m = self.moments()
        xm = m[L.M_WX:L.M_WX + 3] / m[L.M_W]
        x2 = m[L.M_WX2] / m[L.M_W]
        return xm, float(np.sqrt(x2 - xm @ xm))

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_pop_destroy(self.h)
            self.h = None


@dataclass
class PhotonArrays:
    """Host PhotonState arrays (JuMC/src/photon.jl:11-18), Julia layout."""

    x: np.ndarray        # (n, 3)
    v: np.ndarray        # (n, 3)
    nu: np.ndarray       # absorption rate (1/s)
    w: np.ndarray
    s: np.ndarray
    active: np.ndarray   # uint8

    @staticmethod
    def empty(n: int) -> "PhotonArrays":
        return PhotonArrays(np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n), np.zeros(n),
                            np.zeros(n, np.uint8))


class Photons:
    """The photon population of a streamer run (MCStreamer/src/main.jl:115-121): FP64,
    collisions at maxrate numax (ZhelezniakCollisions)."""

    def __init__(self, capacity: int, numax: float, seed: int = 0, ctx: Optional[Context] = None,
                 photons: Optional[PhotonArrays] = None):
        self.ctx = ctx or Context.default()
        self.capacity, self.numax = int(capacity), float(numax)
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_photons_create(self.ctx.h, self.capacity, self.numax, int(seed), C.byref(h)))
        self.h = h
        if photons is not None:
            self.upload(photons)

    def upload(self, p: PhotonArrays) -> None:
        n = len(p.w)
        a = [np.ascontiguousarray(q, dtype=np.float64) for q in (p.x, p.v, p.nu, p.w, p.s)]
        act = np.ascontiguousarray(p.active, dtype=np.uint8)
        self.ctx.check(self.ctx.lib.mcs_photons_upload(self.h, *(L.dptr(q) for q in a), L.u8ptr(act), n))

    def count(self) -> int:
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_photons_count(self.h, C.byref(n)))
        return n.value

    def moments(self) -> np.ndarray:
        """[actives, weight] over the active photons (population.jl:114-131)."""
        out = np.zeros(2)
        self.ctx.check(self.ctx.lib.mcs_photons_moments(self.h, L.dptr(out)))
        return out

    def actives(self) -> int:
        return int(self.moments()[0])

    def repack(self) -> None:
        """repack!(photons) (population.jl:191-215)."""
        self.ctx.check(self.ctx.lib.mcs_photons_repack(self.h))

    def weight(self) -> float:
        return float(self.moments()[1])

    def download(self) -> PhotonArrays:
        n = self.count()
        out = PhotonArrays.empty(n)
        nn = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_photons_download(self.h, L.dptr(out.x), L.dptr(out.v), L.dptr(out.nu),
                                                         L.dptr(out.w), L.dptr(out.s), L.u8ptr(out.active), n,
                                                         C.byref(nn)))
        return out

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_photons_destroy(self.h)
            self.h = None


def advance_mixed(electrons: "Population", photons: Photons, efield, dt: float, tracker=None) -> None:
    """advance!(mpopl, efield, dt, tracker) with MultiPopulation(electron, photon)
    (mixed_population.jl:24-54): photo-emission adds photons, photo-ionization electrons."""
    electrons.ctx.check(electrons.ctx.lib.mcs_advance_mixed(electrons.h, photons.h, electrons.collisions.h,
                                                            efield.h, dt,
                                                            tracker.h if tracker is not None else None))


class MultiPopulation:
    """MultiPopulation (mixed_population.jl:4-17) restricted to the electron population."""

    def __init__(self, **index):
        self.index = index

    def __iter__(self):
        return iter(self.index.values())


def _pops(mpopl):
    if isinstance(mpopl, Population):
        return [mpopl]
    return list(mpopl)


def advance(mpopl, efield, dt: float, tracker=None) -> None:
    """advance!(mpopl, efield, dt, tracker) (JuMC/src/mixed_population.jl:24-54)."""
    for popl in _pops(mpopl):
        popl.ctx.check(popl.ctx.lib.mcs_advance(popl.h, popl.collisions.h, efield.h, dt,
                                                tracker.h if tracker is not None else None))


def collisions(mpopl, dt: float, tracker=None) -> None:
    """collisions!(mpopl, dt, tracker) (JuMC/src/mixed_population.jl:61-77)."""
    for popl in _pops(mpopl):
        popl.ctx.check(popl.ctx.lib.mcs_collisions(popl.h, popl.collisions.h, dt,
                                                   tracker.h if tracker is not None else None))


def repack(popl: Population) -> None:
    """repack!(popl) (JuMC/src/population.jl:191-215)."""
    popl.ctx.check(popl.ctx.lib.mcs_repack(popl.h))


def nparticles(popl: Population) -> int:
    return popl.nparticles()


def nactives(popl: Population) -> int:
    return popl.nactives()
