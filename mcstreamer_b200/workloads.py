"""Synthetic inputs of the benchmark workloads (seeded, deterministic).

streamer(cfg): the 3-D streamer steps.
  "cfg1": 128x128x256 cells, h = 4 um; E = -15 MV/m z + the field of a Gaussian positive
          charge (sigma 40 um, peak 1e20 e/m^3) at the mesh centre, on nodes;
          4,194,304 particles of weight 1e3 in a Gaussian cloud (sigma 50 um) at the centre,
          1 eV with isotropic directions; synthetic gas 0; dt = 2e-13 s; seed 1.
  "cfg2": 512x512x1024 cells, h = 2 um, the same physical field and cloud (so the mesh
          covers 1 x 1 x 2 mm at twice the resolution); 67,108,864 particles with weights
          log-uniform on [1e2, 1e4]; seed 2.
Particles are generated on the host and sorted by cell key (the layout the cell-sorted
resampling maintains), then uploaded.

batched_swarms(): the batched swarm workload ("cfg3"): 256 instances with E/N log-spaced
  10-1000 Td, electron counts log-uniform 4,096-1,048,576 and one of the synthetic gases
  0, 1, 2 each (seeded, seed 3); N = 2.5e25 m^-3, dt = 1e-13 s, 5000 steps per solve,
  isotropic Maxwellian at 1 eV, Swarm.resample! to the initial count (tol 0.1).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import constants as co
from .jumc import ParticleArrays

STREAMER = {
    "cfg1": dict(nx=128, ny=128, nz=256, h=4e-6, n=4_194_304, weight=(1e3, 1e3), dt=2e-13, seed=1),
    "cfg2": dict(nx=512, ny=512, nz=1024, h=2e-6, n=67_108_864, weight=(1e2, 1e4), dt=2e-13, seed=2),
}
E_BACKGROUND = (0.0, 0.0, -15e6)    # V/m
CHARGE_SIGMA = 40e-6                # m
CHARGE_PEAK = 1e20                  # e / m^3
CLOUD_SIGMA = 50e-6                 # m
CLOUD_ENERGY_EV = 1.0


@dataclass
class StreamerSpec:
    name: str
    nx: int
    ny: int
    nz: int
    h: float
    n: int
    weight: tuple
    dt: float
    seed: int
    centre: tuple = field(default=None)

    @property
    def nodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def streamer_spec(name: str = "cfg1", n: Optional[int] = None) -> StreamerSpec:
    p = dict(STREAMER[name])
    if n is not None:
        p["n"] = int(n)
    s = StreamerSpec(name=name, **p)
    s.centre = (s.nx * s.h / 2, s.ny * s.h / 2, s.nz * s.h / 2)
    return s


def cell_keys(spec: StreamerSpec, x: np.ndarray) -> np.ndarray:
    fl = np.floor(x / spec.h).astype(np.int64)
    inside = np.all((fl >= 0) & (fl < np.array([spec.nx, spec.ny, spec.nz])), axis=1)
    key = fl[:, 0] + spec.nx * (fl[:, 1] + spec.ny * fl[:, 2])
    return np.where(inside, key, np.iinfo(np.int64).max)


def streamer_particles(spec: StreamerSpec, rank: int = 0, chunk: int = 1 << 22) -> ParticleArrays:
    """The particle cloud of `spec` (shard `rank` has its own seed), sorted by cell key."""
    n = spec.n
    rng = np.random.default_rng([spec.seed, rank])
    p = ParticleArrays.empty(n)
    vabs = np.sqrt(2.0 * CLOUD_ENERGY_EV * co.eV / co.electron_mass)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        m = b - a
        p.x[a:b] = np.asarray(spec.centre) + rng.normal(0.0, CLOUD_SIGMA, (m, 3))
        u = 2.0 * rng.random(m) - 1.0
        ph = 2.0 * np.pi * rng.random(m)
        r = np.sqrt(1.0 - u * u)
        p.v[a:b, 0] = vabs * r * np.cos(ph)
        p.v[a:b, 1] = vabs * r * np.sin(ph)
        p.v[a:b, 2] = vabs * u
        lo, hi = spec.weight
        p.w[a:b] = lo if lo == hi else 10 ** rng.uniform(np.log10(lo), np.log10(hi), m)
        p.s[a:b] = -np.log(1.0 - rng.random(m))
    p.active[:] = 1
    order = np.argsort(cell_keys(spec, p.x), kind="stable")
    return ParticleArrays(p.x[order], p.v[order], p.w[order], p.s[order], p.active[order])


def streamer_field_fn(spec: StreamerSpec):
    from .streamer import gaussian_charge_field
    return gaussian_charge_field(spec.centre, CHARGE_SIGMA, CHARGE_PEAK, e_bg=E_BACKGROUND)


SWARM_DENSITY = 2.5e25   # m^-3
SWARM_DT = 1e-13         # s


@dataclass
class BatchedSwarmSpec:
    en_td: np.ndarray        # (K,) reduced fields
    n: np.ndarray            # (K,) electrons per instance (also the resampling target)
    gas: np.ndarray          # (K,) synthetic gas variant
    seeds: np.ndarray        # (K,) per-instance Philox seeds
    steps: int = 5000
    dt: float = SWARM_DT
    density: float = SWARM_DENSITY
    mean_ev: float = 1.0

    @property
    def k(self) -> int:
        return len(self.n)


def batched_swarms(instances: int = 256, seed: int = 3, nmin: int = 4096, nmax: int = 1_048_576,
                   gases: tuple = (0, 1, 2)) -> BatchedSwarmSpec:
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), instances)).astype(np.int64)
    gas = np.asarray(gases)[rng.integers(0, len(gases), instances)]
    return BatchedSwarmSpec(np.logspace(1.0, 3.0, instances), n, gas,
                            np.arange(instances, dtype=np.uint64) + np.uint64(seed) * np.uint64(1_000_003))


def swarm_instance_particles(spec: BatchedSwarmSpec, k: int) -> ParticleArrays:
    """Initial electrons of instance k: isotropic Maxwellian at spec.mean_ev, at the origin."""
    from .swarm import initial_particles
    return initial_particles(int(spec.n[k]), "maxwellian", int(spec.seeds[k]), mean_ev=spec.mean_ev)
