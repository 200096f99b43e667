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

poisson_spec(): the electrostatic solve of poisson! on the reference's sample grid
  (MCStreamer samples/input.toml: R = 1.5 cm, L = 10 cm, 1536 x 10240 cells, 9 multigrid
  levels, tolerance 1e8 e, 2 + 2 smoothing sweeps): a negative-streamer channel along the
  axis, 4,194,304 electrons of weight 1.5e6 (radial Gaussian sigma 0.5 mm, z uniform on
  [2, 6] cm, a tenth of them in a Gaussian head of sigma 1 mm at z = 6 cm) over the
  analytic ion density of the channel body alone, background field -1.5 MV/m; seed 1.
  Each solve starts from a zero potential.

photon_step_spec(): advance! over electrons and photons (photo-emission, photon flight,
  photo-ionization) in the cylindrical streamer geometry; see PhotonStepSpec.

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


@dataclass
class PoissonSpec:
    R: float = 0.015
    L: float = 0.1
    M: int = 1536
    N: int = 10240
    levels: int = 9
    n: int = 4_194_304
    weight: float = 1.5e6
    sigma_r: float = 5e-4
    z0: float = 0.02
    z1: float = 0.06
    head_frac: float = 0.1
    head_sigma: float = 1e-3
    eb: float = -1.5e6
    seed: int = 1


def poisson_spec() -> PoissonSpec:
    return PoissonSpec()


def poisson_electrons(spec: PoissonSpec) -> ParticleArrays:
    """The channel's electrons (at rest: only their positions and weights matter here)."""
    rng = np.random.default_rng(spec.seed)
    n = spec.n
    nh = int(round(spec.head_frac * n))
    x = np.empty((n, 3))
    rr = spec.sigma_r * np.sqrt(-2.0 * np.log1p(-rng.random(n)))
    th = 2.0 * np.pi * rng.random(n)
    x[:, 0] = rr * np.cos(th)
    x[:, 1] = rr * np.sin(th)
    x[:n - nh, 2] = rng.uniform(spec.z0, spec.z1, n - nh)
    x[n - nh:, 2] = spec.z1 + spec.head_sigma * rng.standard_normal(nh)
    x[:, 2] = np.clip(x[:, 2], 1e-6, spec.L - 1e-6)
    p = ParticleArrays.empty(n)
    p.x[:] = x
    p.w[:] = spec.weight
    p.s[:] = 1.0
    p.active[:] = 1
    return p


def poisson_ion_charge(spec: PoissonSpec) -> np.ndarray:
    """qfixed: the expected charge of the channel body's electrons, positive, as int64 cell
    charges (2^-32 e, index i + j*(M+2))."""
    M, N = spec.M, spec.N
    dr, dz = spec.R / M, spec.L / N
    rf = np.arange(M + 1) * dr
    zf = np.arange(N + 1) * dz
    # electrons per cell of the body: n_body * P(r-shell) * P(z-slab)
    n_body = spec.n - int(round(spec.head_frac * spec.n))
    pr = np.diff(-np.exp(-rf ** 2 / (2 * spec.sigma_r ** 2)))
    pz = np.diff(np.clip((zf - spec.z0) / (spec.z1 - spec.z0), 0.0, 1.0))
    q = np.zeros((M + 2, N + 2), order="F")
    q[1:M + 1, 1:N + 1] = n_body * spec.weight * pr[:, None] * pz[None, :]
    return np.rint(q * 2.0 ** 32).astype(np.int64).ravel(order="F")


def poisson_electron_charge(spec: PoissonSpec, x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """density!(grid, qpart, electrons, val = -1) as int64 cell charges: nearest cell,
    rho and z cells by floor, particles outside skipped (poisson.jl:65-84)."""
    M, N = spec.M, spec.N
    dr, dz = spec.R / M, spec.L / N
    i = np.floor(np.hypot(x[:, 0], x[:, 1]) / dr).astype(np.int64) + 1
    j = np.floor(x[:, 2] / dz).astype(np.int64) + 1
    ok = (i >= 1) & (i <= M) & (j >= 0) & (j <= N + 1)
    q = np.zeros((M + 2) * (N + 2), dtype=np.int64)
    np.add.at(q, i[ok] + j[ok] * (M + 2), np.rint(-w[ok] * 2.0 ** 32).astype(np.int64))
    return q


@dataclass
class PhotonStepSpec:
    """advance! over electrons and photons in the cylindrical streamer geometry: a
    0.5 x 2 mm grid of 128 x 512 cells whose face field is a uniform -15 MV/m; 4,194,304
    electrons of weight 1e3 in a Gaussian cloud (sigma 100 um) at the axis midpoint, 5 eV
    Maxwellian, FP32; 1,048,576 photons from the same cloud (isotropic, log-uniform nu over the
    table's band, weight 1); synthetic gas 0 with its photo-emission process (absorber 20% of
    the gas, photon_multiplier 1000, photon_weight 1, as the reference's sample input);
    dt = 1e-12 s; seed 1."""
    R: float = 5e-4
    L: float = 2e-3
    M: int = 128
    N: int = 512
    n_e: int = 4_194_304
    n_ph: int = 1_048_576
    weight: float = 1e3
    sigma: float = 1e-4
    mean_ev: float = 5.0
    ez: float = -1.5e7
    dt: float = 1e-12
    photon_multiplier: float = 1000.0
    photon_weight: float = 1.0
    seed: int = 1


def photon_step_spec() -> PhotonStepSpec:
    return PhotonStepSpec()


def photon_step_electrons(spec: PhotonStepSpec, n: Optional[int] = None) -> ParticleArrays:
    n = spec.n_e if n is None else n
    rng = np.random.default_rng(spec.seed)
    p = ParticleArrays.empty(n)
    p.x[:] = rng.normal(0.0, spec.sigma, (n, 3))
    p.x[:, 2] += 0.5 * spec.L
    sig = np.sqrt((2.0 / 3.0) * spec.mean_ev * co.eV / co.electron_mass)
    p.v[:] = rng.normal(0.0, sig, (n, 3))
    p.w[:] = spec.weight
    p.s[:] = -np.log(rng.random(n))
    p.active[:] = 1
    return p


def photon_step_photons(spec: PhotonStepSpec, lmin: float, lmax: float, n: Optional[int] = None):
    """(x, v, nu, w, s, active) of the initial photons."""
    n = spec.n_ph if n is None else n
    rng = np.random.default_rng(spec.seed + 1)
    x = rng.normal(0.0, spec.sigma, (n, 3))
    x[:, 2] += 0.5 * spec.L
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    nu = np.exp(lmin + (lmax - lmin) * rng.random(n))
    return (x, d * co.speed_of_light, nu, np.full(n, spec.photon_weight), -np.log(rng.random(n)),
            np.ones(n, np.uint8))


# ---------------------------------------------------------------------------------------
# The electron fluid: the sample grid with fluid_threshold = 1e20 (samples/input.toml), the
# cells of a channel denser than the threshold carried by the fluid (initdens.jl:78-82).
# ---------------------------------------------------------------------------------------
@dataclass
class FluidSpec:
    poisson: PoissonSpec = field(default_factory=PoissonSpec)
    peak: float = 1e21          # channel density on the axis (m^-3)
    threshold: float = 1e20     # fluid_threshold (m^-3)
    dt: float = 1e-12


def fluid_spec() -> FluidSpec:
    return FluidSpec()


def fluid_density(spec: FluidSpec) -> np.ndarray:
    """ne (M+4, N+4), Fortran order, two ghost layers: the channel body of the Poisson
    workload (Gaussian in r of width sigma_r, z0 <= z <= z1) at a peak density `peak`, where
    it exceeds the threshold, zero elsewhere."""
    p = spec.poisson
    M, N = p.M, p.N
    rc = (np.arange(M) + 0.5) * (p.R / M)
    zc = (np.arange(N) + 0.5) * (p.L / N)
    dens = spec.peak * np.exp(-rc[:, None] ** 2 / (2 * p.sigma_r ** 2)) * ((zc >= p.z0) & (zc <= p.z1))[None, :]
    ne = np.zeros((M + 4, N + 4), order="F")
    ne[2:M + 2, 2:N + 2] = np.where(dens > spec.threshold, dens, 0.0)
    return ne


# ---------------------------------------------------------------------------------------
# initfromfiles! on the sample grid: the fluid workload's channel as the init files' electron
# density, PoissonInitSampling(ntarget = 10) and fluid_threshold = 1e20 (samples/input.toml).
# ---------------------------------------------------------------------------------------
@dataclass
class InitSpec:
    fluid: FluidSpec = field(default_factory=FluidSpec)
    p: int = 10
    seed: int = 1


def init_spec() -> InitSpec:
    return InitSpec()


def init_densities(spec: InitSpec):
    """(ne, q) as loadinit returns them, (M, N) Fortran-ordered: the channel of peak
    `fluid.peak` (m^-3) everywhere, and a net charge of 1 % of its electron density."""
    f = spec.fluid
    p = f.poisson
    rc = (np.arange(p.M) + 0.5) * (p.R / p.M)
    zc = (np.arange(p.N) + 0.5) * (p.L / p.N)
    ne = f.peak * np.exp(-rc[:, None] ** 2 / (2 * p.sigma_r ** 2)) * ((zc >= p.z0) & (zc <= p.z1))[None, :]
    ne = np.asfortranarray(ne)
    q = np.asfortranarray(0.01 * 1.6021766208e-19 * ne)
    return ne, q


def loop_spec() -> InitSpec:
    """The streamer loop's initial state: initfromfiles! over a channel of peak 1e17 m^-3 with
    the fluid above 5e16 m^-3.  Electron weights max(1, ne dV / p) stay below ~2e3 on the sample
    grid, so photo-emission (photon_multiplier 1000) makes about one photon per event, as in
    the photon workload; the 1e21 m^-3 channel of the init workload would weigh electrons at up
    to 6e6 and emit thousands of photons per event."""
    return InitSpec(fluid=FluidSpec(peak=1e17, threshold=5e16))
