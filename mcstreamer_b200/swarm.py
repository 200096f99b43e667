"""Python mirror of Swarm (Swarm/src/Swarm.jl): swarm transport coefficients from a
JuMC run in a uniform field, with the time loop and its per-step sums on the GPU.

swarm() follows Swarm.swarm (Swarm.jl:48-186): for each reduced field E/N a fresh
population is advanced nt steps; per step the unweighted means <x>, <x^2> over active
particles give sigma^2(t) (Swarm.jl:126-130) and Swarm.resample! keeps the population
near n0 (:136-138).  Diffusion is half the slope of a least-squares line through the last
100 sigma^2 values (:144-150), the drift W = <v_z> (:152), mobility -W/E (:153), the rate
coefficients k_j = <nu_j(eps)> over active particles (:156, collrate :242-248), and
nu = g.k, alpha = g+.k/|W|, eta = g-.k/|W| (:159-161).  The mean energy is the weighted
mean of population.jl:136-150.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from . import constants as co
from .jumc import CollisionTable, Context, FixedField, ParticleArrays, Population
from .lxcat import LXCatTable

# Swarm.jl:26: NAIR_STP = bar / (k * 273.15)
NAIR_STP = 1e5 / (1.38064852e-23 * 273.15)


def gains(proc) -> np.ndarray:
    """gains (Swarm.jl:229-239): +1 ionization, -1 attachment, 0 otherwise."""
    out = []
    for p in proc:
        if p.kind == L.ATTACHMENT:
            out.append(-1)
        elif p.kind in (L.IONIZATION, L.IONIZATION_UNIFORM):
            out.append(1)
        else:
            out.append(0)
    return np.array(out, dtype=np.float64)


def resample(popl: Population, n: int, tol: float = 0.1) -> None:
    """Swarm.resample!(popl, n, tol) (Swarm.jl:193-223): Russian roulette / Poisson cloning."""
    popl.ctx.check(popl.ctx.lib.mcs_swarm_resample(popl.h, int(n), float(tol)))


def collrate(popl: Population, table: CollisionTable) -> np.ndarray:
    """Mean over active particles of the rate vector (collrate, Swarm.jl:242-248)."""
    m = popl.moments(table)
    return m[L.MOMENTS_BASE:L.MOMENTS_BASE + len(table)] / m[L.M_COUNT]


def diffusion_fit(t: np.ndarray, sigma2: np.ndarray, l: int = 100) -> np.ndarray:
    """[ones(l) t] \\ sigma2 over the last l steps; returns D = slope/2 per axis (Swarm.jl:144-146)."""
    tt = t[-l:]
    A = np.stack([np.ones_like(tt), tt], axis=1)
    coef, *_ = np.linalg.lstsq(A, sigma2[-l:], rcond=None)
    return coef[1] / 2.0


@dataclass
class SwarmResult:
    en: float
    mobility: float
    diffusion_l: float
    diffusion_t: float
    diffusion: float
    nu: float
    alpha: float
    eta: float
    drift: float
    mean_energy: float
    k: np.ndarray
    steps: int
    sigma2: np.ndarray = field(repr=False, default=None)
    counts: np.ndarray = field(repr=False, default=None)
    sums: np.ndarray = field(repr=False, default=None)    # the per-step sums (nt, MCS_STEP_MOMENTS)


def initial_particles(n0: int, init: str, seed: int, mean_ev: float = 1.0) -> ParticleArrays:
    """Swarm.jl:104-106 starts all electrons at rest at the origin ("cold"); the benchmark
    workloads start from an isotropic Maxwellian with <eps> = mean_ev ("maxwellian")."""
    p = ParticleArrays.empty(n0)
    p.w[:] = 1.0
    p.active[:] = 1
    rng = np.random.default_rng(seed)
    if init == "maxwellian":
        sig = np.sqrt((2.0 / 3.0) * mean_ev * co.eV / co.electron_mass)
        p.v[:] = rng.normal(0.0, sig, (n0, 3))
    p.s[:] = -np.log(1.0 - rng.random(n0))
    return p


def coefficients(en_td: float, eb: float, dt: float, mom: np.ndarray, mfin: np.ndarray, proc,
                 l: int = 100) -> SwarmResult:
    """The Swarm.swarm estimators (Swarm.jl:124-161) from the per-step sums of the run
    (mom, (nt, MCS_STEP_MOMENTS): sigma^2(t) of the active electrons) and the moments of the
    final population (mfin, MCS_MOMENTS_BASE + one rate sum per table row): D from the
    least-squares slope of the last l sigma^2, W = <v_z>, k_j = <nu_j(eps)> and nu, alpha,
    eta of the final population; the weighted mean energy."""
    nt = len(mom)
    cnt = mom[:, L.S_COUNT]
    X = mom[:, L.S_X:L.S_X + 3] / cnt[:, None]
    X2 = mom[:, L.S_X2:L.S_X2 + 3] / cnt[:, None]
    sigma2 = X2 - X ** 2
    t = np.arange(nt) * dt
    D = diffusion_fit(t, sigma2, min(l, nt))
    W = mfin[L.M_V + 2] / mfin[L.M_COUNT]
    k = mfin[L.MOMENTS_BASE:L.MOMENTS_BASE + len(proc)] / mfin[L.M_COUNT]
    g = gains(proc)
    return SwarmResult(
        en=en_td, mobility=-W / eb, diffusion_l=D[2], diffusion_t=(D[0] + D[1]) / 2,
        diffusion=(D[0] + D[1] + D[2]) / 3, nu=float(g @ k), alpha=float(np.maximum(g, 0) @ k / abs(W)),
        eta=float(-np.minimum(g, 0) @ k / abs(W)), drift=W, mean_energy=mfin[L.M_WE] / mfin[L.M_W], k=k,
        steps=nt, sigma2=sigma2, counts=cnt, sums=mom)


def time_averages(r: SwarmResult, start: int) -> dict:
    """Drift <v_z> and mean energy per electron averaged over steps [start, nt) of the per-step
    sums: tighter estimates than the final-population values of Swarm.jl:152-156."""
    m = r.sums[start:]
    c = m[:, L.S_COUNT]
    return {"drift": float(np.mean(m[:, L.S_V + 2] / c)), "mean_energy": float(np.mean(m[:, L.S_E] / c))}


def swarm_one(table: CollisionTable, en_td: float, density: float, n0: int, dt: float, nt: int,
              maxp: Optional[int] = None, precision: str = "fp64", seed: int = 0, init: str = "cold",
              resampling: bool = True, tol: float = 0.1, l: int = 100, repack_every: int = 1) -> SwarmResult:
    """One E/N point of Swarm.swarm (Swarm.jl:102-173).  repack_every > 0 compacts the holes
    the roulette leaves (the reference lets them accumulate up to 0.9 maxp instead)."""
    ctx = table.ctx
    maxp = maxp or max(4 * n0, 1024)
    pop = Population(maxp, initial_particles(n0, init, seed), table, precision=precision, seed=seed)
    eb = en_td * density * co.Td
    fld = FixedField(eb, ctx)
    try:
        mom = np.zeros((nt, L.STEP_MOMENTS))
        ctx.check(ctx.lib.mcs_swarm_run(pop.h, table.h, fld.h, dt, nt, n0 if resampling else 0, tol,
                                        repack_every, L.dptr(mom)))
        return coefficients(en_td, eb, dt, mom, pop.moments(table), table.proc, l)
    finally:
        fld.close()
        pop.close()


def swarm(en: Sequence[float], table: LXCatTable, density: float = NAIR_STP, n0: int = 10_000,
          dt: Optional[float] = None, trelax: float = 2e-9, nt: Optional[int] = None, precision: str = "fp64",
          seed: int = 0, init: str = "cold", resampling: bool = True, ctx: Optional[Context] = None,
          maxp: Optional[int] = None) -> list[SwarmResult]:
    """Swarm.swarm(en; ...) (Swarm.jl:48-186).  dt defaults to 1/maxrate/4 and nt to
    ceil(trelax/dt) as in Swarm.jl:76-77."""
    ctab = CollisionTable(table, ctx)
    dt = dt if dt is not None else 1.0 / table.maxrate / 4
    nt = nt if nt is not None else int(np.ceil(trelax / dt))
    try:
        return [swarm_one(ctab, e, density, n0, dt, nt, maxp=maxp, precision=precision, seed=seed + i,
                          init=init, resampling=resampling) for i, e in enumerate(en)]
    finally:
        ctab.close()


def stats(samples: Sequence[Sequence[SwarmResult]]) -> dict[str, np.ndarray]:
    """stats (Swarm.jl:253-269): mean and standard error std/sqrt(n) over replicas."""
    keys = ["mobility", "diffusion_l", "diffusion_t", "diffusion", "nu", "alpha", "eta", "drift", "mean_energy"]
    out: dict[str, np.ndarray] = {"en": np.array([r.en for r in samples[0]])}
    for k in keys:
        a = np.array([[getattr(r, k) for r in rep] for rep in samples])
        out[k] = a.mean(axis=0)
        out[k + "_err"] = a.std(axis=0, ddof=1) / np.sqrt(len(samples)) if len(samples) > 1 else np.zeros(a.shape[1])
    return out


def _block_mean(series, block: int) -> tuple[float, float]:
    """Mean and 3 sigma of the mean from batch means over blocks of `block` samples."""
    a = np.asarray(series, dtype=np.float64)
    nb = len(a) // block
    if nb < 2:
        return float(a.mean()) if len(a) else 0.0, float("inf")
    b = a[len(a) - nb * block:].reshape(nb, block).mean(axis=1)
    return float(b.mean()), float(3.0 * b.std(ddof=1) / np.sqrt(nb))


def fp32_batched_vs_fp64(ctx: Context, table: CollisionTable, ens: Sequence[float], density: float, n0: int,
                         nt: int, warm: int, dt: float, seed: int = 500, chunk: int = 10) -> dict:
    """The batched FP32 form (SwarmBatch, all E/N in one batch) against independent FP64 runs
    of the same swarms (mcs_swarm_run, repack every step), each started from n0 electrons of a
    1 eV Maxwellian.  Over steps [warm, nt): drift W = <v_z>, mean energy <eps> (eV) and the
    ionization rate coefficient k_ion = <nu_ion>/N, each with 3 sigma of its mean from batch
    means (blocks of 30 steps; 3 samples for the FP64 rate, read every `chunk` steps).
    Returns {en: {key: (fp32, 3 sigma, fp64, 3 sigma)}}."""
    from .batch import SwarmBatch
    ion = [j for j, p in enumerate(table.proc) if p.kind in (L.IONIZATION, L.IONIZATION_UNIFORM)]
    f32 = {en: {"W": [], "E": [], "k": []} for en in ens}
    with SwarmBatch(ctx, len(ens), 4 * n0 * len(ens)) as b:
        slots = {en: b.add_maxwellian(table, en * co.Td * density, seed + i, n0, 4 * n0, n0, 1.0)
                 for i, en in enumerate(ens)}
        for _ in range(nt // chunk):
            b.step(dt, chunk)
            for en, k in slots.items():
                s = b.read_log(k, chunk)
                c = s[:, L.S_COUNT]
                f32[en]["W"] += list(s[:, L.S_V + 2] / c)
                f32[en]["E"] += list(s[:, L.S_E] / c / co.eV)
                f32[en]["k"] += list(s[:, L.B_NU] / c / density)
    out = {}
    for i, en in enumerate(ens):
        pop = Population(4 * n0, None, table, precision="fp64", seed=seed + 1000 + i)
        pop.init_maxwellian(n0, 1.0)
        fld = FixedField(en * co.Td * density, ctx)
        W, E, K = [], [], []
        mom = np.zeros((chunk, L.STEP_MOMENTS))
        try:
            for _ in range(nt // chunk):
                ctx.check(ctx.lib.mcs_swarm_run(pop.h, table.h, fld.h, dt, chunk, n0, 0.1, 1, L.dptr(mom)))
                W += list(mom[:, L.S_V + 2] / mom[:, L.S_COUNT])
                E += list(mom[:, L.S_E] / mom[:, L.S_COUNT] / co.eV)
                if ion:
                    m = pop.moments(table)
                    K.append(m[L.MOMENTS_BASE + ion[0]] / m[L.M_COUNT] / density)
        finally:
            fld.close()
            pop.close()
        r = {}
        for key, ser64, blk in (("W", W[warm:], 30), ("E", E[warm:], 30), ("k", K[warm // chunk:], 3)):
            a32, e32 = _block_mean(f32[en][key][warm:], 30)
            a64, e64 = _block_mean(ser64, blk) if len(ser64) else (0.0, float("inf"))
            r[key] = (a32, e32, a64, e64)
        out[en] = r
    return out
