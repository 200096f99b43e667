"""Shared helpers of the parity tests: seeded inputs and comparisons."""
from __future__ import annotations

import numpy as np

from mcstreamer_b200 import constants as co
from mcstreamer_b200.jumc import ParticleArrays
from mcstreamer_b200 import lxcat
from oracle import jumc_ref as R
from oracle import pyoracle as po


def maxwellian(n: int, seed: int, mean_ev: float = 1.0, x0=(0.0, 0.0, 0.0), spread: float = 0.0) -> ParticleArrays:
    """Isotropic Maxwellian with <eps> = mean_ev (kT = 2/3 mean), s = -log(U)."""
    rng = np.random.default_rng(seed)
    sig = np.sqrt((2.0 / 3.0) * mean_ev * co.eV / co.electron_mass)
    v = rng.normal(0.0, sig, (n, 3))
    x = np.tile(np.asarray(x0, dtype=np.float64), (n, 1))
    if spread:
        x = x + rng.normal(0.0, spread, (n, 3))
    return ParticleArrays(x, v, np.ones(n), -np.log(1.0 - rng.random(n)), np.ones(n, np.uint8))


def broad(n: int, seed: int, emax_ev: float = 120.0, x0=(0.0, 0.0, 0.0), spread: float = 0.0) -> ParticleArrays:
    """Energies uniform on [0, emax_ev] with isotropic directions: every process fires."""
    rng = np.random.default_rng(seed)
    e = rng.random(n) * emax_ev * co.eV
    vabs = np.sqrt(2.0 * e / co.electron_mass)
    u = 2.0 * rng.random(n) - 1.0
    ph = 2.0 * np.pi * rng.random(n)
    r = np.sqrt(1.0 - u * u)
    v = vabs[:, None] * np.stack([r * np.cos(ph), r * np.sin(ph), u], axis=1)
    x = np.tile(np.asarray(x0, dtype=np.float64), (n, 1))
    if spread:
        x = x + rng.normal(0.0, spread, (n, 3))
    w = np.ones(n)
    return ParticleArrays(x, v, w, -np.log(1.0 - rng.random(n)), np.ones(n, np.uint8))


def oracle_pop(p: ParticleArrays, cap: int, seed: int, step: int = 0) -> po.OraclePop:
    return po.OraclePop(p.x, p.v, p.w, p.s, p.active, cap=cap, seed=seed, step=step)


def oracle_arrays(op: po.OraclePop) -> ParticleArrays:
    x, v, w, s, a = op.arrays()
    return ParticleArrays(x, v, w, s, a)


def relerr(a: np.ndarray, b: np.ndarray, atol: float = 0.0) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(a), np.abs(b))
    err = np.abs(a - b)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(err <= atol, 0.0, err / np.where(den > 0, den, 1.0))
    return r


def vec_relerr(a: np.ndarray, b: np.ndarray, atol: float = 0.0) -> np.ndarray:
    """|a - b| / max(|a|, |b|) per row (3-vectors), 0 where |a - b| <= atol."""
    d = np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=1)
    den = np.maximum(np.linalg.norm(a, axis=1), np.linalg.norm(b, axis=1))
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(d <= atol, 0.0, d / np.where(den > 0, den, 1.0))


def particle_mismatch(g: ParticleArrays, o: ParticleArrays, rtol: float, xatol: float = 0.0,
                      vatol: float = 0.0, satol: float = 0.0, n: int | None = None) -> np.ndarray:
    """Boolean mask of slots whose state differs beyond the tolerance."""
    n = n if n is not None else min(g.n, o.n)
    bad = np.zeros(n, dtype=bool)
    bad |= vec_relerr(g.x[:n], o.x[:n], xatol) > rtol
    bad |= vec_relerr(g.v[:n], o.v[:n], vatol) > rtol
    bad |= relerr(g.w[:n], o.w[:n]) > rtol
    bad |= relerr(g.s[:n], o.s[:n], satol) > rtol
    bad |= g.active[:n] != o.active[:n]
    return bad


def attaching_table(uniform_sharing: bool):
    """Synthetic gas 1 with attachment raised to 3e-20 m^2 below 5 eV, so that removals (and
    the sub-stepping of removed electrons) happen often in a few steps."""
    recs = lxcat.synthetic_records(1, uniform_sharing=uniform_sharing)
    for r in recs:
        if r["kind"] == "ATTACHMENT":
            r["data"] = [[e, 3e-20 if e < 5.0 else 0.0] for e, _ in r["data"]]
    return lxcat.load_lxcat_records(recs, {"SYN": lxcat.SYNTHETIC_DENSITY}, lxcat.DEFAULT_ENERGY)


def serial_run(rt, p, efield, dt, seed, tracker=None, steps=1):
    """Run the restatement with one serial uniform stream (numpy's generator, values in
    (0, 1]) and record every slot's draws per step: the injected-uniform input."""
    gen = np.random.default_rng(seed)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 16 * len(p.w))
    per_step = []
    for _ in range(steps):
        recs = {}

        def draws(i):
            recs[i] = R.CountingSource(lambda: 1.0 - gen.random())
            return recs[i]
        n = rp.n
        R.advance(rp, rt, efield, dt, tracker=tracker, draws=draws)
        per_step.append([recs[i].values if i in recs else [] for i in range(n)])
    return rp, per_step
