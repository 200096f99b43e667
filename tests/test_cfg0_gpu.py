"""The plain swarm workload (Swarm.swarm, Swarm/src/Swarm.jl:102-173) at 100 Td on a reduced
step count: every coefficient of Swarm.jl:144-161 -- drift W, D_L, D_T, mean energy, k_ion,
nu, alpha, eta -- from FP32 device runs against FP64 runs of the CPU oracle.

* FP64 device runs follow the oracle's trajectories seed for seed (same draws, FP64
  arithmetic): every coefficient agrees to rel 1e-9 after 400 steps.
* FP32 device runs are statistically equivalent: each coefficient's replica mean lies within
  3 sigma (the replica standard errors of both sides combined) of the oracle's.
"""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, swarm
from oracle import pyoracle as po

N0, EN, DENS, DT, NT = 16384, 100.0, 2.5e25, 1e-13, 400
KEYS = ("drift", "diffusion_l", "diffusion_t", "mean_energy", "k_ion", "nu", "alpha", "eta")


def row(r, proc):
    ion = [j for j, p in enumerate(proc) if p.kind in (L.IONIZATION, L.IONIZATION_UNIFORM)][0]
    d = {k: getattr(r, k) for k in ("drift", "diffusion_l", "diffusion_t", "mean_energy", "nu", "alpha", "eta")}
    d["k_ion"] = float(r.k[ion]) / DENS
    return d


def oracle_run(t, seed):
    ot = po.OracleTable.from_lxcat(t)
    eb = EN * co.Td * DENS
    p = swarm.initial_particles(N0, "maxwellian", seed)
    op = po.OraclePop(p.x, p.v, p.w, p.s, p.active, cap=4 * N0, seed=seed)
    mom, fin = po.swarm_run(op, ot, po.field_uniform(0, 0, eb), DT, NT, N0, 0.1, 1)
    return swarm.coefficients(EN, eb, DT, mom, fin, t.proc)


@pytest.mark.gpu
def test_cfg0_coefficients_fp32_within_3_sigma_of_the_fp64_oracle(ctx):
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    dev = {prec: [row(swarm.swarm_one(tab, EN, DENS, N0, DT, NT, maxp=4 * N0, precision=prec, seed=s,
                                      init="maxwellian"), t.proc) for s in range(8)] for prec in ("fp32", "fp64")}
    orc = [row(oracle_run(t, s), t.proc) for s in range(4)]
    for s in range(4):
        for k in KEYS:
            a, b = dev["fp64"][s][k], orc[s][k]
            assert abs(a - b) <= 1e-9 * max(abs(b), 1e-300), f"seed {s} {k}: device FP64 {a} vs oracle {b}"
    for k in KEYS:
        a = np.array([r[k] for r in dev["fp32"]])
        b = np.array([r[k] for r in orc])
        e = np.hypot(3 * a.std(ddof=1) / np.sqrt(len(a)), 3 * b.std(ddof=1) / np.sqrt(len(b)))
        assert abs(a.mean() - b.mean()) <= e, f"{k}: FP32 {a.mean():.6g} vs oracle {b.mean():.6g} (3 sigma {e:.3g})"
    assert np.mean([r["k_ion"] for r in orc]) > 0 and np.mean([r["eta"] for r in orc]) > 0
    tab.close()
