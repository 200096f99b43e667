"""Swarm runs (Swarm/src/Swarm.jl:48-186): the fused device loop against the oracle, an
analytic limit, and FP32 against FP64 coefficients within 3 sigma of the replica error."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, swarm
from oracle import pyoracle as po

DENS = 2.5e25


def _oracle_swarm(table, p0, cap, seed, ez, dt, nt, n0, tol=0.1):
    otab = po.OracleTable.from_lxcat(table)
    op = po.OraclePop(p0.x, p0.v, p0.w, p0.s, p0.active, cap=cap, seed=seed)
    f = po.field_uniform(0, 0, ez)
    rows = []
    for _ in range(nt):
        assert po.advance(op, otab, f, dt) == 0
        rows.append(po.moments(op)[:12])
        assert po.swarm_resample(op, n0, tol) == 0
    return np.array(rows), op


@pytest.mark.gpu
def test_swarm_loop_fp64_matches_oracle_every_step(ctx):
    t = lxcat.synthetic_table(1)         # ionization 12.1 eV, stronger attachment: resample fires
    tab = jumc.CollisionTable(t, ctx)
    n0, nt, dt, seed = 4096, 150, 1e-13, 3
    ez = 300 * co.Td * DENS
    p0 = swarm.initial_particles(n0, "maxwellian", seed, mean_ev=4.0)
    pop = jumc.Population(16 * n0, p0, tab, precision="fp64", seed=seed)
    fld = jumc.FixedField(ez, ctx)
    mom = np.zeros((nt, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_swarm_run(pop.h, tab.h, fld.h, dt, nt, n0, 0.1, 0, L.dptr(mom)))
    ref, op = _oracle_swarm(t, p0, 16 * n0, seed, ez, dt, nt, n0)
    np.testing.assert_array_equal(mom[:, L.S_COUNT], ref[:, 0])
    np.testing.assert_allclose(mom, ref, rtol=1e-10, atol=1e-300)
    assert pop.nparticles() == op.n
    assert len(set(mom[:, L.S_COUNT])) > 3           # the population changed size
    fld.close(); pop.close(); tab.close()


def _constant_frequency_gas(nu0, mass_ratio):
    """Elastic cross section sigma = nu0 / (N v): collision frequency nu0 at every energy."""
    e = lxcat.LOG_GRID_EV
    v = np.sqrt(2 * e * co.eV / co.electron_mass)
    rec = {"kind": "ELASTIC", "target": "M", "mass_ratio": mass_ratio, "comment": "Maxwell gas",
           "data": [[float(a), float(b)] for a, b in zip(e, nu0 / (DENS * v))]}
    return lxcat.load_lxcat_records([rec], {"M": DENS}, lxcat.EnergyGrid(0.0, 1000 * co.eV, 20001))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_constant_collision_frequency_drift(ctx, precision):
    """Momentum balance for a constant elastic collision frequency nu0:
    W = -(e/m) E (1 + mu) / nu0 (mean of v' = v_cm = mu/(1+mu) v per collision)."""
    nu0, mu = 4e12, 1e-3
    t = _constant_frequency_gas(nu0, mu)
    tab = jumc.CollisionTable(t, ctx)
    n0, nt, dt = 131072, 300, 5e-14
    E = 2e6
    p0 = swarm.initial_particles(n0, "maxwellian", 11, mean_ev=2.0)
    pop = jumc.Population(2 * n0, p0, tab, precision=precision, seed=11)
    fld = jumc.FixedField(E, ctx)
    mom = np.zeros((nt, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_swarm_run(pop.h, tab.h, fld.h, dt, nt, 0, 0.1, 0, L.dptr(mom)))
    W = mom[-100:, L.S_V + 2] / mom[-100:, L.S_COUNT]
    expect = -(co.elementary_charge / co.electron_mass) * E * (1 + mu) / nu0
    assert W.mean() == pytest.approx(expect, rel=0.02)
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_fp32_swarm_coefficients_within_3_sigma_of_fp64(ctx):
    """The FP32 form reproduces the FP64 swarm coefficients within 3 sigma of the replica
    standard error (Swarm.stats, Swarm.jl:253-269)."""
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    R, n0, nt, dt = 6, 32768, 600, 1e-13
    out = {}
    for prec in ("fp64", "fp32"):
        reps = [[swarm.swarm_one(tab, 300.0, DENS, n0, dt, nt, precision=prec, seed=100 + r, init="maxwellian")]
                for r in range(R)]
        out[prec] = swarm.stats(reps)
    for key in ("drift", "mean_energy", "diffusion_l", "diffusion_t"):
        a, b = out["fp64"][key][0], out["fp32"][key][0]
        se = np.hypot(out["fp64"][key + "_err"][0], out["fp32"][key + "_err"][0])
        assert abs(a - b) <= 3 * se + 1e-12 * abs(a), (key, a, b, se)
    tab.close()


@pytest.mark.gpu
def test_batched_fp32_coefficients_match_fp64(ctx):
    """The batched FP32 form against independent FP64 runs of the same swarms at three E/N:
    drift, mean energy and ionization rate agree within 3 sigma of the combined statistical
    error, and within 1 % wherever that error is below 0.5 %."""
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    ctx.set_flags(L.FLAG_CLAMP_ENERGY)
    try:
        res = swarm.fp32_batched_vs_fp64(ctx, tab, (300.0, 600.0, 1000.0), DENS, 131072, 600, 300, 1e-13)
    finally:
        ctx.set_flags(0)
        tab.close()
    for en, r in res.items():
        for key, (a32, e32, a64, e64) in r.items():
            err3 = np.hypot(e32, e64)
            assert abs(a32 - a64) <= err3 + 1e-12 * abs(a64), (en, key, a32, a64, err3)
            if err3 < 0.005 * abs(a64):
                assert abs(a32 - a64) <= 0.01 * abs(a64), (en, key, a32, a64)
    assert all(r["k"][2] > 0 for r in res.values())   # ionizing at every E/N tested


@pytest.mark.gpu
@pytest.mark.parametrize("lam", [0.4, 3.0, 12.5, 37.0])
def test_device_swarm_resample_clone_counts(ctx, lam):
    """Swarm.resample! on the device: per-particle clone counts equal the oracle's (same
    Philox streams, same inversion / PTRS sampler) and follow the Poisson law."""
    from tests.helpers import maxwellian, oracle_pop
    from tests.test_oracle import _clone_counts, _poisson_chi2_pvalue
    n = 20000
    p = maxwellian(n, 7)
    p.x[:, 0] = np.arange(n) * 1e-9 + 1e-6
    cap = int((lam + 2) * n) + 10 * n
    n0 = int(round(n * (1 + lam)))
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(cap, p, tab, precision="fp64", seed=11)
    swarm.resample(pop, n0, 0.1)
    got = _clone_counts(p, pop.download().x, n)
    pop.close(); tab.close()
    op = oracle_pop(p, cap, 11)
    po.swarm_resample(op, n0, 0.1)
    np.testing.assert_array_equal(got, _clone_counts(p, op.x[:op.n], n))
    assert _poisson_chi2_pvalue(got, (n0 - n) / n) > 1e-4
