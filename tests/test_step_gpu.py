"""Per-particle parity of the electron step (advance!, collisions!) against the CPU oracle.

Both sides consume identical Philox uniforms (one block per collision event, keyed by slot,
step and event number), so a single step matches the FP64 oracle per particle (rel 1e-12 in
FP64 mode) and, in FP32 mode, within rel 1e-5 except for particles whose discrete decisions
flip (counted and bounded).
"""
import numpy as np
import pytest

from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat
from oracle import pyoracle as po
from tests.helpers import broad, maxwellian, oracle_arrays, oracle_pop, particle_mismatch, relerr

E100TD = 100 * co.Td * 2.5e25
RTOL64 = 1e-12
RTOL32 = 1e-5


def _setup(ctx, n, variant=0, uniform_sharing=True, precision="fp64", seed=11, cap_factor=3, gen=broad, **kw):
    t = lxcat.synthetic_table(variant, uniform_sharing=uniform_sharing)
    tab = jumc.CollisionTable(t, ctx)
    p0 = gen(n, seed, **kw)
    pop = jumc.Population(cap_factor * n, p0, tab, precision=precision, seed=seed)
    otab = po.OracleTable.from_lxcat(t)
    opop = oracle_pop(p0, cap_factor * n, seed)
    return t, tab, p0, pop, otab, opop


def _close(*objs):
    for o in objs:
        o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("uniform_sharing", [False, True])
def test_advance_fp64_one_step_matches_oracle(ctx, uniform_sharing):
    n = 65536
    t, tab, p0, pop, otab, opop = _setup(ctx, n, uniform_sharing=uniform_sharing)
    fld = jumc.FixedField(5 * E100TD, ctx)
    dt = 4e-13
    jumc.advance(pop, fld, dt)
    assert po.advance(opop, otab, po.field_uniform(0, 0, 5 * E100TD), dt) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n, (g.n, o.n)
    assert g.n > n, "no ionization happened; the test needs secondaries"
    bad = particle_mismatch(g, o, RTOL64, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0, f"{bad.sum()} of {g.n} slots differ; worst x {relerr(g.x, o.x).max():.3g}"
    _close(pop, fld, tab)


@pytest.mark.gpu
def test_advance_fp64_multistep_matches_oracle(ctx):
    n = 8192
    t, tab, p0, pop, otab, opop = _setup(ctx, n, gen=maxwellian, mean_ev=5.0, cap_factor=4)
    fld = jumc.FixedField(3 * E100TD, ctx)
    of = po.field_uniform(0, 0, 3 * E100TD)
    for _ in range(20):
        jumc.advance(pop, fld, 1e-13)
        assert po.advance(opop, otab, of, 1e-13) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n
    assert (o.active == 0).sum() > 0, "no attachment happened; the test needs removals"
    bad = particle_mismatch(g, o, 1e-11, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0, f"{bad.sum()} slots differ"
    assert pop.step == 20
    _close(pop, fld, tab)


@pytest.mark.gpu
def test_advance_fp32_one_step_within_tolerance(ctx):
    n = 65536
    t, tab, p0, pop, otab, opop = _setup(ctx, n, precision="fp32")
    fld = jumc.FixedField(5 * E100TD, ctx)
    dt = 2e-13
    jumc.advance(pop, fld, dt)
    assert po.advance(opop, otab, po.field_uniform(0, 0, 5 * E100TD), dt) == 0
    g, o = pop.download(), oracle_arrays(opop)
    # parents: compare per slot; discrete flips (process choice, sub-step count) are counted
    bad = particle_mismatch(g, o, RTOL32, xatol=1e-12, vatol=1e-2, satol=1e-5, n=n)
    frac = bad.sum() / n
    assert frac < 2e-3, f"flip fraction {frac:.2e}"
    assert abs(g.n - o.n) <= max(8, 0.01 * (o.n - n))
    _close(pop, fld, tab)


@pytest.mark.gpu
def test_collisions_fixed_step_matches_oracle(ctx):
    n = 32768
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=5)
    dt = 3e-14
    for _ in range(3):
        jumc.collisions(pop, dt)
        assert po.collisions(opop, otab, dt) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n
    bad = particle_mismatch(g, o, RTOL64, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0
    _close(pop, tab)


@pytest.mark.gpu
def test_secondaries_follow_parent_order(ctx):
    """Appended secondaries are in ascending (parent slot, event #): the serial order."""
    n = 20000
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=3)
    fld = jumc.FixedField(8 * E100TD, ctx)
    jumc.advance(pop, fld, 5e-13)
    assert po.advance(opop, otab, po.field_uniform(0, 0, 8 * E100TD), 5e-13) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n and g.n > n + 100
    np.testing.assert_allclose(g.x[n:], o.x[n:], rtol=1e-12, atol=1e-30)
    np.testing.assert_allclose(g.v[n:], o.v[n:], rtol=1e-12, atol=1e-30)
    np.testing.assert_array_equal(g.active[n:], o.active[n:])
    _close(pop, fld, tab)


@pytest.mark.gpu
def test_repack_matches_reference_permutation(ctx):
    n = 50000
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=9)
    rng = np.random.default_rng(1)
    p0.active[:] = (rng.random(n) < 0.6).astype(np.uint8)
    pop.upload(p0)
    opop = oracle_pop(p0, 3 * n, 9)
    jumc.repack(pop)
    po.repack(opop)
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n == int(p0.active.sum())
    np.testing.assert_array_equal(g.x, o.x)
    np.testing.assert_array_equal(g.v, o.v)
    np.testing.assert_array_equal(g.s, o.s)
    assert g.active.all()
    _close(pop, tab)


@pytest.mark.gpu
@pytest.mark.parametrize("frac", [0.5, 1.5, 40.0])
def test_swarm_resample_matches_oracle(ctx, frac):
    from mcstreamer_b200 import swarm
    n = 40000
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=4, cap_factor=60)
    n0 = int(n * frac)
    swarm.resample(pop, n0, 0.1)
    assert po.swarm_resample(opop, n0, 0.1) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n
    np.testing.assert_array_equal(g.active, o.active)
    np.testing.assert_array_equal(g.x, o.x)
    np.testing.assert_array_equal(g.s, o.s)
    _close(pop, tab)


@pytest.mark.gpu
def test_moments_match_oracle(ctx):
    n = 30000
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=2, spread=1e-4)
    p0.active[::7] = 0
    pop.upload(p0)
    opop = oracle_pop(p0, 3 * n, 2)
    m = pop.moments(tab)
    mo = po.moments(opop, otab)
    np.testing.assert_allclose(m, mo, rtol=1e-12, atol=1e-300)
    _close(pop, tab)


@pytest.mark.gpu
def test_energy_out_of_table_is_reported(ctx):
    n = 64
    t, tab, p0, pop, otab, opop = _setup(ctx, n, seed=1)
    p0.v[:] = 0.0
    p0.v[:, 2] = np.sqrt(2 * 1500 * co.eV / co.electron_mass)   # 1500 eV > table max
    p0.s[:] = 1e-3                                              # collide immediately
    pop.upload(p0)
    fld = jumc.FixedField(0.0, ctx)
    with pytest.raises(Exception) as ei:
        jumc.advance(pop, fld, 1e-13)
        ctx.sync()
    assert "ENERGY_RANGE" in str(ei.value)
    ctx.sync()   # status was cleared
    _close(pop, fld, tab)
