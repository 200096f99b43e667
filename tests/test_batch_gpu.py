"""Batched swarms: every instance of a batch evolves exactly as the same swarm run alone
(mcs_swarm_run with repack_every = 1, FP32), whatever else shares the batch, whichever
kernel shape runs it, with or without the CUDA graph, and when it joins mid-run."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, swarm
from mcstreamer_b200.batch import BatchedSwarms, Solve, SwarmBatch

DENS = 2.5e25
DT = 1e-13


def _cases():
    # (table variant, E/N in Td, seed, n0, capacity)
    return [(1, 300.0, 3, 3000, 12000), (0, 120.0, 5, 1500, 6000), (1, 600.0, 7, 5000, 20000),
            (2, 80.0, 9, 700, 4000)]


def _alone(ctx, tab, en, seed, n0, cap, nt):
    p0 = swarm.initial_particles(n0, "maxwellian", seed, mean_ev=4.0)
    pop = jumc.Population(cap, p0, tab, precision="fp32", seed=seed)
    fld = jumc.FixedField(en * co.Td * DENS, ctx)
    mom = np.zeros((nt, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_swarm_run(pop.h, tab.h, fld.h, DT, nt, n0, 0.1, 1, L.dptr(mom)))
    out = pop.download()
    fld.close(); pop.close()
    return out, mom


def _add(b, tab, en, seed, n0, cap):
    p0 = swarm.initial_particles(n0, "maxwellian", seed, mean_ev=4.0)
    return b.add(tab, en * co.Td * DENS, seed, n0, cap, p0)


def _same(a, b):
    assert a.n == b.n
    np.testing.assert_array_equal(a.active, b.active)
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.v, b.v)
    np.testing.assert_array_equal(a.w, b.w)
    np.testing.assert_array_equal(a.s, b.s)


@pytest.fixture(scope="module")
def tables(ctx):
    tabs = {v: jumc.CollisionTable(lxcat.synthetic_table(v), ctx) for v in (0, 1, 2)}
    yield tabs
    for t in tabs.values():
        t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_batched_instances_equal_alone(ctx, tables, graph):
    nt = 40
    cases = _cases()
    with SwarmBatch(ctx, 8, 64000) as b:
        slots = [_add(b, tables[v], en, seed, n0, cap) for v, en, seed, n0, cap in cases]
        b.step(DT, nt, graph=graph)
        n, steps = b.state()
        for (v, en, seed, n0, cap), k in zip(cases, slots):
            alone, mom = _alone(ctx, tables[v], en, seed, n0, cap, nt)
            got = b.download(k)
            _same(got, alone)
            assert steps[k] == nt
            log = b.read_log(k, nt)
            np.testing.assert_array_equal(log[:, L.S_COUNT], mom[:, L.S_COUNT])
            np.testing.assert_allclose(log[:, :L.STEP_MOMENTS], mom, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_same_tiles_give_identical_sums(ctx, tables):
    """With the single path's tile (256 threads x 2 particles) the per-step sums are reduced
    in the same order, so they are bit-identical too."""
    nt = 30
    v, en, seed, n0, cap = _cases()[0]
    alone, mom = _alone(ctx, tables[v], en, seed, n0, cap, nt)
    with SwarmBatch(ctx, 2, 2 * cap) as b:
        b.set_variant(5)
        assert SwarmBatch.variant_shape(5) == (256, 2)
        k = _add(b, tables[v], en, seed, n0, cap)
        b.step(DT, nt)
        _same(b.download(k), alone)
        np.testing.assert_array_equal(b.read_log(k, nt)[:, :L.STEP_MOMENTS], mom)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 3, 8, 11, 12, 14, 16, 17])
def test_kernel_shape_does_not_change_result(ctx, tables, variant):
    nt = 25
    v, en, seed, n0, cap = _cases()[2]
    alone, mom = _alone(ctx, tables[v], en, seed, n0, cap, nt)
    with SwarmBatch(ctx, 2, 2 * cap) as b:
        b.set_variant(variant)
        k = _add(b, tables[v], en, seed, n0, cap)
        b.step(DT, nt)
        _same(b.download(k), alone)
        log = b.read_log(k, nt)
        np.testing.assert_array_equal(log[:, L.S_COUNT], mom[:, L.S_COUNT])
        np.testing.assert_allclose(log[:, :L.STEP_MOMENTS], mom, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_join_and_leave_mid_run(ctx, tables):
    """Continuous batching: an instance that joins after others have stepped, and into the
    region another one left, still equals its run alone."""
    cases = _cases()
    with SwarmBatch(ctx, 4, 40000) as b:
        a = _add(b, tables[cases[0][0]], *cases[0][1:])
        c = _add(b, tables[cases[1][0]], *cases[1][1:])
        b.step(DT, 10)
        b.remove(a)
        d = _add(b, tables[cases[3][0]], *cases[3][1:])
        b.step(DT, 30)
        _same(b.download(c), _alone(ctx, tables[cases[1][0]], *cases[1][1:], 40)[0])
        _same(b.download(d), _alone(ctx, tables[cases[3][0]], *cases[3][1:], 30)[0])
        n, steps = b.state()
        assert steps[c] == 40 and steps[d] == 30


@pytest.mark.gpu
def test_autotune_restores_state(ctx, tables):
    nt = 20
    cases = _cases()[:3]
    with SwarmBatch(ctx, 4, 64000) as b:
        slots = [_add(b, tables[v], en, seed, n0, cap) for v, en, seed, n0, cap in cases]
        b.step(DT, 5)
        chosen, times = b.autotune(DT, trial_steps=2)
        assert 0 <= chosen < L.BATCH_VARIANTS and (times > 0).all()
        assert SwarmBatch.variant_shape(chosen)[0] in (128, 256, 512)
        b.step(DT, nt - 5)
        for (v, en, seed, n0, cap), k in zip(cases, slots):
            _same(b.download(k), _alone(ctx, tables[v], en, seed, n0, cap, nt)[0])


@pytest.mark.gpu
def test_capacity_overflow_is_an_error(ctx, tables):
    with SwarmBatch(ctx, 2, 2000) as b:
        # n0 above the region: Swarm.resample! clones past the capacity
        p0 = swarm.initial_particles(1800, "maxwellian", 3, mean_ev=4.0)
        b.add(tables[1], 300.0 * co.Td * DENS, 3, 4000, 1900, p0)
        with pytest.raises(L.MCSError) as e:
            b.step(DT, 5)
            b.sync()
        assert e.value.code == L.ERR_CAPACITY


@pytest.mark.gpu
def test_batched_solves_driver(ctx, tables):
    solves = [Solve(tables[v], en, seed, n0, 30, DENS, mean_ev=4.0, capacity=cap, tag=i)
              for i, (v, en, seed, n0, cap) in enumerate(_cases() * 2)]
    bs = BatchedSwarms(ctx, 3, 50000, DT, chunk=8)
    try:
        res = bs.run(solves, window=20)
    finally:
        bs.close()
    assert [r.tag for r in res] == list(range(len(solves)))
    for r, sv in zip(res, solves):
        _, mom = _alone(ctx, sv.table, sv.en_td, sv.seed, sv.n0, sv.capacity, sv.nt)
        np.testing.assert_array_equal(r.sums[:, L.S_COUNT], mom[:, L.S_COUNT])
        np.testing.assert_allclose(r.sums[:, :L.STEP_MOMENTS], mom, rtol=1e-12, atol=0)
        assert r.steps == 30


@pytest.mark.gpu
def test_device_maxwellian_join_equals_population_init(ctx, tables):
    nt, n, cap, seed, en = 15, 3000, 9000, 21, 500.0
    pop = jumc.Population(cap, None, tables[1], precision="fp32", seed=seed)
    pop.init_maxwellian(n, 2.0)
    fld = jumc.FixedField(en * co.Td * DENS, ctx)
    ctx.check(ctx.lib.mcs_swarm_run(pop.h, tables[1].h, fld.h, DT, nt, n, 0.1, 1, None))
    alone = pop.download()
    fld.close(); pop.close()
    with SwarmBatch(ctx, 2, cap) as b:
        k = b.add_maxwellian(tables[1], en * co.Td * DENS, seed, n, cap, n, 2.0)
        b.step(DT, nt)
        _same(b.download(k), alone)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_device_maxwellian_matches_restatement(ctx, tables, precision, rtol):
    """The device draw against a restatement from the oracle's Philox uniforms (INIT stream)."""
    from oracle import pyoracle as po
    n, seed, mean_ev = 512, 77, 3.0
    pop = jumc.Population(n, None, tables[0], precision=precision, seed=seed)
    pop.init_maxwellian(n, mean_ev)
    got = pop.download()
    pop.close()
    sigma = np.sqrt((2.0 / 3.0) * mean_ev * co.elementary_charge / co.electron_mass)
    u = np.array([[po.uniform(seed, i, 0, 3, k) for k in range(5)] for i in range(n)])
    r0, r1 = np.sqrt(-2.0 * np.log(u[:, 0])), np.sqrt(-2.0 * np.log(u[:, 2]))
    v = sigma * np.stack([r0 * np.cos(2 * np.pi * u[:, 1]), r0 * np.sin(2 * np.pi * u[:, 1]),
                          r1 * np.cos(2 * np.pi * u[:, 3])], axis=1)
    np.testing.assert_allclose(got.v, v, rtol=rtol, atol=rtol * sigma)
    np.testing.assert_allclose(got.s, -np.log(u[:, 4]), rtol=rtol, atol=0)
    assert (got.x == 0).all() and (got.w == 1).all() and (got.active == 1).all()


@pytest.mark.gpu
def test_many_tile_instances_equal_alone(ctx, tables):
    """Instances of hundreds of tiles each, ionizing: every tile's secondaries wait for the
    prefix of the instance's tiles before them (appended after the CTA's next tile), so the
    appends of one instance are spread over many CTAs at once.  Each instance still equals
    its run alone, slot for slot."""
    nt = 12
    cases = [(1, 600.0, 11, 600000, 1400000), (0, 300.0, 12, 420000, 900000), (2, 1000.0, 13, 250000, 600000)]
    with SwarmBatch(ctx, 4, 3000000) as b:
        slots = [_add(b, tables[v], en, seed, n0, cap) for v, en, seed, n0, cap in cases]
        b.step(DT, nt, graph=True)
        for (v, en, seed, n0, cap), k in zip(cases, slots):
            alone, mom = _alone(ctx, tables[v], en, seed, n0, cap, nt)
            _same(b.download(k), alone)
            log = b.read_log(k, nt)
            np.testing.assert_array_equal(log[:, L.S_COUNT], mom[:, L.S_COUNT])
