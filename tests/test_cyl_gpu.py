"""The reference's own streamer geometry: cylindrical Grid(R, L, M, N) with the staggered
bilinear FieldInterp (MCStreamer/src/gridfields.jl:115-190), NGP density!
(poisson.jl:65-84) and the CollisionTracker (gridfields.jl:198-224), against the oracle."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import jumc, lxcat, streamer
from oracle import pyoracle as po
from tests.helpers import broad, oracle_arrays, oracle_pop, particle_mismatch

R, LEN, M, N = 1e-4, 2e-4, 24, 48


def _faces():
    i = np.arange(M + 3)[:, None] / M
    j = np.arange(N + 3)[None, :] / N
    er = 2e6 * i * (1 - 0.3 * j) + 1e5 * np.sin(7 * j)
    ez = -1.5e7 + 3e6 * np.cos(3 * i) * j
    return er, ez


def _particles(n, seed):
    p = broad(n, seed, emax_ev=80.0)
    rng = np.random.default_rng(seed)
    r = R * np.sqrt(rng.random(n)) * 0.98
    th = 2 * np.pi * rng.random(n)
    p.x[:, 0] = r * np.cos(th)
    p.x[:, 1] = r * np.sin(th)
    p.x[:, 2] = LEN * (0.02 + 0.96 * rng.random(n))
    return p


@pytest.mark.gpu
def test_cyl_step_with_tracker_matches_oracle(ctx):
    n = 40_000
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    er, ez = _faces()
    grid.set_efield(er, ez)
    p0 = _particles(n, 31)
    pop = jumc.Population(3 * n, p0, tab, precision="fp64", seed=31)
    fld = streamer.FieldInterp(grid)
    grid.zero(L.Q_FIXED)
    ofield = po.field_cyl(R, LEN, M, N, er.T.ravel(), ez.T.ravel())
    otrk = po.tracker_cyl(R, LEN, M, N)
    opop = oracle_pop(p0, 3 * n, 31)
    for _ in range(3):
        jumc.advance(pop, fld, 3e-13, streamer.CollisionTracker(grid))
        assert po.advance(opop, po.OracleTable.from_lxcat(t), ofield, 3e-13, tracker=otrk) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n and g.n > n
    bad = particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0, f"{bad.sum()} slots differ"
    qf = grid.read_density(L.Q_FIXED)
    qo = otrk._q.reshape(N + 2, M + 2).T
    np.testing.assert_allclose(qf, qo, rtol=1e-12, atol=1e-6 * np.abs(qo).max())
    assert np.abs(qo).sum() > 0
    fld.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_cyl_density_matches_oracle(ctx):
    n = 100_000
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    p0 = _particles(n, 5)
    p0.w[:] = np.rint(10 ** np.random.default_rng(1).uniform(0, 3, n))
    p0.x[::50, 2] = 1.2 * LEN                        # some outside: skipped like checkbounds
    pop = jumc.Population(n, p0, tab, precision="fp64")
    grid.zero(L.Q_PART)
    streamer.density(grid, pop, -1.0)
    q = grid.read_density(L.Q_PART)
    otrk = po.tracker_cyl(R, LEN, M, N)
    po.deposit(oracle_pop(p0, n, 0), otrk, -1.0)
    qo = otrk._q.reshape(N + 2, M + 2).T
    np.testing.assert_allclose(q, qo, rtol=1e-12, atol=0)
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_cyl_field_too_high_is_reported(ctx):
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    er, ez = _faces()
    grid.set_efield(er, ez * 100.0)                  # |E| > 1e8 V/m (gridfields.jl:179-187)
    p0 = _particles(256, 2)
    pop = jumc.Population(1024, p0, tab, precision="fp64")
    fld = streamer.FieldInterp(grid)
    with pytest.raises(Exception) as ei:
        jumc.advance(pop, fld, 1e-14)
        ctx.sync()
    assert "FIELD_TOO_HIGH" in str(ei.value)
    fld.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_cyl_step_fp32_within_tolerance(ctx):
    """The FP32 push gathers from FP32 copies of the faces: one step against the FP64 oracle
    within single-precision tolerance, discrete flips (process choice, sub-step count) counted."""
    n = 65_536
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    er, ez = _faces()
    grid.set_efield(er, ez)
    p0 = _particles(n, 17)
    pop = jumc.Population(3 * n, p0, tab, precision="fp32", seed=17)
    fld = streamer.FieldInterp(grid)
    ofield = po.field_cyl(R, LEN, M, N, er.T.ravel(), ez.T.ravel())
    opop = oracle_pop(p0, 3 * n, 17)
    try:
        jumc.advance(pop, fld, 2e-13)
        assert po.advance(opop, po.OracleTable.from_lxcat(t), ofield, 2e-13) == 0
        g, o = pop.download(), oracle_arrays(opop)
        bad = particle_mismatch(g, o, 1e-5, xatol=1e-12, vatol=1e-2, satol=1e-5, n=n)
        assert bad.sum() / n < 2e-3, f"flip fraction {bad.sum() / n:.2e}"
        assert abs(g.n - o.n) <= max(8, 0.01 * (o.n - n))
    finally:
        fld.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_cyl_field_too_high_is_reported_fp32(ctx):
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    er, ez = _faces()
    grid.set_efield(er, ez * 100.0)
    pop = jumc.Population(1024, _particles(256, 2), tab, precision="fp32")
    fld = streamer.FieldInterp(grid)
    try:
        with pytest.raises(Exception) as ei:
            jumc.advance(pop, fld, 1e-14)
            ctx.sync()
        assert "FIELD_TOO_HIGH" in str(ei.value)
    finally:
        fld.close(); pop.close(); grid.close(); tab.close()
