"""The device step fed the reference's own draw order (mcs_set_uniform_source).

A serial run of the independent restatement (oracle/jumc_ref.py, written from
JuMC/src/mixed_population.jl:24-54, collisions.jl:159-192, electron.jl:108-139, util.jl:4-17)
draws from one serial uniform stream, as a single-threaded run of the reference does; every
particle's draws of every step are recorded and injected into the device population, which
must then reproduce the serial run particle by particle: rel 1e-12 in FP64, rel 1e-5 in FP32.
The expected values come from the restatement, not from oracle.cpp."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, streamer
from mcstreamer_b200.jumc import ParticleArrays
from oracle import jumc_ref as R
from oracle import pyoracle as po
from tests.helpers import (attaching_table, broad, oracle_arrays, oracle_pop, particle_mismatch, serial_run)

EZ = 5 * 100 * co.Td * 2.5e25


def restated(rp: R.Population) -> ParticleArrays:
    x, v, w, s, a = rp.arrays()
    return ParticleArrays(x, v, w, s, a)


@pytest.mark.gpu
@pytest.mark.parametrize("uniform_sharing", [True, False])
def test_injected_fp64_fixed_field_replays_the_serial_run(ctx, uniform_sharing):
    t = attaching_table(uniform_sharing)
    rt = R.Table.from_lxcat(t)
    p = broad(1500, 3, emax_ev=60.0)
    rp, per_step = serial_run(rt, p, R.FixedField([0.0, 0.0, EZ]), 4e-13, 7, steps=3)
    tab = jumc.CollisionTable(t, ctx)
    fld = jumc.FixedField(EZ, ctx)
    pop = jumc.Population(16 * len(p.w), p, tab, precision="fp64", seed=3)
    for per in per_step:
        pop.set_uniforms(per)
        jumc.advance(pop, fld, 4e-13)
    g, o = pop.download(), restated(rp)
    assert g.n == o.n and o.n > len(p.w)
    bad = particle_mismatch(g, o, 1e-12)
    assert bad.sum() == 0, f"{bad.sum()} of {g.n} slots differ from the serial run"
    assert (o.active == 0).sum() > 5
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_injected_fp64_field_interp_and_tracker_replay_the_serial_run(ctx):
    """The reference's streamer geometry: FieldInterp on a grid whose step(grid.rc) is not
    R / M, and the CollisionTracker's qfixed density."""
    Rr, Ln, M, N = 3e-4, 7e-4, 24, 100
    i = np.arange(M + 3)[:, None] / M
    j = np.arange(N + 3)[None, :] / N
    er = 2e6 * i * (1 - 0.3 * j) + 1e5 * np.sin(7 * j)
    ez = -1.5e7 + 3e6 * np.cos(3 * i) * j
    p = broad(1200, 31, emax_ev=80.0)
    rng = np.random.default_rng(31)
    r = Rr * np.sqrt(rng.random(len(p.w))) * 0.98
    th = 2 * np.pi * rng.random(len(p.w))
    p.x[:, 0], p.x[:, 1] = r * np.cos(th), r * np.sin(th)
    p.x[:, 2] = Ln * (0.02 + 0.96 * rng.random(len(p.w)))
    t = lxcat.synthetic_table(0)
    rt = R.Table.from_lxcat(t)
    g = R.GridCyl(Rr, Ln, M, N)
    rtk = R.TrackerCyl(g)
    rp, per_step = serial_run(rt, p, R.FieldInterp(g, er, ez), 3e-13, 5, tracker=rtk, steps=2)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(Rr, Ln, M, N, ctx=ctx)
    grid.set_efield(er, ez)
    grid.zero(L.Q_FIXED)
    fld = streamer.FieldInterp(grid)
    pop = jumc.Population(16 * len(p.w), p, tab, precision="fp64", seed=31)
    for per in per_step:
        pop.set_uniforms(per)
        jumc.advance(pop, fld, 3e-13, streamer.CollisionTracker(grid))
    gd, o = pop.download(), restated(rp)
    assert gd.n == o.n and o.n > len(p.w)
    bad = particle_mismatch(gd, o, 1e-12)
    assert bad.sum() == 0, f"{bad.sum()} slots differ"
    qf = grid.read_density(L.Q_FIXED)
    qo = rtk.q.reshape(N + 2, M + 2).T
    assert np.abs(qo).sum() > 0
    np.testing.assert_allclose(qf, qo, rtol=1e-12, atol=1e-9 * np.abs(qo).max())
    fld.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_injected_fp32_within_tolerance(ctx):
    """FP32 push and sampling fed the same draws: rel 1e-5, a few discrete flips allowed."""
    t = attaching_table(True)
    rt = R.Table.from_lxcat(t)
    p = broad(4000, 5, emax_ev=60.0)
    rp, per_step = serial_run(rt, p, R.FixedField([0.0, 0.0, EZ]), 4e-13, 11, steps=1)
    tab = jumc.CollisionTable(t, ctx)
    fld = jumc.FixedField(EZ, ctx)
    pop = jumc.Population(16 * len(p.w), p, tab, precision="fp32", seed=5)
    pop.set_uniforms(per_step[0])
    jumc.advance(pop, fld, 4e-13)
    g, o = pop.download(), restated(rp)
    assert abs(g.n - o.n) <= max(2, o.n // 100)
    n = min(g.n, len(p.w))
    bad = particle_mismatch(g, o, 1e-5, xatol=1e-12, vatol=1e-2, satol=1e-5, n=n)
    assert bad.sum() <= max(4, n // 200), f"{bad.sum()} of {n} parents differ beyond rel 1e-5"
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_injected_uniforms_running_out_then_philox_again(ctx):
    """Too few values fail the step with MCS_ERR_UNIFORMS; switching back to the Philox
    streams gives the oracle's step again."""
    t = lxcat.synthetic_table(0)
    rt = R.Table.from_lxcat(t)
    p = broad(400, 2)
    _, per_step = serial_run(rt, p, R.FixedField([0.0, 0.0, EZ]), 4e-13, 2)
    tab = jumc.CollisionTable(t, ctx)
    fld = jumc.FixedField(EZ, ctx)
    pop = jumc.Population(8 * len(p.w), p, tab, precision="fp64", seed=2)
    pop.set_uniforms([a[:-1] for a in per_step[0]])
    with pytest.raises(L.MCSError) as e:
        jumc.advance(pop, fld, 4e-13)
        ctx.sync()
    assert e.value.code == L.ERR_UNIFORMS
    pop.close()
    pop = jumc.Population(8 * len(p.w), p, tab, precision="fp64", seed=2)
    pop.set_uniforms(per_step[0])
    pop.set_uniforms(None)
    jumc.advance(pop, fld, 4e-13)
    op = oracle_pop(p, 8 * len(p.w), 2)
    assert po.advance(op, po.OracleTable.from_lxcat(t), po.field_uniform(0, 0, EZ), 4e-13) == 0
    g, o = pop.download(), oracle_arrays(op)
    assert g.n == o.n
    assert particle_mismatch(g, o, 1e-12).sum() == 0
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_injected_uniforms_rejected_on_mesh_layout(ctx):
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.Grid3D(8, 8, 8, 4e-6, precision="fp32", ctx=ctx)
    pop = jumc.Population(1000, None, tab, precision="fp32", seed=1, mesh=grid)
    with pytest.raises(L.MCSError) as e:
        pop.set_uniforms([[0.5]])
    assert e.value.code == L.ERR_UNSUPPORTED
    pop.close(); grid.close(); tab.close()
