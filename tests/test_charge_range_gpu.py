"""The int64 fixed-point charge range (2^-32 e units) is guarded: a particle charge of 2^30 e
or more, or a cell sum of 2^30 e or more, is reported as MCS_ERR_CHARGE_RANGE instead of
wrapping silently (density!, MCStreamer/src/poisson.jl:65-84; the tracker,
gridfields.jl:198-224; the charge poisson! assembles, poisson.jl:17-26)."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import jumc, lxcat, streamer
from mcstreamer_b200.poisson import MGConfig, PoissonSolver
from tests.helpers import broad

R, LEN, M, N = 1e-4, 2e-4, 16, 32


def _pop(ctx, tab, w, n=64):
    p = broad(n, 1)
    p.x[:, 0] = 0.3 * R
    p.x[:, 1] = 0.0
    p.x[:, 2] = 0.5 * LEN
    p.w[:] = w
    return jumc.Population(128, p, tab, precision="fp64")


@pytest.mark.gpu
def test_particle_charge_beyond_range_is_reported(ctx):
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    pop = _pop(ctx, tab, 2e9)          # above 2^30 e
    grid.zero(L.Q_PART)
    with pytest.raises(L.MCSError) as e:
        streamer.density(grid, pop, 1.0)
        ctx.sync()
    assert e.value.code == L.ERR_CHARGE_RANGE
    assert grid.read_fixed(L.Q_PART).sum() == 0      # nothing wrapped into the cells
    pop.close()
    # below the bound: deposited exactly (the cell holds 2 x 1e9 e, under its 2^31 e)
    pop = _pop(ctx, tab, 1e9, n=2)
    streamer.density(grid, pop, 1.0)
    ctx.sync()
    assert grid.read_fixed(L.Q_PART).sum() == 2 * round(1e9 * 2 ** 32)
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_cell_sum_near_wrapping_is_reported_by_poisson(ctx):
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    solver = PoissonSolver(grid, MGConfig(levels=3))
    q = np.zeros((M + 2) * (N + 2), dtype=np.int64)
    q[5 + 7 * (M + 2)] = -(1 << 62)
    grid.write_fixed(L.Q_FIXED, q)
    grid.zero(L.Q_PART)
    with pytest.raises(L.MCSError) as e:
        solver.run(-1e6)
    assert e.value.code == L.ERR_CHARGE_RANGE
    q[5 + 7 * (M + 2)] = -(1 << 61)
    grid.write_fixed(L.Q_FIXED, q)
    solver.run(-1e6)
    solver.close(); grid.close()
