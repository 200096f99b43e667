"""Cell-key radix sort and per-cell resampling (resample!, MCStreamer/src/resample.jl:7-84)
against the CPU oracle, which restates the reference's serial passes on the population
sorted with a stable sort (so both append clones in the same order)."""
import numpy as np
import pytest

from mcstreamer_b200 import jumc, lxcat, streamer
from oracle import pyoracle as po
from tests.helpers import broad, oracle_arrays, oracle_pop

NX, NY, NZ, H = 8, 8, 16, 4e-6
CENTRE = (NX * H / 2, NY * H / 2, NZ * H / 2)


def _cloud(n, seed, spread=5e-6, weights="int"):
    p = broad(n, seed, emax_ev=10.0, x0=CENTRE, spread=spread)
    rng = np.random.default_rng(seed + 1)
    u = 10 ** rng.uniform(0, 3, n)
    if weights == "int":
        p.w[:] = np.rint(u)                # integer weights 1..1000 (splits need w > 2)
    elif weights == "dyadic":
        p.w[:] = np.rint(u * 2 ** 20) / 2 ** 20   # 20 fraction bits: merges take the exact warp sums
    else:
        p.w[:] = u                         # full FP64 mantissas: merges take the serial pass
    p.active[rng.random(n) < 0.05] = 0
    return p


def _setup(ctx, n, precision="fp64", mesh=False, seed=7, capf=4, weights="int"):
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.Grid3D(NX, NY, NZ, H, precision=precision, ctx=ctx)
    p0 = _cloud(n, seed, weights=weights)
    pop = jumc.Population(capf * n, p0, tab, precision=precision, seed=seed, mesh=grid if mesh else None)
    ofield = po.field_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0), np.zeros(3 * (NX + 1) * (NY + 1) * (NZ + 1)))
    return tab, grid, p0, pop, ofield


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", [False, True])
def test_sort_is_stable_by_cell(ctx, mesh):
    n = 200_000
    tab, grid, p0, pop, ofield = _setup(ctx, n, mesh=mesh)
    ctx.check(ctx.lib.mcs_sort_cells(pop.h, grid.h_))
    g = pop.download()
    key = np.where(p0.active == 1, grid.cell_key(p0.x), np.iinfo(np.int64).max)
    order = np.argsort(key, kind="stable")
    np.testing.assert_array_equal(g.active, p0.active[order])
    np.testing.assert_array_equal(g.s, p0.s[order])
    np.testing.assert_array_equal(g.w, p0.w[order])
    if not mesh:
        np.testing.assert_array_equal(g.x, p0.x[order])
    # the oracle's restated sort gives the same permutation
    op = oracle_pop(p0, n, 0)
    po.sort_cells(op, ofield)
    o = oracle_arrays(op)
    np.testing.assert_array_equal(g.s, o.s)
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
@pytest.mark.parametrize("ntarget,nmax,weights", [(10, 15, "int"), (64, 96, "int"), (20, 15, "int"),
                                                  (200, 300, "int"), (64, 96, "dyadic"), (64, 96, "real")])
def test_resample_cells_matches_oracle(ctx, ntarget, nmax, weights):
    """Integer and dyadic weights take the merge cells' exact warp sums, full FP64
    mantissas the serial pass; (20, 15) and (200, 300) take the thread-per-cell form."""
    n = 150_000
    tab, grid, p0, pop, ofield = _setup(ctx, n, mesh=False, weights=weights)
    w0 = p0.w[p0.active == 1].sum()
    ctx.check(ctx.lib.mcs_resample_cells(pop.h, grid.h_, ntarget, nmax))
    g = pop.download()
    op = oracle_pop(p0, 4 * n, 7)
    po.sort_cells(op, ofield)
    assert po.resample_cells(op, ofield, ntarget, nmax, 0) == 0
    o = oracle_arrays(op)
    assert g.n == o.n and g.n > n
    np.testing.assert_array_equal(g.active, o.active)
    np.testing.assert_array_equal(g.x, o.x)
    np.testing.assert_allclose(g.w, o.w, rtol=1e-12)
    # resample! conserves the total weight (main.jl:303-304 asserts rtol 1e-5) when
    # ntarget <= nmax; with ntarget > nmax a cell that splits past nmax falls into the
    # merge branch with x = 0 (resample.jl:31-76), in the reference as here
    w1 = g.w[g.active == 1].sum()
    if ntarget <= nmax:
        assert w1 == pytest.approx(w0, rel=1e-9)
    # overfull cells are left with at most ntarget equal-weight particles
    keys = grid.cell_key(g.x[g.active == 1])
    _, counts = np.unique(keys[keys < np.iinfo(np.int64).max], return_counts=True)
    if ntarget <= nmax:
        assert counts.max() <= max(ntarget, nmax)
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_resample_cells_mesh_fp32_conserves_weight(ctx):
    n = 150_000
    tab, grid, p0, pop, ofield = _setup(ctx, n, precision="fp32", mesh=True)
    w0 = p0.w[p0.active == 1].astype(np.float32).astype(np.float64).sum()
    ctx.check(ctx.lib.mcs_resample_cells(pop.h, grid.h_, 64, 96))
    g = pop.download()
    w1 = g.w[g.active == 1].sum()
    assert w1 == pytest.approx(w0, rel=1e-5)
    op = oracle_pop(p0, 4 * n, 7)
    po.sort_cells(op, ofield)
    po.resample_cells(op, ofield, 64, 96, 0)
    assert abs(g.n - op.n) <= 0.01 * (op.n - n) + 8
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
@pytest.mark.parametrize("weights", ["real", "int"])
def test_resample_cells_fp32_matches_oracle_bitwise(ctx, weights):
    """An FP32 population whose inputs are FP32 values: the sort keys, the FP64 weight sums,
    the selections and the splits are the oracle's, so every stored value equals the
    oracle's FP64 result rounded to FP32 (clone weights wtotal / ntarget; a split particle
    keeps w - round(w / 2), which FP32 holds exactly)."""
    n = 150_000
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.Grid3D(NX, NY, NZ, H, precision="fp32", ctx=ctx)
    p0 = _cloud(n, 11, weights=weights)
    for a in (p0.x, p0.v, p0.w, p0.s):
        a[...] = a.astype(np.float32).astype(np.float64)
    pop = jumc.Population(4 * n, p0, tab, precision="fp32", seed=11)
    ofield = po.field_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0), np.zeros(3 * (NX + 1) * (NY + 1) * (NZ + 1)))
    ctx.check(ctx.lib.mcs_resample_cells(pop.h, grid.h_, 64, 96))
    g = pop.download()
    op = oracle_pop(p0, 4 * n, 11)
    po.sort_cells(op, ofield)
    assert po.resample_cells(op, ofield, 64, 96, 0) == 0
    o = oracle_arrays(op)
    assert g.n == o.n and g.n > n
    np.testing.assert_array_equal(g.active, o.active)
    for name in ("x", "v", "w", "s"):
        np.testing.assert_array_equal(getattr(g, name), getattr(o, name).astype(np.float32).astype(np.float64),
                                      err_msg=name)
    pop.close(); grid.close(); tab.close()
