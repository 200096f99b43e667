"""The device path against the committed golden fixtures of tests/golden/ (written by
tests/golden/make_golden.py from the oracle): one FP64 step, Swarm.resample! and repack!,
the cell sort and resample!, and the int64 CIC deposit."""
import json
from pathlib import Path

import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, streamer, swarm
from tests.helpers import vec_relerr

GOLDEN = Path(__file__).resolve().parent / "golden"


def _load(name):
    return json.loads((GOLDEN / name).read_text())


def _pa(d):
    return jumc.ParticleArrays(np.array(d["x"]), np.array(d["v"]), np.array(d["w"]), np.array(d["s"]),
                               np.array(d["active"], np.uint8))


def _same(got, want):
    assert got.n == want.n
    for f in ("x", "v", "w", "s", "active"):
        np.testing.assert_array_equal(getattr(got, f), getattr(want, f))


@pytest.mark.gpu
def test_device_step_matches_golden(ctx):
    g = _load("step_fp64.json")
    t = lxcat.load_lxcat_records(lxcat.synthetic_records(0, uniform_sharing=False), {"SYN": 2.5e25},
                                 lxcat.EnergyGrid(0.0, 1000 * co.eV, g["neps"]))
    tab = jumc.CollisionTable(t, ctx)
    p = _pa(g["input"])
    pop = jumc.Population(4 * p.n, p, tab, precision="fp64", seed=g["seed"])
    fld = jumc.FixedField(g["ez"], ctx)
    ctx.check(ctx.lib.mcs_advance(pop.h, tab.h, fld.h, g["dt"], None))
    got, want = pop.download(), _pa(g["output"])
    assert got.n == want.n
    assert vec_relerr(got.x, want.x).max() < 1e-12
    assert vec_relerr(got.v, want.v).max() < 1e-12
    np.testing.assert_array_equal(got.w, want.w)
    np.testing.assert_array_equal(got.active, want.active)
    np.testing.assert_allclose(got.s, want.s, rtol=1e-12)
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_device_swarm_resample_and_repack_match_golden(ctx):
    g = _load("swarm_resample.json")
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    pop = jumc.Population(g["cap"], _pa(g["input"]), tab, precision="fp64", seed=g["seed"], step=g["step"])
    swarm.resample(pop, g["n0"][0], 0.1)
    _same(pop.download(), _pa(g["after_clone"]))
    swarm.resample(pop, g["n0"][1], 0.1)
    _same(pop.download(), _pa(g["after_drop"]))
    ctx.check(ctx.lib.mcs_repack(pop.h))
    _same(pop.download(), _pa(g["after_repack"]))
    pop.close(); tab.close()


@pytest.mark.gpu
def test_device_resample_cells_matches_golden(ctx):
    g = _load("resample_cells.json")
    nx, ny, nz, h = g["mesh"]
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.Grid3D(nx, ny, nz, h, precision="fp64", ctx=ctx)
    pop = jumc.Population(g["cap"], _pa(g["input"]), tab, precision="fp64", seed=g["seed"])
    ctx.check(ctx.lib.mcs_resample_cells(pop.h, grid.h_, g["ntarget"], g["nmax"]))
    _same(pop.download(), _pa(g["output"]))
    pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_deposit_matches_golden(ctx, precision):
    """int64 CIC at 2^-32 e: the fixture's node charges exactly from FP64 positions.  FP32
    positions move the corner shares slightly, so FP32 is held to the exact total (each
    particle deposits exactly llrint(w val 2^32)) and a per-node bound."""
    g = _load("deposit_cic.json")
    nx, ny, nz, h = g["mesh"]
    x, w = np.array(g["x"]), np.array(g["w"])
    n = len(w)
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.Grid3D(nx, ny, nz, h, precision=precision, ctx=ctx)
    pop = jumc.Population(n, jumc.ParticleArrays(x, np.zeros((n, 3)), w, np.ones(n), np.ones(n, np.uint8)), tab,
                          precision=precision, seed=0)
    grid.zero(L.Q_PART)
    streamer.density(grid, pop, g["val"])
    q = grid.read_fixed(L.Q_PART)
    want = np.zeros(g["n_nodes"], np.int64)
    want[g["nodes"]] = g["q"]
    if precision == "fp64":
        np.testing.assert_array_equal(q, want)
    else:
        assert q.sum() == want.sum()
        assert np.abs(q - want).max() < 2**32 * 1e-3 * np.abs(g["val"]) * w.max()
    pop.close(); grid.close(); tab.close()
