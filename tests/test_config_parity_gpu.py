"""Parity on the streamer configurations' own meshes and fields, against the CPU oracle.

cfg1: 128x128x256 cells of 4 um; cfg2: 512x512x1024 cells of 2 um.  Both carry the
configurations' field -- the Gaussian charge (sigma 40 um, 1e20 e/m^3) at the mesh centre
plus -15 MV/m -- computed on the device, and 65,536 electrons drawn from the configuration's
own cloud (sigma 50 um, 1 eV, its weights).  The oracle steps the same electrons in the
field the device holds, read back over a window of nodes around the cloud (the whole cfg1
mesh; 192 cells a side for cfg2, whose 270M-node field does not fit host arrays in a test),
with the tracker and the particle deposit on the same window.  A step is advance! with the
CollisionTracker, then density!(qpart, -1) of the post-step electrons (one fused launch on
the device).
"""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import jumc, lxcat, streamer, workloads
from oracle import pyoracle as po
from tests.helpers import oracle_arrays, oracle_pop, particle_mismatch, vec_relerr


def _setup(ctx, name: str, precision: str, n: int, half: int):
    spec = workloads.streamer_spec(name)
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.Grid3D(spec.nx, spec.ny, spec.nz, spec.h, precision=precision, ctx=ctx)
    grid.set_efield_gaussian(spec.centre, workloads.CHARGE_SIGMA, workloads.CHARGE_PEAK, workloads.E_BACKGROUND)
    c = (spec.nx // 2, spec.ny // 2, spec.nz // 2)
    dims = (spec.nx, spec.ny, spec.nz)
    lo = tuple(max(0, ci - half) for ci in c)
    hi = tuple(min(d, ci + half) for ci, d in zip(c, dims))          # node indices, inclusive
    # the configuration's cloud, electrons at least 8 cells inside the window
    p = workloads.streamer_particles(workloads.streamer_spec(name, n=2 * n))
    u = p.x / spec.h
    keep = np.all((u >= np.array(lo) + 8) & (u < np.array(hi) - 8), axis=1)
    idx = np.nonzero(keep)[0][:n]
    p = jumc.ParticleArrays(p.x[idx], p.v[idx], p.w[idx], p.s[idx], p.active[idx])
    pop = jumc.Population(3 * len(idx), p, tab, precision=precision, seed=spec.seed, mesh=grid)
    e = grid.read_efield_box(lo, hi)
    nb = tuple(h - l for l, h in zip(lo, hi))                       # window cells
    origin = tuple(spec.h * l for l in lo)
    ofield = po.field_cart3d(*nb, spec.h, origin, e.reshape(-1))
    return spec, t, tab, grid, pop, ofield, lo, hi, nb, origin


@pytest.mark.gpu
@pytest.mark.parametrize("name,half", [("cfg1", 1 << 20), ("cfg2", 96)])
def test_config_mesh_step_fp64_matches_oracle(ctx, name, half):
    spec, t, tab, grid, pop, ofield, lo, hi, nb, origin = _setup(ctx, name, "fp64", 65536, half)
    n = pop.nparticles()
    opop = oracle_pop(pop.download(), 3 * n, spec.seed)   # positions as the device holds them
    otab = po.OracleTable.from_lxcat(t)
    trk = po.tracker_cart3d(*nb, spec.h, origin)
    fld = streamer.FieldInterp(grid)
    grid.zero(L.Q_FIXED)
    grid.zero(L.Q_PART)
    streamer.advance_deposit(pop, fld, spec.dt, streamer.CollisionTracker(grid), grid, -1.0)
    assert po.advance(opop, otab, ofield, spec.dt, tracker=trk) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n
    bad = particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0, f"{bad.sum()} slots differ, worst {vec_relerr(g.x, o.x).max():.3g}"
    # node totals are exact; a node's value may differ by the per-corner rounding of
    # fractions that differ at 1e-16 of a position (cell indices up to 1024, so ~1e-13 of a
    # cell): up to ~5 units of 2^-32 e per electron of weight 1e4 at the node -- 32 units where
    # few electrons meet, 1e-12 of the node's charge where many do
    def close(a, b):
        d = np.abs(a - b)
        bad = d > np.maximum(32, 1e-12 * np.abs(b))
        if bad.any():
            k = int(np.argmax(np.where(bad, d, -1)))
            print(f"worst node {k}: |diff| {d[k]}, value {b[k]}, {int(bad.sum())} nodes beyond the bound")
        return not bad.any()
    qf = grid.read_fixed_box(L.Q_FIXED, lo, hi)
    assert qf.sum() == trk._q.sum()
    assert close(qf, trk._q)
    qp = grid.read_fixed_box(L.Q_PART, lo, hi)
    dep = po.tracker_cart3d(*nb, spec.h, origin)
    po.deposit(opop, dep, -1.0)
    assert qp.sum() == dep._q.sum() and qp.sum() < 0
    assert close(qp, dep._q)
    fld.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,half", [("cfg1", 1 << 20), ("cfg2", 96)])
def test_config_mesh_step_fp32_within_tolerance(ctx, name, half):
    spec, t, tab, grid, pop, ofield, lo, hi, nb, origin = _setup(ctx, name, "fp32", 65536, half)
    n = pop.nparticles()
    opop = oracle_pop(pop.download(), 3 * n, spec.seed)
    otab = po.OracleTable.from_lxcat(t)
    fld = streamer.FieldInterp(grid)
    jumc.advance(pop, fld, spec.dt)
    assert po.advance(opop, otab, ofield, spec.dt) == 0
    g, o = pop.download(), oracle_arrays(opop)
    bad = particle_mismatch(g, o, 1e-5, xatol=1e-13, vatol=1e-2, satol=1e-5, n=n)
    assert bad.sum() / n < 2e-3, f"{bad.sum()} of {n} parents differ"
    assert abs(g.n - o.n) <= max(8, 0.01 * (o.n - n))
    fld.close(); pop.close(); grid.close(); tab.close()
