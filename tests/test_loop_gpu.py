"""The streamer loop on the device (loop.nsteps, MCStreamer/src/main.jl:218-318) against the
oracle chain of the same calls, and its invariants over several steps.

Step 1 runs every part of the loop: poisson! (from electrons sampled by initfromfiles!, a
needle fluid and qfixed densities), h5export output, the mixed advance with the tracker,
the diagnostics, repack!/resample! (resample fires at t = 0) and the fluid.  The oracle
redoes the step from the same initial state: poisson_ref.poisson, po.advance_mixed in the
oracle's own face fields, the photon and electron repack!, the cell sort and resample!,
setdne!/euler! and repack!.  Potentials agree within 1e-11 (the solve's tolerances), so the
particles and the fluid are compared at 1e-8 with a small allowance for Monte Carlo
decisions that the 1e-11 field differences can flip."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import fieldsio, jumc, loop, lxcat, streamer
from mcstreamer_b200.fluid import MOBILITY, Fluid
from mcstreamer_b200.initdens import NoiselessInitSampling, initfromfiles
from mcstreamer_b200.poisson import MGConfig, PoissonSolver, read_faces
from oracle import fluid_ref as F
from oracle import poisson_ref as P
from oracle import pyoracle as po
from tests.helpers import oracle_arrays, oracle_pop, vec_relerr

M, N, LEVELS = 64, 256, 4
R, LEN = 1e-3, 4e-3
EB, DT = -1.5e6, 1e-12
SEED = 31


def _channel():
    rc = (np.arange(M) + 0.5) * (R / M)
    zc = (np.arange(N) + 0.5) * (LEN / N)
    ne = 4e19 * np.exp(-rc[:, None] ** 2 / (2 * (2e-4) ** 2)) * ((zc > 1e-3) & (zc < 3e-3))[None, :]
    return np.asfortranarray(ne), np.asfortranarray(0.02 * 1.6021766208e-19 * ne)


def _streamer(ctx, t):
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    solver = PoissonSolver(grid, MGConfig(levels=LEVELS))
    fluid = Fluid(grid)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(400_000, None, tab, precision="fp64", seed=SEED)
    ne, q = _channel()
    initfromfiles(NoiselessInitSampling(10), grid, pop, ne=ne, q=q, seed=3)
    fluid.set_needle(5e-4, 1e-4, 3e-3, 0.0, 2e19)
    photons = jumc.Photons(2_000_000, t.photon_numax, seed=7, ctx=ctx)
    s = loop.Streamer(grid, solver, pop, streamer.FieldInterp(grid), photons, fluid)
    return s, tab


def _close(s, tab):
    s.efield.close(); s.photons.close(); s.fluid.close(); s.electrons.close(); s.solver.close(); s.grid.close()
    tab.close()


@pytest.mark.gpu
def test_first_loop_step_matches_the_oracle_chain(ctx, tmp_path):
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    s, tab = _streamer(ctx, t)
    try:
        p0 = s.electrons.download()
        ne0, _, qfd0 = s.fluid.download()
        assert p0.n > 20_000
        out = loop.nsteps(s, 1, 10, 15, EB, DT, DT, 1e-10, DT, outpath=str(tmp_path / "out"))
        assert out[0]["resampled"]
        # poisson! of the initial state
        qp = s.grid.read_fixed(L.Q_PART)
        u = P.cells(M, N)
        er, ez = P.faces(M, N), P.faces(M, N)
        P.poisson(P.default_conf(R, LEN, M, N, levels=LEVELS), np.zeros_like(qp), qp, u, er, ez, EB, R, LEN,
                  qfd=qfd0.ravel(order="F"), ne=ne0.ravel(order="F"))
        scale = np.abs(u).max()
        assert np.abs(s.solver.u - u).max() <= 1e-11 * scale
        der, dez = read_faces(s.grid)
        assert np.abs(dez - ez).max() <= 1e-9 * np.abs(ez).max()
        # the rest of the step in the oracle
        cap = 400_000
        opop = oracle_pop(p0, cap, SEED)
        oph = po.OraclePhotons(2_000_000, t.photon_numax, seed=7)
        ofield = po.field_cyl(R, LEN, M, N, er.T.ravel(), ez.T.ravel())
        otrk = po.tracker_cyl(R, LEN, M, N)
        assert po.advance_mixed(opop, oph, po.OracleTable.from_lxcat(t), ofield, DT, otrk) == 0
        po.photons_repack(oph)
        po.repack(opop)
        po.sort_cells(opop, ofield)
        assert po.resample_cells(opop, ofield, 10, 15, 0) == 0
        ne, dne = ne0.copy(order="F"), F.centers(M, N)
        F.setdne(ne, dne, er, ez, R, LEN, M, N, MOBILITY)
        F.euler(ne, dne, DT, M, N)
        po.repack(opop)
        g, o = s.electrons.download(), oracle_arrays(opop)
        assert abs(g.n - o.n) <= max(3, 1e-4 * o.n), (g.n, o.n)
        n = min(g.n, o.n)
        bad = (vec_relerr(g.x[:n], o.x[:n], 1e-30) > 1e-8) | (g.w[:n] != o.w[:n]) | (g.active[:n] != o.active[:n])
        assert bad.sum() <= max(5, 1e-3 * n), f"{bad.sum()} of {n} electrons differ"
        assert s.photons.count() == oph.n
        ne_d, _, _ = s.fluid.download()
        np.testing.assert_allclose(ne_d, ne, rtol=1e-8, atol=1e-8 * np.abs(ne).max())
        # the output written at t = 0 is h5export's layout
        f = fieldsio.load_fields(str(tmp_path / "out" / "0000.h5"))
        assert f["grid"]["M"] == M and f["er"].shape == (M + 1, N) and f["ez"].shape == (M, N + 1)
        assert f["qfixed"].shape == (M, N) and np.abs(f["u"]).max() > 0
    finally:
        _close(s, tab)


@pytest.mark.gpu
def test_loop_is_deterministic_and_keeps_its_invariants(ctx):
    """Five steps twice from the same state: identical diagnostics and populations; the
    weight checks of the resample block hold; the photons stay active-only after repack!."""
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    runs = []
    for _ in range(2):
        s, tab = _streamer(ctx, t)
        try:
            out = loop.nsteps(s, 5, 10, 15, EB, DT, 2 * DT, 1.0, 2 * DT)
            g = s.electrons.download()
            ph = s.photons.download()
            runs.append((out, g, ph))
            assert [d["resampled"] for d in out if "resampled" in d] == [True] * 3
            assert (g.active == 1).all()
            assert all(d["active_superelectrons"] > 0 and d["mean_energy"] > 0 for d in out)
        finally:
            _close(s, tab)
    (o1, g1, p1), (o2, g2, p2) = runs
    assert o1 == o2
    np.testing.assert_array_equal(g1.x, g2.x)
    np.testing.assert_array_equal(g1.w, g2.w)
    np.testing.assert_array_equal(p1.x, p2.x)
