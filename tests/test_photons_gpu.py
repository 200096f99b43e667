"""Photons on the device against the CPU restatement: advance! over electrons and photons
(photo-emission, straight flight, photo-ionization with the tracker) in FP64, particle by
particle, with the populations grown in the same serial order."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, streamer
from oracle import pyoracle as po
from tests.helpers import broad, oracle_arrays, oracle_pop, particle_mismatch, vec_relerr

R, LEN, M, N = 2e-4, 4e-4, 32, 64
DT = 1e-12


def _electrons(n, seed, wmax_log=2.5, emax_ev=150.0):
    p = broad(n, seed, emax_ev=emax_ev)
    rng = np.random.default_rng(seed)
    r = R * 0.8 * np.sqrt(rng.random(n))
    th = 2 * np.pi * rng.random(n)
    p.x[:, 0] = r * np.cos(th)
    p.x[:, 1] = r * np.sin(th)
    p.x[:, 2] = LEN * (0.2 + 0.6 * rng.random(n))
    p.w[:] = np.rint(10 ** rng.uniform(1, wmax_log, n))
    return p


# s, the free-flight budget left, is a -log(u) draw minus most of itself (trem * maxrate): the
# ulp by which CUDA's and the host's log may differ survives the cancellation, so s is
# compared to an absolute 1e-12 (it is of order 1).
SATOL = 1e-12


def _photon_mismatch(g, o, rtol):
    n = min(len(g.w), len(o[3]))
    x, v, nu, w, s, act = (a[:n] for a in o)
    bad = vec_relerr(g.x[:n], x) > rtol
    bad |= vec_relerr(g.v[:n], v) > rtol
    bad |= np.abs(g.nu[:n] - nu) > rtol * np.abs(nu)
    bad |= np.abs(g.s[:n] - s) > SATOL
    bad |= g.w[:n] != w
    bad |= g.active[:n] != act
    return bad


@pytest.mark.gpu
def test_mixed_advance_matches_oracle(ctx):
    n, steps = 20_000, 3
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    p0 = _electrons(n, 13)
    pop = jumc.Population(20 * n, p0, tab, precision="fp64", seed=31)
    ph = jumc.Photons(1_000_000, t.photon_numax, seed=7, ctx=ctx)
    fld = jumc.FixedField(-1e7, ctx)
    grid.zero(L.Q_FIXED)
    opop = oracle_pop(p0, 20 * n, 31)
    oph = po.OraclePhotons(1_000_000, t.photon_numax, seed=7)
    otab = po.OracleTable.from_lxcat(t)
    ofield = po.field_uniform(0.0, 0.0, -1e7)
    otrk = po.tracker_cyl(R, LEN, M, N)
    try:
        for _ in range(steps):
            jumc.advance_mixed(pop, ph, fld, DT, streamer.CollisionTracker(grid))
            assert po.advance_mixed(opop, oph, otab, ofield, DT, otrk) == 0
        g, o = pop.download(), oracle_arrays(opop)
        assert g.n == o.n and g.n > n
        bad = particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30, satol=SATOL)
        assert bad.sum() == 0, f"{bad.sum()} electron slots differ"
        gp = ph.download()
        assert len(gp.w) == oph.n and oph.n > 1000
        badp = _photon_mismatch(gp, oph.arrays(), 1e-12)
        assert badp.sum() == 0, f"{badp.sum()} photon slots differ"
        assert (gp.active == 0).any() and (gp.active == 1).any()
        q = grid.read_density(L.Q_FIXED)
        qo = otrk._q.reshape(N + 2, M + 2).T
        np.testing.assert_allclose(q, qo, rtol=1e-12, atol=1e-6 * np.abs(qo).max())
    finally:
        fld.close(); ph.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_photon_flight_and_ionization_match_oracle(ctx):
    """The photon half alone from uploaded photons: flights, photo-ionization counts and the
    electrons appended in serial photon order (a removed photon keeps going)."""
    n, numax = 50_000, 9e12
    rng = np.random.default_rng(4)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    p = jumc.PhotonArrays(rng.uniform(-1e-4, 1e-4, (n, 3)), d * co.speed_of_light, numax * rng.random(n),
                          np.full(n, 3.0), -np.log(rng.random(n)), np.ones(n, np.uint8))
    p.active[::17] = 0
    t = lxcat.synthetic_table(0)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(20 * n, None, tab, precision="fp64", seed=1)
    ph = jumc.Photons(n, numax, seed=9, ctx=ctx, photons=p)
    oph = po.OraclePhotons(n, numax, seed=9, x=p.x, v=p.v, nu=p.nu, w=p.w, s=p.s, active=p.active)
    opop = po.OraclePop(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros(0, np.uint8),
                        cap=20 * n, seed=1)
    try:
        for _ in range(2):
            ctx.check(ctx.lib.mcs_photon_advance(ph.h, pop.h, DT, None))
            assert po.photon_advance(oph, opop, DT) == 0
        g, o = pop.download(), oracle_arrays(opop)
        assert g.n == o.n and g.n > n // 2
        assert particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30, satol=SATOL).sum() == 0
        assert _photon_mismatch(ph.download(), oph.arrays(), 1e-12).sum() == 0
    finally:
        ph.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_photo_emission_needs_the_mixed_advance(ctx):
    t = lxcat.synthetic_photo_table(0)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(4000, _electrons(1000, 3), tab, precision="fp64", seed=2)
    fld = jumc.FixedField(-3e7, ctx)
    try:
        with pytest.raises(L.MCSError) as e:
            jumc.advance(pop, fld, DT)
        assert e.value.code == L.ERR_UNSUPPORTED
    finally:
        fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_photon_capacity_is_an_error(ctx):
    t = lxcat.synthetic_photo_table(0)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(400_000, _electrons(20_000, 5, wmax_log=4.5, emax_ev=400.0), tab, precision="fp64",
                          seed=2)
    ph = jumc.Photons(50, t.photon_numax, seed=1, ctx=ctx)
    fld = jumc.FixedField(-3e7, ctx)
    try:
        with pytest.raises(L.MCSError) as e:
            jumc.advance_mixed(pop, ph, fld, DT)
        assert e.value.code == L.ERR_CAPACITY
        assert ph.count() == 50
    finally:
        fld.close(); ph.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_step_diagnostics(ctx):
    """The per-step line of nsteps (main.jl:269-279) from the device reductions against serial
    sums over the downloaded populations (population.jl:114-158)."""
    n = 20_000
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    tab = jumc.CollisionTable(t, ctx)
    pop = jumc.Population(20 * n, _electrons(n, 21), tab, precision="fp64", seed=5)
    ph = jumc.Photons(1_000_000, t.photon_numax, seed=3, ctx=ctx)
    fld = jumc.FixedField(-1e7, ctx)
    try:
        d0 = streamer.diagnostics(pop, ph)
        assert d0["active_superphotons"] == 0 and d0["physical_photons"] == 0.0
        for _ in range(2):
            jumc.advance_mixed(pop, ph, fld, DT)
        d = streamer.diagnostics(pop, ph)
        g, gp = pop.download(), ph.download()
        act = g.active.astype(bool)
        en = 0.5 * co.electron_mass * np.einsum("ij,ij->i", g.v, g.v)
        assert d["active_superelectrons"] == int(act.sum())
        assert d["physical_electrons"] == pytest.approx(float(g.w[act].sum()), rel=1e-13)
        assert d["mean_energy"] == pytest.approx(float((g.w[act] * en[act]).sum() / g.w[act].sum()), rel=1e-12)
        assert d["max_energy"] == pytest.approx(float(en.max()), rel=1e-15)
        pa = gp.active.astype(bool)
        assert d["active_superphotons"] == int(pa.sum()) > 0
        assert d["physical_photons"] == pytest.approx(float(gp.w[pa].sum()), rel=1e-13)
    finally:
        fld.close(); ph.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_photon_repack_matches_oracle(ctx):
    """repack!(photons): the reference's hole-filling permutation (population.jl:191-215)."""
    n = 100_003
    rng = np.random.default_rng(8)
    d = rng.normal(size=(n, 3))
    p = jumc.PhotonArrays(rng.normal(size=(n, 3)), d, rng.random(n), rng.random(n), rng.random(n),
                          (rng.random(n) < 0.6).astype(np.uint8))
    p.active[-5:] = 0
    ph = jumc.Photons(n, 9e12, ctx=ctx, photons=p)
    oph = po.OraclePhotons(n, 9e12, x=p.x, v=p.v, nu=p.nu, w=p.w, s=p.s, active=p.active)
    try:
        ph.repack()
        po.photons_repack(oph)
        g = ph.download()
        x, v, nu, w, s, act = oph.arrays()
        assert len(g.w) == oph.n == int(p.active.sum())
        np.testing.assert_array_equal(g.x, x)
        np.testing.assert_array_equal(g.nu, nu)
        np.testing.assert_array_equal(g.s, s)
        assert (g.active == 1).all()
        ph.repack()                       # nothing left to move
        assert ph.count() == oph.n
    finally:
        ph.close()
