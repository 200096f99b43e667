"""Photons in the CPU restatement, pinned without a GPU against the laws the reference's code
defines (JuMC/src/electron.jl:88-105,141-144; collisions.jl:125-141; photon.jl; the
mixed_population.jl loop):

* photo-emission: per event rand(Poisson(w / photon_multiplier / photon_weight)) photons at
  the electron, isotropic at speed c, log(nu) uniform on [log nu_min, log nu_max], weight
  photon_weight, nextcoll() ~ Exp(1); the electron is unchanged and nothing is tracked;
* photons fly straight; each null-collision candidate at numax photo-ionizes with
  probability nu / numax, and a removed photon keeps sub-stepping, so the number of
  photo-ionizations of a photon in dt is Poisson(nu dt);
* the electrons it makes are at rest with its weight, active only for the first, appended in
  serial order, and each adds +w to the tracker."""
import numpy as np
import pytest
import scipy.stats as ss

from mcstreamer_b200 import constants as co
from mcstreamer_b200 import lxcat
from oracle import pyoracle as po

NU_PE = 3e12     # constant photo-emission rate (1/s)
MAXRATE = 4e12
LMIN, LMAX = np.log(1e11), np.log(8e12)


def _pe_table(mult, pw):
    """A table of one PHOTOEMISSION row at a constant rate and the null row."""
    neps = 16
    rate = np.zeros((neps, 2))
    rate[:, 0] = NU_PE
    rate[:, 1] = MAXRATE - NU_PE
    return po.OracleTable(rate, np.array([po.PHOTOEMISSION, po.NULL]), np.zeros(2), 0.0, 10 * co.eV, MAXRATE,
                          pe=(np.array([LMIN, 0.0]), np.array([LMAX, 0.0]), mult, pw))


def _electrons(n, w, seed=3):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1e-3, 1e-3, (n, 3))
    return po.OraclePop(x, np.zeros((n, 3)), np.full(n, w), -np.log(rng.random(n)), np.ones(n, np.uint8),
                        cap=n + 4_000_000, seed=11)


def _emission_points(ph, dt):
    """Photons fly straight for dt after their emission in the same step."""
    x, v = ph.arrays()[:2]
    return x - v * dt


@pytest.mark.parametrize("w,mult,pw,n", [(2500.0, 1000.0, 1.0, 20000), (4e4, 1000.0, 1.0, 6000),
                                         (3.0, 1.0, 2.0, 20000)])
def test_photo_emission_law(w, mult, pw, n):
    """lambda = 2.5 and 1.5 take the inversion sampler, 40 the PTRS one."""
    dt = 1e-12
    e = _electrons(n, w)
    x0 = e.x[:n].copy()
    ph = po.OraclePhotons(2_000_000, 9e12, seed=5)
    assert po.advance_mixed(e, ph, _pe_table(mult, pw), po.field_uniform(), dt, threads=4) == 0
    # the emitting electrons are unchanged (at rest, no field); the rest are photo-electrons
    np.testing.assert_array_equal(e.x[:n], x0)
    lam = w / mult / pw
    m = NU_PE * dt
    P = ph.n
    # compound Poisson: mean n m lam, variance n m (lam + lam^2)
    mean, sd = n * m * lam, np.sqrt(n * m * (lam + lam * lam))
    assert abs(P - mean) < 5 * sd, (P, mean, sd)
    x, v, nu, wp, s, act = ph.arrays()
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), co.speed_of_light, rtol=1e-14)
    assert np.abs(v.mean(axis=0)).max() < 5 * co.speed_of_light / np.sqrt(3 * P)
    assert ss.kstest((np.log(nu) - LMIN) / (LMAX - LMIN), "uniform").pvalue > 1e-4
    assert ss.kstest(s, "expon").pvalue > 1e-4
    assert (wp == pw).all()
    # photons that photo-ionized later in the step are the removed ones, one active electron each
    assert int((act == 0).sum()) == int(e.active[n:e.n].sum())
    # every photon was emitted at one of the electrons
    xe = _emission_points(ph, dt)[:300]
    d = np.abs(xe[:, None, :] - x0[None, :, :]).max(axis=2).min(axis=1)
    assert (d < 1e-12).all()


def test_photon_counts_per_event_are_poisson():
    """One event per electron: with nu_pe dt large the event count is known in law, so look
    at electrons of distinct weights and the photons at their positions."""
    n, dt = 4000, 1e-12
    lam = 3.7
    e = _electrons(n, lam * 1000.0, seed=9)
    ph = po.OraclePhotons(400_000, 9e12, seed=1)
    po.advance_mixed(e, ph, _pe_table(1000.0, 1.0), po.field_uniform(), dt, threads=4)
    x = np.round(_emission_points(ph, dt), 12)
    # photons of each parent: contiguous runs at its position (serial parent order)
    _, first, counts = np.unique(x, axis=0, return_index=True, return_counts=True)
    order = np.argsort(first)
    runs = counts[order]
    starts = np.sort(first)
    assert (np.diff(starts) == runs[:-1]).all()
    # per-parent totals: compound Poisson(m, Poisson(lam)); zero-photon parents are absent
    m = NU_PE * dt
    tot = np.concatenate([runs, np.zeros(n - len(runs), int)])
    assert abs(tot.mean() - m * lam) < 5 * np.sqrt(m * (lam + lam * lam) / n)


def _photons(n, nu, seed=2):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    x = rng.uniform(-1e-3, 1e-3, (n, 3))
    return x, d * co.speed_of_light, np.full(n, nu), np.full(n, 2.0), -np.log(rng.random(n)), np.ones(n, np.uint8)


@pytest.mark.parametrize("frac", [0.1, 0.6])
def test_photo_ionization_law(frac):
    n, dt, numax = 40000, 1e-12, 9e12
    nu = frac * numax
    x, v, nuv, w, s, act = _photons(n, nu)
    ph = po.OraclePhotons(n, numax, seed=4, x=x, v=v, nu=nuv, w=w, s=s, active=act)
    e = po.OraclePop(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros(0, np.uint8),
                     cap=10 * n, seed=1)
    trk = po.tracker_cart3d(8, 8, 8, 1e-3, (-4e-3, -4e-3, -4e-3))
    assert po.photon_advance(ph, e, dt, trk, threads=4) == 0
    xe, ve, we, se, ae = e.arrays()
    k = e.n
    # photo-ionizations per photon ~ Poisson(nu dt) (the loop goes on after the removal)
    assert abs(k / n - nu * dt) < 5 * np.sqrt(nu * dt / n)
    xp, vp, _, _, _, ap = ph.arrays()
    first = n - int(ap.sum())
    assert abs(first / n - (1 - np.exp(-nu * dt))) < 5 * np.sqrt((1 - np.exp(-nu * dt)) / n)
    assert int(ae.sum()) == first                      # only the first of each photon is active
    assert (ve == 0).all() and (we == 2.0).all()
    np.testing.assert_allclose(xp, x + v * dt, rtol=1e-12, atol=1e-15)
    # every electron lies on its photon's segment: along-track distance within [0, c dt]
    assert (np.linalg.norm(xe, axis=1) < 1e-2).all()
    assert trk._q.sum() == k * round(2.0 * 2 ** 32)


def test_loader_reads_photoemission_records():
    t = lxcat.synthetic_photo_table(0, photon_multiplier=500.0, photon_weight=3.0)
    j = list(t.kinds).index(po.PHOTOEMISSION)
    nu_abs = co.speed_of_light * 0.2 * lxcat.SYNTHETIC_DENSITY
    assert t.pe_lmin[j] == pytest.approx(np.log(nu_abs * 1e-23), rel=1e-15)
    assert t.pe_lmax[j] == pytest.approx(np.log(nu_abs * 6e-21), rel=1e-15)
    assert t.photon_numax == pytest.approx(nu_abs * 6e-21, rel=1e-14)
    # the cross section is scaled by rescale * photon_multiplier (lxcat.jl:47-60)
    e = t.energy.values()
    v = np.sqrt(2 * e / co.electron_mass)
    hi = e > 200 * co.eV
    np.testing.assert_allclose(t.rate[j][hi], lxcat.SYNTHETIC_DENSITY * v[hi] * 2.5e-20 * 2e-3 * 500.0, rtol=1e-12)
    assert t.photon_multiplier == 500.0 and t.photon_weight == 3.0


def test_photon_repack_is_the_reference_permutation():
    """repack!(photons) (population.jl:191-215): the k-th hole from the start takes the
    k-th active photon from the end, until they meet; checked against that loop written
    again here."""
    n = 257
    rng = np.random.default_rng(6)
    x, v, nu, w, s, act = _photons(n, 1e12, seed=6)
    act = (rng.random(n) < 0.55).astype(np.uint8)
    act[-3:] = 0
    ph = po.OraclePhotons(n, 9e12, x=x, v=v, nu=nu, w=w, s=s, active=act)
    po.photons_repack(ph)
    idx = list(range(n))
    a = act.astype(bool).tolist()
    last = n - 1
    while not a[last]:
        last -= 1
    i = 0
    while i <= last:
        if not a[i]:
            idx[i], a[i] = idx[last], True
            last -= 1
            while not a[last]:
                last -= 1
        i += 1
    idx = idx[:last + 1]
    assert ph.n == len(idx) == int(act.sum())
    xp, vp, nup, wp, sp, ap = ph.arrays()
    np.testing.assert_array_equal(xp, x[idx])
    np.testing.assert_array_equal(nup, nu[idx])
    assert (ap == 1).all()
