"""Device-side workload generators: the Gaussian-charge node field against the host
formula, and the Gaussian electron cloud against a restatement from the oracle's Philox
uniforms (INIT stream)."""
import numpy as np
import pytest

from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, streamer

CENTRE = (40e-6, 48e-6, 120e-6)
SIGMA_Q, PEAK, E_BG = 20e-6, 1e20, (0.0, 0.0, -15e6)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("fp32", 2e-7)])
def test_gaussian_field_matches_host(ctx, precision, rtol):
    fn = streamer.gaussian_charge_field(CENTRE, SIGMA_Q, PEAK, e_bg=E_BG)
    host = streamer.Grid3D(20, 24, 60, 4e-6, precision=precision, ctx=ctx)
    host.set_efield_fn(fn, planes_per_chunk=8)
    dev = streamer.Grid3D(20, 24, 60, 4e-6, precision=precision, ctx=ctx)
    dev.set_efield_gaussian(CENTRE, SIGMA_Q, PEAK, E_BG)
    a, b = host.read_efield(), dev.read_efield()
    scale = np.abs(a).max()
    np.testing.assert_allclose(b, a, rtol=rtol, atol=rtol * scale)
    assert np.abs(b[:, 2]).max() > 15e6   # the charge's own field is present


@pytest.mark.gpu
def test_cloud_matches_restatement(ctx):
    from oracle import pyoracle as po
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    n, seed, sigma, e_ev, wmin, wmax = 300, 42, 50e-6, 1.0, 1e2, 1e4
    pop = jumc.Population(n, None, tab, precision="fp64", seed=seed)
    pop.init_cloud(n, CENTRE, sigma, e_ev, wmin, wmax)
    got = pop.download()
    pop.close(); tab.close()
    u = np.array([[po.uniform(seed, i, 0, 3, k) for k in range(8)] for i in range(n)])
    r0, r1 = np.sqrt(-2 * np.log(u[:, 0])), np.sqrt(-2 * np.log(u[:, 2]))
    x = np.stack([CENTRE[0] + sigma * (r0 * np.cos(2 * np.pi * u[:, 1])),
                  CENTRE[1] + sigma * (r0 * np.sin(2 * np.pi * u[:, 1])),
                  CENTRE[2] + sigma * (r1 * np.cos(2 * np.pi * u[:, 3]))], axis=1)
    vabs = np.sqrt(2 * e_ev * co.elementary_charge / co.electron_mass)
    uz = 2 * u[:, 4] - 1
    st = np.sqrt(1 - uz * uz)
    v = vabs * np.stack([st * np.cos(2 * np.pi * u[:, 5]), st * np.sin(2 * np.pi * u[:, 5]), uz], axis=1)
    w = wmin * np.exp(np.log(wmax / wmin) * u[:, 6])
    np.testing.assert_allclose(got.x, x, rtol=1e-14, atol=1e-19)
    np.testing.assert_allclose(got.v, v, rtol=1e-13, atol=1e-13 * vabs)
    np.testing.assert_allclose(got.w, w, rtol=1e-13)
    np.testing.assert_allclose(got.s, -np.log(u[:, 7]), rtol=1e-14)
    assert got.active.all()


@pytest.mark.gpu
def test_cloud_on_mesh_sorts_by_cell(ctx):
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    g = streamer.Grid3D(32, 32, 64, 4e-6, precision="fp32", ctx=ctx)
    n = 200_000
    pop = jumc.Population(n, None, tab, precision="fp32", seed=5, mesh=g)
    centre = (64e-6, 64e-6, 128e-6)
    pop.init_cloud(n, centre, 20e-6, 1.0, 1e3, 1e3)
    ctx.check(ctx.lib.mcs_sort_cells(pop.h, g.h_))
    got = pop.download()
    keys = g.cell_key(got.x)
    assert (np.diff(keys) >= 0).all()
    assert np.allclose(got.x.mean(axis=0), centre, atol=0.5e-6)
    assert np.allclose(got.x.std(axis=0), 20e-6, rtol=0.02)
    assert np.allclose(got.w, 1e3)
    pop.close(); tab.close()
