"""initfromfiles! on the device against its CPU restatement (orc_init_from_density): the
electron counts, weights and the cells' qfixed densities bit for bit, positions and s within
the last place of the device's and the host's cos, sin and log; both samplers, FP64 and FP32
populations, fluid cells, appending after existing electrons, the capacity error, and the
HDF5 loader path."""

import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import h5, jumc, lxcat, streamer
from mcstreamer_b200.fluid import Fluid
from mcstreamer_b200.initdens import AfivoLoader, NoiselessInitSampling, PoissonInitSampling, initfromfiles
from oracle import initdens_ref as I
from tests.helpers import broad, vec_relerr

R, LEN = 1e-3, 2e-3
E = 1.6021766208e-19


def _densities(M, N, seed):
    rng = np.random.default_rng(seed)
    dr, dz = R / M, LEN / N
    rc = (np.arange(M) + 0.5) * dr
    V = (2 * np.pi * rc * dr * dz)[:, None]
    n = 10 ** rng.uniform(-2, 2.3, (M, N))          # all three noiseless regimes at p = 10
    ne = np.asfortranarray(n / V)
    q = np.asfortranarray(E * ne * rng.uniform(-0.5, 1.5, (M, N)))
    return ne, q


def _setup(ctx, M, N, cap, precision="fp64"):
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.GridCyl(R, LEN, M, N, ctx=ctx)
    pop = jumc.Population(cap, None, tab, precision=precision, seed=1)
    return tab, grid, pop


@pytest.mark.gpu
@pytest.mark.parametrize("method", [I.NOISELESS, I.POISSON])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_init_matches_oracle(ctx, method, precision):
    M, N, p = 64, 96, 10
    ne, q = _densities(M, N, 3 + method)
    x, w, s, qfd, _ = I.initfromfiles(ne, q, R, LEN, M, N, method, p, seed=11)
    tab, grid, pop = _setup(ctx, M, N, len(w) + 1000, precision)
    try:
        samp = (NoiselessInitSampling if method == I.NOISELESS else PoissonInitSampling)(p)
        added = initfromfiles(samp, grid, pop, ne=ne, q=q, seed=11)
        g = pop.download()
        assert added == len(w) == g.n and g.n > M * N
        np.testing.assert_array_equal(grid.read_qfixed_density(), qfd)
        assert (g.active == 1).all() and (g.v == 0).all()
        if precision == "fp64":
            np.testing.assert_array_equal(g.w, w)
            assert (vec_relerr(g.x, x) < 1e-15).all()
            np.testing.assert_allclose(g.s, s, rtol=1e-15, atol=0)
        else:
            np.testing.assert_array_equal(g.w, w.astype(np.float32))
            assert (vec_relerr(g.x, x.astype(np.float32).astype(np.float64)) < 1e-7).all()
            np.testing.assert_allclose(g.s, s.astype(np.float32), rtol=1e-6)
    finally:
        pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_init_fluid_and_append(ctx):
    """Cells above fluid_threshold go to the fluid; electrons append after existing ones."""
    M, N, p = 48, 80, 8
    ne, q = _densities(M, N, 9)
    ne[10:20, 30:50] = 3e21
    thr = 1e21
    x, w, s, qfd, nf = I.initfromfiles(ne, q, R, LEN, M, N, I.POISSON, p, fluid_threshold=thr, seed=5)
    tab, grid, pop = _setup(ctx, M, N, len(w) + 500)
    fl = Fluid(grid)
    try:
        pop.upload(broad(200, 1))
        added = initfromfiles(PoissonInitSampling(p), grid, pop, ne=ne, q=q, fluid_threshold=thr, seed=5)
        g = pop.download()
        assert added == len(w) and g.n == 200 + len(w)
        np.testing.assert_array_equal(g.w[200:], w)
        assert (vec_relerr(g.x[200:], x) < 1e-15).all()
        ne_d, _, qfd_d = fl.download()
        np.testing.assert_array_equal(ne_d, nf)
        np.testing.assert_array_equal(qfd_d, qfd)
        assert (nf > 0).sum() == 200
    finally:
        fl.close(); pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_init_capacity_changes_nothing(ctx):
    M, N = 32, 40
    ne, q = _densities(M, N, 2)
    x, w, *_ = I.initfromfiles(ne, q, R, LEN, M, N, I.NOISELESS, 10, seed=3)
    tab, grid, pop = _setup(ctx, M, N, len(w) - 1)
    try:
        with pytest.raises(L.MCSError) as e:
            initfromfiles(NoiselessInitSampling(10), grid, pop, ne=ne, q=q, seed=3)
        assert e.value.code == L.ERR_CAPACITY
        assert pop.nparticles() == 0
        assert (grid.read_qfixed_density() == 0).all()
        with pytest.raises(L.MCSError):      # a finite threshold needs a fluid
            initfromfiles(NoiselessInitSampling(10), grid, pop, ne=ne, q=q, fluid_threshold=1e20)
    finally:
        pop.close(); grid.close(); tab.close()


@pytest.mark.gpu
def test_init_from_afivo_files(ctx, tmp_path):
    """The loader path: AfivoLoader files in HDF5 -> initfromfiles!, as main.jl:96-108."""
    M, N, p = 40, 64, 10
    ne, q = _densities(M, N, 7)
    mplus = np.asfortranarray(q / E + 2 * ne)
    mmin = np.asfortranarray(ne.copy())
    qf = E * (mplus - mmin - ne)                      # the charge the loader computes
    r = (np.arange(M) + 0.5) * (R / M)
    z = (np.arange(N) + 0.5) * (LEN / N)
    for name, arrs in (("ne.h5", {"e": ne}), ("q.h5", {"e": ne, "M_plus": mplus, "M_min": mmin})):
        with h5.Writer(str(tmp_path / name)) as wr:
            for k, v in arrs.items():
                wr.write(k, v)
            wr.write("r", r)
            wr.write("z", z)
    x, w, s, qfd, _ = I.initfromfiles(ne, qf, R, LEN, M, N, I.POISSON, p, seed=21)
    tab, grid, pop = _setup(ctx, M, N, len(w) + 10)
    try:
        added = initfromfiles(PoissonInitSampling(p), grid, pop,
                              loader=AfivoLoader(str(tmp_path / "ne.h5"), str(tmp_path / "q.h5")), seed=21)
        g = pop.download()
        assert added == len(w)
        np.testing.assert_array_equal(g.w, w)
        np.testing.assert_array_equal(grid.read_qfixed_density(), qfd)
    finally:
        pop.close(); grid.close(); tab.close()
