"""The device Poisson solve against its CPU restatement (oracle/poisson.cpp, poisson_ref.py).

Every multigrid operation is evaluated in the reference's order and unfused on both sides;
the coarsest direct solve (explicit inverse vs LU), the residual norm and the sine
transforms round differently, so potentials agree to ~1e-15 relative and are checked at
1e-12; iteration counts must be equal."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import jumc, lxcat, streamer
from mcstreamer_b200.poisson import MGConfig, PoissonSolver, poisson, read_faces
from oracle import poisson_ref as P
from tests.helpers import broad

# (M, N, levels): all in the one-CTA kernels, an odd coarsest level (3 x 20, the ratio of
# the reference's 1536 x 10240 sample at 9 levels), grids whose finest one or two levels
# run grid-wide, and one whose grid-wide levels end in partial tiles along r and z.
CASES = [(32, 64, 3), (48, 320, 4), (64, 256, 4), (256, 512, 5), (512, 1024, 6), (320, 1056, 5)]


def _geometry(M, N):
    return 1e-3 * M / 64, 1e-3 * N / 64


def _rhs(M, N, seed):
    R, Ln = _geometry(M, N)
    rng = np.random.default_rng(seed)
    r = (np.arange(M) + 0.5) * R / M
    z = (np.arange(N) + 0.5) * Ln / N
    b = P.cells(M, N)
    b[1:M + 1, 1:N + 1] = (1.6 * np.exp(-(r[:, None] ** 2 + (z[None, :] - 0.4 * Ln) ** 2) / (2 * (R / 5) ** 2))
                           + 0.05 * rng.normal(size=(M, N)))
    return b


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture
def solver(ctx, request):
    made = []

    def make(M, N, levels, **kw):
        R, Ln = _geometry(M, N)
        g = streamer.GridCyl(R, Ln, M, N, ctx=ctx)
        s = PoissonSolver(g, MGConfig(levels=levels, **kw))
        made.append((s, g))
        return s

    yield make
    for s, g in made:
        s.close()
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,levels", CASES)
@pytest.mark.parametrize("maxiter", [0, 2])
def test_fixed_fmg_iterations_match_oracle(solver, M, N, levels, maxiter):
    """tolerance 0: exactly maxiter + 1 fmg! calls, from a nonzero first guess."""
    s = solver(M, N, levels, tolerance=0.0, maxiter=maxiter)
    b = _rhs(M, N, 7)
    u0 = np.asfortranarray(np.random.default_rng(2).normal(size=(M + 2, N + 2)) * 10.0)
    s.set_q(b)
    s.set_u(u0)
    it, _ = s.solve()
    uo = u0.copy(order="F")
    ito, _ = P.mg_solve(P.default_conf(*_geometry(M, N), M, N, levels=levels, tolerance=0.0, maxiter=maxiter),
                        uo, b)
    assert it == ito == maxiter + 1
    assert _rel(s.u, uo) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,levels", CASES)
def test_converged_solve_matches_oracle(solver, M, N, levels):
    s = solver(M, N, levels)
    b = _rhs(M, N, 11)
    s.set_q(b)
    it, eps = s.solve()
    uo = P.cells(M, N)
    ito, epso = P.mg_solve(P.default_conf(*_geometry(M, N), M, N, levels=levels), uo, b)
    assert it == ito and it >= 2
    assert eps == pytest.approx(epso, rel=1e-6)
    assert _rel(s.u, uo) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("smooth1,smooth2", [(1, 1), (1, 2), (2, 1), (3, 3)])
def test_smoothing_counts_match_oracle(solver, smooth1, smooth2):
    """1 or 2 sweeps take the fused tile kernels, 3 the per-operation kernels."""
    M, N, levels = 320, 1056, 5
    s = solver(M, N, levels, smooth1=smooth1, smooth2=smooth2, tolerance=0.0, maxiter=1)
    b = _rhs(M, N, 17)
    s.set_q(b)
    it, _ = s.solve()
    uo = P.cells(M, N)
    conf = P.default_conf(*_geometry(M, N), M, N, levels=levels, tolerance=0.0, maxiter=1, smooth1=smooth1,
                          smooth2=smooth2)
    ito, _ = P.mg_solve(conf, uo, b)
    assert it == ito == 2
    assert _rel(s.u, uo) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,levels", [(48, 320, 4), (256, 512, 5)])
def test_freebc_matches_oracle(solver, M, N, levels):
    s = solver(M, N, levels)
    b = _rhs(M, N, 13)
    s.set_q(b)
    it = s.solve_freebc()
    R, Ln = _geometry(M, N)
    uo, bo = P.cells(M, N), b.copy(order="F")
    it1, it2, bcond = P.solve_freebc(P.default_conf(R, Ln, M, N, levels=levels), uo, bo, R, Ln)
    assert it == (it1, it2)
    np.testing.assert_allclose(s.freebc_f, P.freebc_coefficients(Ln, R, N), rtol=1e-14)
    assert _rel(s.bcond, bcond) < 1e-11
    assert _rel(s.q, bo) < 1e-12
    assert _rel(s.u, uo) < 1e-11


def _cloud(n, M, N, seed):
    R, Ln = _geometry(M, N)
    p = broad(n, seed, emax_ev=20.0)
    rng = np.random.default_rng(seed)
    r = R * 0.3 * np.sqrt(rng.random(n))
    th = 2 * np.pi * rng.random(n)
    p.x[:, 0] = r * np.cos(th)
    p.x[:, 1] = r * np.sin(th)
    p.x[:, 2] = Ln * (0.3 + 0.4 * rng.random(n))
    p.w[:] = np.rint(10 ** rng.uniform(0, 4, n))
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,levels", [(48, 320, 4), (512, 1024, 6)])
def test_poisson_run_matches_oracle(ctx, solver, M, N, levels):
    """poisson!: the electrons' NGP charge (weight -1), assembly through Float32 (bit-exact),
    solve_freebc! and the face fields written into the grid the push gathers from."""
    n, eb = 200_000, -1.5e6
    s = solver(M, N, levels)
    g = s.grid
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    pop = jumc.Population(n, _cloud(n, M, N, 3), tab, precision="fp64")
    try:
        it = poisson(s, pop, eb)
    finally:
        pop.close()
        tab.close()
    R, Ln = _geometry(M, N)
    qf, qp = g.read_fixed(L.Q_FIXED), g.read_fixed(L.Q_PART)
    assert qp.any()
    er_o, ez_o = P.faces(M, N), P.faces(M, N)
    uo = P.cells(M, N)
    bo, it1, it2, _ = P.poisson(P.default_conf(R, Ln, M, N, levels=levels), qf, qp, uo, er_o, ez_o, eb, R, Ln)
    assert it == (it1, it2)
    b_dev = s.q
    b0 = P.assemble_charge(qf, qp, R, Ln, M, N)
    np.testing.assert_array_equal(b_dev[:M, :], bo[:M, :])      # rows below M: no inhomogeneous term
    assert _rel(b_dev, bo) < 1e-12
    assert (b0[1:M + 1, 1:N + 1] < 0).any()
    assert _rel(s.u, uo) < 1e-11
    er, ez = read_faces(g)
    assert _rel(er, er_o) < 1e-10
    assert _rel(ez - eb, ez_o - eb) < 1e-10


@pytest.mark.gpu
def test_assembly_is_bit_exact(ctx, solver):
    M, N = 64, 256
    s = solver(M, N, 4)
    g = s.grid
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    pop = jumc.Population(50_000, _cloud(50_000, M, N, 9), tab, precision="fp64")
    try:
        g.zero(L.Q_PART)
        streamer.density(g, pop, -1.0)
        g.zero(L.Q_FIXED)
        s.assemble()
    finally:
        pop.close()
        tab.close()
    R, Ln = _geometry(M, N)
    want = P.assemble_charge(g.read_fixed(L.Q_FIXED), g.read_fixed(L.Q_PART), R, Ln, M, N)
    np.testing.assert_array_equal(s.q, want)


@pytest.mark.gpu
def test_bad_configuration_is_an_error(ctx):
    g = streamer.GridCyl(1e-3, 2e-3, 48, 320, ctx=ctx)
    try:
        with pytest.raises(L.MCSError):
            PoissonSolver(g, MGConfig(levels=5))       # 48 is not a multiple of 2^5
    finally:
        g.close()
