"""The Poisson solve's CPU restatement, pinned without a GPU.

The reference ships no test or fixture for Multigrid or solve_freebc!, so the restatement is
pinned against what defines it: the discrete system it must converge to (an independent
sparse direct solve), the radius independence that the reference's own
Multigrid/scratch/freebc.jl plots for its free boundary condition, FFTW's RODFT10/RODFT01
definitions, and the AMOS Bessel functions behind besselix/besselkx (scipy.special)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from oracle import poisson_ref as P


def _direct(M, N, s, b, top=None):
    """Solve L u = -s b with the ghost rules of the boundary conditions written out
    (Dirichlet ghost = 2 V - valid at r = R when `top` gives V, else -valid; Dirichlet
    -valid at z = 0, L; Neumann +valid on the axis) and the cylindrical connector."""
    idx = lambda i, j: (i - 1) + (j - 1) * M
    rows, cols, vals = [], [], []
    rhs = -s * b[1:M + 1, 1:N + 1].flatten(order="F")
    for j in range(1, N + 1):
        for i in range(1, M + 1):
            p = idx(i, j)
            fp, fm = 1.0 + 1.0 / (2 * i - 1), 1.0 - 1.0 / (2 * i - 1)
            d = -4.0
            if i < M:
                rows.append(p); cols.append(idx(i + 1, j)); vals.append(fp)
            else:
                d -= fp
                if top is not None:
                    rhs[p] -= 2.0 * top[j] * fp
            if i > 1:
                rows.append(p); cols.append(idx(i - 1, j)); vals.append(fm)
            else:
                d += fm
            for jj in (j - 1, j + 1):
                if 1 <= jj <= N:
                    rows.append(p); cols.append(idx(i, jj)); vals.append(1.0)
                else:
                    d -= 1.0
            rows.append(p); cols.append(p); vals.append(d)
    A = sp.csc_matrix((vals, (rows, cols)), shape=(M * N, M * N))
    return spl.spsolve(A, rhs).reshape((M, N), order="F")


def _gauss(M, N, R, L, width, peak=1.6, zc=0.5):
    dr, dz = R / M, L / N
    r = (np.arange(M) + 0.5) * dr
    z = (np.arange(N) + 0.5) * dz
    b = P.cells(M, N)
    b[1:M + 1, 1:N + 1] = peak * np.exp(-(r[:, None] ** 2 + (z[None, :] - zc * L) ** 2) / (2 * width ** 2))
    return b


@pytest.mark.parametrize("M,N,levels", [(32, 64, 4), (48, 160, 4), (64, 256, 5), (24, 40, 3)])
def test_multigrid_converges_to_the_discrete_solution(M, N, levels):
    """Odd coarsest levels included (48 x 160 / 2^4 = 3 x 10, 24 x 40 / 2^3 = 3 x 5): the
    reference's red-black sweep then also updates the ghost row, which changes the path but
    not the fixed point."""
    R, L = 1e-3 * M / 32, 1e-3 * N / 32
    b = _gauss(M, N, R, L, R / 4)
    conf = P.MGConf(P.default_conf(R, L, M, N).s, levels=levels, tolerance=1e6 * P.ELEMENTARY_CHARGE)
    u = P.cells(M, N)
    it, eps = P.mg_solve(conf, u, b)
    assert 2 <= it <= conf.maxiter
    assert eps < conf.s * conf.tolerance
    ud = _direct(M, N, conf.s, b)
    assert np.abs(u[1:M + 1, 1:N + 1] - ud).max() <= 1e-11 * np.abs(ud).max()


def test_each_fmg_call_cuts_the_residual():
    M, N, levels = 64, 256, 5
    R, L = 2e-3, 8e-3
    b = _gauss(M, N, R, L, R / 4)
    conf = P.default_conf(R, L, M, N, levels=levels, tolerance=0.0, maxiter=0)
    u = P.cells(M, N)
    prev = P.residual_rms(conf.s, u, b)
    for _ in range(3):
        P.mg_solve(conf, u, b)
        cur = P.residual_rms(conf.s, u, b)
        assert cur < prev / 50
        prev = cur


def test_inhomogeneous_top_value_matches_ghost_rule():
    """Multigrid/scratch/inhombc.jl's case: no charge, a fixed potential V(z) at r = R added
    through setinhom!; the solve must equal the system whose ghost is 2 V - valid."""
    M, N, levels = 32, 128, 4
    conf = P.MGConf(1.0, levels=levels, tolerance=1e-13)
    b = P.cells(M, N)
    top = np.zeros(N + 2)
    top[1:N + 1] = 15.0 * np.sin(np.pi * (np.arange(N) + 0.5) / N) + 3.0
    P.set_inhom_top(conf, b, top)
    u = P.cells(M, N)
    P.mg_solve(conf, u, b)
    ud = _direct(M, N, 1.0, P.cells(M, N), top=top)
    assert np.abs(u[1:M + 1, 1:N + 1] - ud).max() <= 1e-10 * np.abs(ud).max()


def test_free_boundary_is_radius_independent():
    """Multigrid/scratch/freebc.jl: with the free condition at r = R the potential inside R
    does not depend on where R is; a grounded wall at R changes it by tens of percent."""
    L, N = 0.02, 256
    h = L / N
    sols = {}
    for xf in (1, 4):
        M = 32 * xf
        R = M * h
        conf = P.default_conf(R, L, M, N, levels=4)
        b = _gauss(M, N, R, L, 8 * h)
        b_dir = b.copy(order="F")
        u = P.cells(M, N)
        P.solve_freebc(conf, u, b, R, L)
        ud = P.cells(M, N)
        P.mg_solve(conf, ud, b_dir)
        sols[xf] = (u, ud)
    (u1, d1), (u4, d4) = sols[1], sols[4]
    scale = np.abs(u4).max()
    assert np.abs(u1[1:33, 1:N + 1] - u4[1:33, 1:N + 1]).max() < 5e-4 * scale
    assert np.abs(d1[1:33, 1:N + 1] - d4[1:33, 1:N + 1]).max() > 0.1 * scale


def test_sine_transforms_are_fftw_rodft():
    rng = np.random.default_rng(3)
    for n in (1, 2, 7, 64):
        x = rng.normal(size=n)
        j = np.arange(n)
        y2 = np.array([2 * np.sum(x * np.sin(np.pi * (j + 0.5) * (k + 1) / n)) for k in range(n)])
        y3 = np.array([(-1) ** k * x[-1] + 2 * np.sum(x[:-1] * np.sin(np.pi * (j[:-1] + 1) * (k + 0.5) / n))
                       for k in range(n)])
        np.testing.assert_allclose(P.dst2(x), y2, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(P.dst3(x), y3, rtol=1e-12, atol=1e-12)


def test_library_bessel_coefficients_match_amos():
    from mcstreamer_b200.poisson import freebc_coefficients
    for L, R, N in [(0.1, 0.015, 10240), (0.02, 0.004, 256), (80.0, 20.0, 1024), (1.0, 1e-3, 64)]:
        np.testing.assert_allclose(freebc_coefficients(L, R, N), P.freebc_coefficients(L, R, N), rtol=1e-14)


def test_face_fields_of_a_linear_potential():
    M, N, R, L, eb = 6, 8, 1.0, 2.0, -3.0
    dr, dz = R / M, L / N
    i, j = np.meshgrid(np.arange(M + 2), np.arange(N + 2), indexing="ij")
    u = np.asfortranarray(2.0 * i + 5.0 * j, dtype=np.float64)
    er, ez = P.faces(M, N), P.faces(M, N)
    P.efield_faces(u, eb, R, L, er, ez)
    np.testing.assert_allclose(er[:, 0:N + 2][1:M + 2], -2.0 / dr)
    np.testing.assert_allclose(ez[0:M + 2, 1:N + 2], eb - 5.0 / dz)
    assert (er[0, :] == 0).all() and (er[M + 2, :] == 0).all()
    assert (ez[:, 0] == 0).all() and (ez[:, N + 2] == 0).all()


def test_charge_assembly_rounds_through_float32():
    M, N, R, L = 4, 6, 1e-3, 2e-3
    rng = np.random.default_rng(5)
    qf = rng.integers(-2 ** 40, 2 ** 40, size=(M + 2) * (N + 2))
    qp = rng.integers(-2 ** 40, 2 ** 40, size=(M + 2) * (N + 2))
    b = P.assemble_charge(qf, qp, R, L, M, N)
    dv = P.cell_volumes(R, L, M, N)
    i, j = 2, 3
    k = i + j * (M + 2)
    q0 = (qf[k] * 2.0 ** -32 / dv[i - 1] + qp[k] * 2.0 ** -32 / dv[i - 1]) * P.ELEMENTARY_CHARGE
    assert b[i, j] == float(np.float32(q0))
    assert (b[0, :] == 0).all() and (b[:, 0] == 0).all() and (b[M + 1, :] == 0).all()
