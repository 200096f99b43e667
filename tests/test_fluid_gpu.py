"""The electron fluid on the device against its CPU restatement (oracle/fluid.cpp): setdne!
(with setnebc!), euler!, the fused step and the charge assembly bit for bit, setneedle!
within exp's rounding.  Inputs mix smooth and flat regions, so the 0/0 and x/0 slope ratios
the limiter sees in the reference occur, and faces of both signs, signed zeros included."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import streamer
from mcstreamer_b200.fluid import MOBILITY, Fluid
from mcstreamer_b200.poisson import MGConfig, PoissonSolver, read_faces
from oracle import fluid_ref as F
from oracle import poisson_ref as P

SHAPES = [(5, 7), (64, 128), (130, 257), (300, 40)]


def _geometry(M, N):
    return 1e-3 * M / 64, 1e-3 * N / 64


def _state(M, N, seed):
    rng = np.random.default_rng(seed)
    ne = F.centers(M, N)
    r = np.linspace(0, 1, M)[:, None]
    z = np.linspace(0, 1, N)[None, :]
    v = 1e19 * np.exp(-((r / 0.3) ** 2) - ((z - 0.5) / 0.2) ** 2)
    v = np.where(rng.random((M, N)) < 0.3, np.round(v, -18), v)     # plateaus: 0/0 and x/0 ratios
    v[:, : N // 5] = 2e18                                             # a flat band
    ne[2:M + 2, 2:N + 2] = v
    ne[0, 0] = 7.0                                                    # stale corner ghost
    er = np.asfortranarray(3e6 * rng.normal(size=(M + 3, N + 3)))
    ez = np.asfortranarray(-1e7 + 8e6 * rng.normal(size=(M + 3, N + 3)))
    er[::7, ::5] = 0.0
    ez[1::6, ::4] = -0.0
    er[2::9, 1::3] = -0.0
    return ne, er, ez


@pytest.fixture
def fluid(ctx):
    made = []

    def make(M, N):
        R, Ln = _geometry(M, N)
        g = streamer.GridCyl(R, Ln, M, N, ctx=ctx)
        f = Fluid(g)
        made.append((f, g))
        return f, g

    yield make
    for f, g in made:
        f.close()
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("M,N", SHAPES)
def test_derivatives_match_oracle(fluid, M, N):
    f, g = fluid(M, N)
    R, Ln = _geometry(M, N)
    ne, er, ez = _state(M, N, M + N)
    g.set_efield(er, ez)
    f.upload(ne=ne)
    f.derivatives()
    ne_d, dne_d, _ = f.download()
    dne = F.centers(M, N)
    F.setdne(ne, dne, er, ez, R, Ln, M, N, MOBILITY)
    np.testing.assert_array_equal(ne_d, ne)
    np.testing.assert_array_equal(dne_d, dne)
    assert np.abs(dne[2:M + 2, 2:N + 2]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("M,N", SHAPES)
def test_fused_steps_match_oracle(fluid, M, N):
    """setdne! + euler! fused, five steps, against the two oracle loops; then the separate
    entry points once more."""
    f, g = fluid(M, N)
    R, Ln = _geometry(M, N)
    ne, er, ez = _state(M, N, 3 * M + N)
    g.set_efield(er, ez)
    f.upload(ne=ne)
    dne = F.centers(M, N)
    dt = 2e-12
    for _ in range(5):
        f.step(dt)
        F.setdne(ne, dne, er, ez, R, Ln, M, N, MOBILITY)
        F.euler(ne, dne, dt, M, N)
    ne_d, dne_d, _ = f.download()
    np.testing.assert_array_equal(dne_d, dne)
    np.testing.assert_array_equal(ne_d, ne)
    f.derivatives(0.5 * MOBILITY)
    f.euler(dt)
    F.setdne(ne, dne, er, ez, R, Ln, M, N, 0.5 * MOBILITY)
    F.euler(ne, dne, dt, M, N)
    ne_d, dne_d, _ = f.download()
    np.testing.assert_array_equal(dne_d, dne)
    np.testing.assert_array_equal(ne_d, ne)
    assert f.launches() == 7


@pytest.mark.gpu
def test_needle_matches_oracle(fluid):
    M, N = 96, 320
    f, g = fluid(M, N)
    R, Ln = _geometry(M, N)
    ne, qfd = F.centers(M, N), P.cells(M, N)
    rng = np.random.default_rng(5)
    qfd[1:M + 1, 1:N + 1] = 1e17 * rng.random((M, N))
    ne[2:M + 2, 2:N + 2] = 1e16 * rng.random((M, N))
    f.upload(ne=ne, qfd=qfd)
    args = (0.3 * Ln, 0.1 * R, 0.6 * Ln, 0.0, 5e19)
    f.set_needle(*args)
    F.setneedle(ne, qfd, R, Ln, M, N, *args)
    ne_d, _, qfd_d = f.download()
    # the device's exp and the host's may differ in the last place
    np.testing.assert_allclose(ne_d, ne, rtol=1e-15, atol=0)
    np.testing.assert_allclose(qfd_d, qfd, rtol=1e-15, atol=0)


@pytest.mark.gpu
def test_assembly_with_fluid_is_bit_exact(ctx):
    """poisson!'s q0 = (qfixed + qpart - ne) e with the fluid's ne and the needle's qfixed,
    over int64 deposits, through Float32."""
    M, N = 64, 256
    R, Ln = _geometry(M, N)
    g = streamer.GridCyl(R, Ln, M, N, ctx=ctx)
    s = PoissonSolver(g, MGConfig(levels=4))
    f = Fluid(g)
    try:
        rng = np.random.default_rng(9)
        qf = rng.integers(-2 ** 50, 2 ** 50, size=(M + 2) * (N + 2)).astype(np.int64)
        qp = rng.integers(-2 ** 50, 0, size=(M + 2) * (N + 2)).astype(np.int64)
        g.write_fixed(L.Q_FIXED, qf)
        g.write_fixed(L.Q_PART, qp)
        ne, er, ez = _state(M, N, 4)
        qfd = P.cells(M, N)
        qfd[1:M + 1, 1:N + 1] = 1.1 * ne[2:M + 2, 2:N + 2]
        f.upload(ne=ne, qfd=qfd)
        s.assemble()
        want = P.assemble_charge(qf, qp, R, Ln, M, N, qfd=qfd.ravel(order="F"), ne=ne.ravel(order="F"))
        np.testing.assert_array_equal(s.q, want)
        # the fused step swaps ne's buffers: assembly follows the current one
        g.set_efield(er, ez)
        f.step(1e-12)
        ne_d, _, _ = f.download()
        s.assemble()
        want = P.assemble_charge(qf, qp, R, Ln, M, N, qfd=qfd.ravel(order="F"), ne=ne_d.ravel(order="F"))
        np.testing.assert_array_equal(s.q, want)
    finally:
        f.close()
        s.close()
        g.close()


@pytest.mark.gpu
def test_fluid_after_poisson_fields(ctx):
    """The streamer loop's order: poisson! writes the faces, the fluid steps through them."""
    M, N = 64, 256
    R, Ln = _geometry(M, N)
    g = streamer.GridCyl(R, Ln, M, N, ctx=ctx)
    s = PoissonSolver(g, MGConfig(levels=4))
    f = Fluid(g)
    try:
        f.set_needle(0.25 * Ln, 0.08 * R, 0.5 * Ln, 0.0, 1e20)
        s.assemble()
        s.solve_freebc()
        s.fields(-1.5e6)
        er, ez = read_faces(g)
        ne, _, _ = f.download()
        dne = F.centers(M, N)
        for _ in range(3):
            f.step(5e-12)
            F.setdne(ne, dne, er, ez, R, Ln, M, N, MOBILITY)
            F.euler(ne, dne, 5e-12, M, N)
        ne_d, dne_d, _ = f.download()
        np.testing.assert_array_equal(ne_d, ne)
        np.testing.assert_array_equal(dne_d, dne)
        assert np.abs(dne).max() > 0
    finally:
        f.close()
        s.close()
        g.close()


@pytest.mark.gpu
def test_fluid_rules(ctx):
    g = streamer.GridCyl(1e-3, 2e-3, 16, 32, ctx=ctx)
    f = Fluid(g)
    with pytest.raises(L.MCSError):
        Fluid(g)                                  # one fluid per grid
    g3 = streamer.Grid3D(8, 8, 8, 1e-6, ctx=ctx)
    with pytest.raises(L.MCSError):
        Fluid(g3)                                 # cylindrical grids only
    g3.close()
    g.close()
    with pytest.raises(L.MCSError):
        f.step(1e-12)                             # its grid is gone
    f.close()
