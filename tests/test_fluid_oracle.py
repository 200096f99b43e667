"""The electron fluid's CPU restatement (oracle/fluid.cpp) pinned without a GPU against what
the reference's code defines (MCStreamer/src/fluid.jl): the Koren limiter's branches, the
Neumann ghosts of setnebc!, the upwind direction and the limiter at a hand-worked step
profile, the exact cancellation of a uniform flux, the telescoping of the face fluxes, and
setneedle!'s profile.  No reference test exists for the fluid."""
import math

import numpy as np
import pytest

from oracle import fluid_ref as F
from oracle import poisson_ref as P


@pytest.mark.parametrize("theta,want", [(-1.0, 0.0), (0.0, 0.0), (0.2, 0.2), (0.4, 0.4),
                                        (1.0, 1.0 / 3.0 + 1.0 / 6.0), (3.999, 1.0 / 3.0 + 3.999 / 6.0),
                                        (4.0, 1.0), (1e300, 1.0), (math.inf, 1.0), (-math.inf, 0.0),
                                        (math.nan, 0.0)])
def test_koren_limiter_branches(theta, want):
    """koren_limiter (fluid.jl:107-112); NaN (a 0/0 slope ratio) falls through to 0."""
    assert F.koren(theta) == want


def test_setnebc_ghosts_are_the_clamped_interior():
    """setnebc!'s row and column copies, in its order, leave every ghost (corners included)
    equal to the nearest interior cell; the interior is untouched."""
    M, N = 5, 7
    rng = np.random.default_rng(1)
    ne = np.asfortranarray(rng.normal(size=(M + 4, N + 4)))
    inner = ne[2:M + 2, 2:N + 2].copy()
    F.setnebc(ne, M, N)
    ii = np.clip(np.arange(-1, M + 3), 1, M) + 1
    jj = np.clip(np.arange(-1, N + 3), 1, N) + 1
    np.testing.assert_array_equal(ne, ne[np.ix_(ii, jj)])
    np.testing.assert_array_equal(ne[2:M + 2, 2:N + 2], inner)


def _faces(M, N, er=0.0, ez=0.0):
    return np.full((M + 3, N + 3), er, order="F"), np.full((M + 3, N + 3), ez, order="F")


def test_step_profile_by_hand():
    """A step 1 -> 5 in z at j = 4, flow towards +z (v = -ez * mobility = 1, dz = 1):
    face fluxes F1..F7 = 1, 1, 1, 1, 5, 5, 5 (0/0 slopes limit to 0, 4/0 to 1), so only
    cell 4 changes, by F4 - F5 = -4; the ghost rows take -F1 and +F7."""
    M, N = 2, 6
    ne = F.centers(M, N)
    ne[2:M + 2, 2:N + 2] = np.array([1, 1, 1, 5, 5, 5], float)[None, :]
    dne = F.centers(M, N)
    er, ez = _faces(M, N, er=0.0, ez=-1.0)
    F.setdne(ne, dne, er, ez, 2.0, 6.0, M, N, mobility=1.0)
    np.testing.assert_array_equal(dne[2:M + 2, 2:N + 2], np.array([0, 0, 0, -4, 0, 0], float)[None, :].repeat(M, 0))
    np.testing.assert_array_equal(dne[2:M + 2, 1], -1.0)
    np.testing.assert_array_equal(dne[2:M + 2, N + 2], 5.0)
    # the same profile carried towards -z (v = -1): upstream is now j + 1 and cell 3 gains
    dne2 = F.centers(M, N)
    er, ez = _faces(M, N, er=0.0, ez=1.0)
    F.setdne(ne, dne2, er, ez, 2.0, 6.0, M, N, mobility=1.0)
    np.testing.assert_array_equal(dne2[2:M + 2, 2:N + 2], np.array([0, 0, 4, 0, 0, 0], float)[None, :].repeat(M, 0))


def test_uniform_flux_cancels_and_fluxes_telescope():
    M, N, R, Ln = 9, 13, 1e-3, 2e-3
    rng = np.random.default_rng(2)
    ne = F.centers(M, N)
    ne[2:M + 2, 2:N + 2] = 1e18 * (1 + rng.random((M, N)))
    dne = F.centers(M, N)
    er, ez = _faces(M, N, er=3e6, ez=-2e6)
    F.setdne(ne.copy(order="F"), dne, er, ez, R, Ln, M, N)
    # varying ne: the sum over the interior and the first ghost ring telescopes to zero
    assert abs(dne.sum()) <= 1e-12 * np.abs(dne).sum()
    assert np.abs(dne[2:M + 2, 2:N + 2]).max() > 0
    # uniform ne in a uniform field: every face carries the same flux, interior dne == 0
    ne[2:M + 2, 2:N + 2] = 3e18
    F.setdne(ne, dne, er, ez, R, Ln, M, N)
    np.testing.assert_array_equal(dne[2:M + 2, 2:N + 2], 0.0)


def test_euler_and_needle():
    M, N, R, Ln = 6, 10, 1e-3, 4e-3
    ne, qfd = F.centers(M, N), P.cells(M, N)
    sz, sr, pz, ne0 = 5e-4, 2e-4, 1.5e-3, 1e20
    F.setneedle(ne, qfd, R, Ln, M, N, sz, sr, pz, 7.0, ne0)
    rc = (np.arange(M) + 0.5) * (R / M)
    zc = (np.arange(N) + 0.5) * (Ln / N)
    z1 = np.maximum(0.0, zc - pz)
    want = ne0 * np.exp(-(rc[:, None] ** 2) / sr ** 2 - (z1[None, :] ** 2) / sz ** 2)
    np.testing.assert_allclose(ne[2:M + 2, 2:N + 2], want, rtol=1e-15)
    np.testing.assert_array_equal(qfd[1:M + 1, 1:N + 1], ne[2:M + 2, 2:N + 2])
    assert (ne[:, :2] == 0).all() and (qfd[0] == 0).all()
    # below the needle's tip (zc <= position_z) the profile is flat in z
    below = zc <= pz
    np.testing.assert_array_equal(ne[2:M + 2, 2:N + 2][:, below], ne[2:M + 2, 2:2 + 1].repeat(below.sum(), 1))
    dne = F.centers(M, N)
    dne[2:M + 2, 2:N + 2] = 1e27
    before = ne.copy()
    F.euler(ne, dne, 1e-12, M, N)
    np.testing.assert_array_equal(ne[2:M + 2, 2:N + 2], before[2:M + 2, 2:N + 2] + 1e-12 * 1e27)
    np.testing.assert_array_equal(ne[:2], before[:2])


def test_assembly_subtracts_the_fluid():
    """poisson.jl:21-24: q0 = (qfixed + qpart - ne) e; a needle alone (qfixed = ne) is neutral."""
    M, N, R, Ln = 8, 12, 1e-3, 2e-3
    ne, qfd = F.centers(M, N), P.cells(M, N)
    F.setneedle(ne, qfd, R, Ln, M, N, 5e-4, 3e-4, 1e-3, 0.0, 1e20)
    z = np.zeros((M + 2) * (N + 2), np.int64)
    b = P.assemble_charge(z, z, R, Ln, M, N, qfd=qfd.ravel(order="F"), ne=ne.ravel(order="F"))
    np.testing.assert_array_equal(b, 0.0)
    ne2 = ne.copy(order="F")
    ne2[2:M + 2, 2:N + 2] *= 0.5
    b = P.assemble_charge(z, z, R, Ln, M, N, qfd=qfd.ravel(order="F"), ne=ne2.ravel(order="F"))
    want = ((qfd[1:M + 1, 1:N + 1] - ne2[2:M + 2, 2:N + 2]) * P.ELEMENTARY_CHARGE).astype(np.float32)
    np.testing.assert_array_equal(b[1:M + 1, 1:N + 1], want)


def _numpy_setdne(ne, er, ez, dr, dz, mob):
    """setdne! restated independently with whole-array numpy operations: the ghosts by
    np.pad-style edge copies, each face's flux from its upwind triple, and every cell's terms
    added in the reference's order (z faces, then r faces)."""
    M, N = ne.shape[0] - 4, ne.shape[1] - 4
    inner = ne[2:M + 2, 2:N + 2]
    g = np.pad(inner, 2, mode="edge")                     # setnebc!: nearest interior cell

    def kor(a, b):
        with np.errstate(divide="ignore", invalid="ignore"):
            th = a / b
        return np.where(th >= 4.0, 1.0, np.where(th > 0.4, 1.0 / 3.0 + th / 6.0, np.where(th > 0.0, th, 0.0)))

    # z faces j = 1..N+1 of columns i = 1..M (g index j + 1 is cell j)
    v = -ez[1:M + 1, 1:N + 2] * mob
    neg = np.signbit(v)
    jf = np.arange(1, N + 2)[None, :] + 1                 # g column of cell j
    col = lambda k: np.take_along_axis(g[2:M + 2], np.broadcast_to(k, v.shape), axis=1)
    nu = np.where(neg, col(jf), col(jf - 1))
    nd = np.where(neg, col(jf - 1), col(jf))
    nu2 = np.where(neg, col(jf + 1), col(jf - 2))
    Fz = v * (nu + kor(nu - nu2, nd - nu) * (nd - nu)) / dz
    # r faces i = 1..M+1 of rows j = 1..N
    v = -er[1:M + 2, 1:N + 1] * mob
    neg = np.signbit(v)
    if_ = np.arange(1, M + 2)[:, None] + 1
    row = lambda k: np.take_along_axis(g[:, 2:N + 2], np.broadcast_to(k, v.shape), axis=0)
    nu = np.where(neg, row(if_), row(if_ - 1))
    nd = np.where(neg, row(if_ - 1), row(if_))
    nu2 = np.where(neg, row(if_ + 1), row(if_ - 2))
    Fr = v * (nu + kor(nu - nu2, nd - nu) * (nd - nu)) / dr
    d = 0.0 + Fz[:, :-1]
    d = d - Fz[:, 1:]
    d = d + Fr[:-1, :]
    d = d - Fr[1:, :]
    return g, d


def test_oracle_agrees_with_an_independent_numpy_restatement():
    """Two restatements written apart (loops in C++, whole-array numpy here) agree bit for
    bit on random fields with signed zeros, plateaus and both flow directions."""
    M, N, R, Ln = 13, 21, 1e-3, 3e-3
    rng = np.random.default_rng(11)
    ne = F.centers(M, N)
    vals = 1e18 * rng.random((M, N))
    vals[rng.random((M, N)) < 0.3] = 5e17                 # plateaus: 0/0 and x/0 slopes
    ne[2:M + 2, 2:N + 2] = vals
    er = np.asfortranarray(rng.normal(size=(M + 3, N + 3)) * 1e6)
    ez = np.asfortranarray(rng.normal(size=(M + 3, N + 3)) * 1e6)
    er[::4, ::3] = -0.0
    ez[1::5, ::2] = 0.0
    dne = F.centers(M, N)
    F.setdne(ne, dne, er, ez, R, Ln, M, N, F.MOBILITY)
    g, d = _numpy_setdne(ne, er, ez, R / M, Ln / N, F.MOBILITY)
    np.testing.assert_array_equal(ne, g)                  # the ghosts setnebc! left
    np.testing.assert_array_equal(dne[2:M + 2, 2:N + 2], d)
    ne2 = ne.copy(order="F")
    F.euler(ne2, dne, 3e-12, M, N)
    np.testing.assert_array_equal(ne2[2:M + 2, 2:N + 2], ne[2:M + 2, 2:N + 2] + 3e-12 * d)
