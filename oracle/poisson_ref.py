"""CPU restatement of MCStreamer's poisson! -- TEST INFRASTRUCTURE (the checker, never the
product).

The multigrid itself is the C++ restatement in poisson.cpp (liboracle.so); this module adds
the steps around it, in numpy/scipy:

* charge assembly from the int64 cell deposits (MCStreamer/src/poisson.jl:12-34, with the
  NullDenoiser's Float32 round trip);
* solve_freebc! (MCStreamer/src/freebc.jl:4-36).  It uses scipy.special.ive/kve, the same
  AMOS routines behind SpecialFunctions.besselix/besselkx, and scipy.fft.dst types 2 and 3,
  whose unnormalised definitions are FFTW's RODFT10 and RODFT01;
* the face fields (poisson.jl:47-57).

Arrays are Fortran-ordered numpy arrays indexed like the reference's parent arrays minus
one: u[i, j], i in 0..M+1 along r, j in 0..N+1 along z (faces 0..M+2, 0..N+2).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.fft
import scipy.special

from . import pyoracle

ELEMENTARY_CHARGE = 1.6021766208e-19
EPSILON_0 = 8.854187817620389e-12

_pd = C.POINTER(C.c_double)
_ready = False


def _lib():
    global _ready
    L = pyoracle.lib()
    if not _ready:
        L.orc_mg_solve.restype = C.c_int
        L.orc_mg_solve.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                   _pd, _pd, _pd]
        L.orc_mg_residual_rms.restype = C.c_double
        L.orc_mg_residual_rms.argtypes = [C.c_int, C.c_int, C.c_double, _pd, _pd]
        L.orc_mg_apply_bc.argtypes = [_pd, C.c_int, C.c_int]
        L.orc_mg_gauss_seidel.argtypes = [_pd, _pd, C.c_int, C.c_int]
        L.orc_mg_residual.argtypes = [_pd, _pd, _pd, C.c_double, C.c_int, C.c_int]
        L.orc_mg_restrict.argtypes = [_pd, _pd, C.c_int, C.c_int]
        L.orc_mg_interpolate.argtypes = [_pd, _pd, C.c_int, C.c_int, C.c_int]
        _ready = True
    return L


def _p(a):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_pd)


def cells(M, N):
    return np.zeros((M + 2, N + 2), order="F")


def faces(M, N):
    return np.zeros((M + 3, N + 3), order="F")


class MGConf:
    """MGConfig of MCStreamer/src/main.jl:138-144 (bc and connector are fixed)."""

    def __init__(self, s, levels=9, tolerance=1.0e8 * ELEMENTARY_CHARGE, smooth1=2, smooth2=2, maxiter=50):
        self.s, self.levels, self.tolerance = float(s), int(levels), float(tolerance)
        self.smooth1, self.smooth2, self.maxiter = int(smooth1), int(smooth2), int(maxiter)


def mg_solve(conf: MGConf, u, b):
    """Multigrid.solve(conf, u, b): u improved in place.  Returns (fmg! calls, last RMS)."""
    M, N = u.shape[0] - 2, u.shape[1] - 2
    eps = C.c_double(0.0)
    it = _lib().orc_mg_solve(M, N, conf.s, conf.levels, conf.tolerance, conf.smooth1, conf.smooth2,
                             conf.maxiter, _p(u), _p(b), C.byref(eps))
    if it < 0:
        raise ValueError("M and N must be multiples of 2^levels")
    return it, eps.value


def residual_rms(s, u, b):
    M, N = u.shape[0] - 2, u.shape[1] - 2
    return _lib().orc_mg_residual_rms(M, N, float(s), _p(u), _p(b))


def apply_bc(a):
    _lib().orc_mg_apply_bc(_p(a), a.shape[0] - 2, a.shape[1] - 2)


def gauss_seidel(u, b):
    _lib().orc_mg_gauss_seidel(_p(u), _p(b), u.shape[0] - 2, u.shape[1] - 2)


def residual(r, u, b, s):
    _lib().orc_mg_residual(_p(r), _p(u), _p(b), float(s), u.shape[0] - 2, u.shape[1] - 2)


def restrict(rh, r):
    _lib().orc_mg_restrict(_p(rh), _p(r), rh.shape[0] - 2, rh.shape[1] - 2)


def interpolate(f, h, add):
    _lib().orc_mg_interpolate(_p(f), _p(h), h.shape[0] - 2, h.shape[1] - 2, int(bool(add)))


def grid_steps(R, L, M, N):
    return R / M, L / N


def cell_volumes(R, L, M, N):
    """dV(grid, i) = 2 pi rc dr dz (MCStreamer/src/grid.jl:76), rc = (i - 1/2) dr."""
    dr, dz = grid_steps(R, L, M, N)
    rc = ((np.arange(1, M + 1) - 1).astype(np.float64) + 0.5) * dr
    return 2.0 * np.pi * rc * dr * dz


def assemble_charge(qfixed, qpart, R, L, M, N, qfd=None, ne=None):
    """q of poisson! from int64 cell charges (2^-32 elementary charges, index i + j*(M+2)):
    q0 = (qfixed + qpart - ne) e as densities, then the NullDenoiser's Float32 copy.  qfixed
    is the int64 deposit plus qfd, its FP64 density part ((M+2)x(N+2), the needle's); ne is
    the fluid density ((M+4)x(N+4) with two ghost layers), zero without a fluid."""
    dv = cell_volumes(R, L, M, N)[:, None]
    qf = np.asarray(qfixed, dtype=np.int64).reshape((M + 2, N + 2), order="F")[1:M + 1, 1:N + 1]
    qp = np.asarray(qpart, dtype=np.int64).reshape((M + 2, N + 2), order="F")[1:M + 1, 1:N + 1]
    df = qf.astype(np.float64) * 2.0 ** -32 / dv
    dp = qp.astype(np.float64) * 2.0 ** -32 / dv
    fd = 0.0 if qfd is None else np.asarray(qfd).reshape((M + 2, N + 2), order="F")[1:M + 1, 1:N + 1]
    nd = 0.0 if ne is None else np.asarray(ne).reshape((M + 4, N + 4), order="F")[2:M + 2, 2:N + 2]
    q0 = (((df + fd) + dp) - nd) * ELEMENTARY_CHARGE
    b = cells(M, N)
    b[1:M + 1, 1:N + 1] = q0.astype(np.float32).astype(np.float64)
    return b


def freebc_coefficients(L, R, N):
    """f_n = L k (I1/I0 + K1/K0)(k R) / 2 with k = (pi / L) n, n = 1..N (freebc.jl:17-20)."""
    k = (np.pi / L) * np.arange(1, N + 1)
    x = k * R
    return L * k * (scipy.special.ive(1, x) / scipy.special.ive(0, x)
                    + scipy.special.kve(1, x) / scipy.special.kve(0, x)) / 2


def dst2(x):
    """FFTW RODFT10: Y_k = 2 sum_j X_j sin(pi (j + 1/2)(k + 1) / n)."""
    return scipy.fft.dst(np.asarray(x, dtype=np.float64), type=2)


def dst3(x):
    """FFTW RODFT01: Y_k = (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j + 1)(k + 1/2) / n)."""
    return scipy.fft.dst(np.asarray(x, dtype=np.float64), type=3)


def freebc_boundary(u, R, L, M, N):
    """bcond of solve_freebc! (freebc.jl:12-28) from a solution with homogeneous b.c."""
    dr, _ = grid_steps(R, L, M, N)
    grad = (u[M + 1, 1:N + 1] - u[M, 1:N + 1]) / dr
    f = freebc_coefficients(L, R, N)
    bm = -(dr / 2) * dst2(grad)
    am = bm / f
    am1 = np.zeros_like(am)
    am1[-1] = am[-1]
    bcond = np.zeros(N + 2)
    bcond[1:N + 1] = dst3(am) / 2 + dst3(am1)
    return bcond


def set_inhom_top(conf: MGConf, b, bcond):
    """Multigrid.setinhom!(conf, b, TopBnd(), bcond) (boundaries.jl:141-153)."""
    M = b.shape[0] - 2
    b[M, :] += ((2 / conf.s) * (1.0 + 1.0 / (2 * M - 1))) * bcond


def solve_freebc(conf: MGConf, u, b, R, L):
    """solve_freebc!(u, b, grid, mg, ws) in place (b gets the inhomogeneous term).  Returns
    (fmg! calls of the first solve, of the second, bcond)."""
    M, N = u.shape[0] - 2, u.shape[1] - 2
    it1, _ = mg_solve(conf, u, b)
    bcond = freebc_boundary(u, R, L, M, N)
    set_inhom_top(conf, b, bcond)
    it2, _ = mg_solve(conf, u, b)
    u[M + 1, :] += 2 * bcond
    return it1, it2, bcond


def efield_faces(u, eb, R, L, er, ez):
    """poisson.jl:47-57: er, ez on the (M+3)x(N+3) face arrays (entries not listed there are
    left as they are)."""
    M, N = u.shape[0] - 2, u.shape[1] - 2
    dr, dz = grid_steps(R, L, M, N)
    er[1:M + 2, 1:N + 2] = (u[0:M + 1, 1:N + 2] - u[1:M + 2, 1:N + 2]) / dr
    ez[1:M + 2, 1:N + 2] = eb + (u[1:M + 2, 0:N + 1] - u[1:M + 2, 1:N + 2]) / dz
    ez[0, :] = ez[1, :]
    ez[M + 1, :] = ez[M, :]
    er[:, 0] = er[:, 1]
    er[:, N + 1] = er[:, N]


def poisson(conf: MGConf, qfixed, qpart, u, er, ez, eb, R, L, qfd=None, ne=None):
    """poisson! after density!: returns (b, it1, it2, bcond); u, er, ez updated in place.
    qfd and ne: qfixed's FP64 density part and the fluid density (see assemble_charge)."""
    M, N = u.shape[0] - 2, u.shape[1] - 2
    b = assemble_charge(qfixed, qpart, R, L, M, N, qfd=qfd, ne=ne)
    it1, it2, bcond = solve_freebc(conf, u, b, R, L)
    efield_faces(u, eb, R, L, er, ez)
    return b, it1, it2, bcond


def default_conf(R, L, M, N, levels=9, **kw):
    """main.jl:138-144: s = dz^2 / eps0, tolerance 1e8 e, smoothing 2 + 2."""
    _, dz = grid_steps(R, L, M, N)
    return MGConf(dz ** 2 / EPSILON_0, levels=levels, **kw)
