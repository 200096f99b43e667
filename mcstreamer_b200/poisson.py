"""The electrostatic solve of MCStreamer's poisson! on the device.

Mirrors MCStreamer/src/poisson.jl (poisson!), MCStreamer/src/freebc.jl (solve_freebc!) and
Multigrid.solve (Multigrid/src/Multigrid.jl:449-467) with the MGConfig that
MCStreamer/src/main.jl:131-144 builds: Dirichlet at z = 0, z = L and r = R, Neumann on the
axis, CylindricalConnector{1}, one ghost layer, s = dz^2 / eps0, tolerance 1e8 e, two
smoothing sweeps before and after each coarse-grid correction.

Cell arrays (u, q) are (M+2, N+2) Fortran-ordered numpy arrays indexed like the
reference's OffsetArrays: a[i, j], i = 0..M+1 along r and j = 0..N+1 along z.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib as L
from . import constants as co
from .jumc import Population
from .streamer import GridCyl, density


class MGConfig:
    """The multigrid settings of MGConfig (Multigrid.jl:41-74) that MCStreamer varies."""

    def __init__(self, levels: int = 9, smooth1: int = 2, smooth2: int = 2, maxiter: int = 50,
                 tolerance: float = 1.0e8 * co.elementary_charge, s: Optional[float] = None):
        self.levels, self.smooth1, self.smooth2 = int(levels), int(smooth1), int(smooth2)
        self.maxiter, self.tolerance = int(maxiter), float(tolerance)
        self.s = s   # None: dz^2 / eps0 of the grid (main.jl:138)


class PoissonSolver:
    """Device workspace of the solve on one cylindrical grid (Multigrid.allocate plus the
    potential and charge arrays of GridFields)."""

    def __init__(self, grid: GridCyl, conf: Optional[MGConfig] = None):
        self.grid, self.ctx = grid, grid.ctx
        self.conf = conf or MGConfig()
        self.M, self.N = grid.M, grid.N
        h = C.c_void_p()
        c = self.conf
        self.ctx.check(self.ctx.lib.mcs_poisson_create(grid.h_, c.levels, c.smooth1, c.smooth2, c.maxiter,
                                                       c.tolerance, c.s if c.s is not None else 0.0, C.byref(h)))
        self.h = h

    # -- arrays --------------------------------------------------------------------------
    def _put(self, which: int, a: np.ndarray) -> None:
        a = np.asarray(a, dtype=np.float64)
        if a.shape != (self.M + 2, self.N + 2):
            raise ValueError(f"expected shape {(self.M + 2, self.N + 2)}, got {a.shape}")
        flat = np.ascontiguousarray(a.ravel(order="F"))
        self.ctx.check(self.ctx.lib.mcs_poisson_upload(self.h, which, L.dptr(flat)))

    def _get(self, which: int) -> np.ndarray:
        out = np.zeros((self.M + 2) * (self.N + 2))
        self.ctx.check(self.ctx.lib.mcs_poisson_download(self.h, which, L.dptr(out)))
        return out.reshape((self.M + 2, self.N + 2), order="F")

    def set_u(self, u: np.ndarray) -> None:
        self._put(L.PSN_U, u)

    def set_q(self, q: np.ndarray) -> None:
        self._put(L.PSN_B, q)

    @property
    def u(self) -> np.ndarray:
        return self._get(L.PSN_U)

    @property
    def q(self) -> np.ndarray:
        return self._get(L.PSN_B)

    @property
    def bcond(self) -> np.ndarray:
        out = np.zeros(self.N + 2)
        self.ctx.check(self.ctx.lib.mcs_poisson_download(self.h, L.PSN_BCOND, L.dptr(out)))
        return out

    @property
    def freebc_f(self) -> np.ndarray:
        out = np.zeros(self.N)
        self.ctx.check(self.ctx.lib.mcs_poisson_download(self.h, L.PSN_FREEBC_F, L.dptr(out)))
        return out

    def zero(self, which: int = L.PSN_U) -> None:
        self.ctx.check(self.ctx.lib.mcs_poisson_zero(self.h, which))

    def launches(self) -> int:
        """Kernels this workspace has launched so far (graph nodes included)."""
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_poisson_launches(self.h, C.byref(n)))
        return n.value

    def profile(self, reps: int = 20) -> Tuple[float, float, float]:
        """ms of one finest-level red-black pass, one finest-level residual and one fused
        finest-level post-smoothing launch (0.0 when unfused)."""
        g, r, t = C.c_float(0.0), C.c_float(0.0), C.c_float(0.0)
        self.ctx.check(self.ctx.lib.mcs_poisson_profile(self.h, int(reps), C.byref(g), C.byref(r), C.byref(t)))
        return g.value, r.value, t.value

    # -- the reference's functions ---------------------------------------------------------
    def solve(self) -> Tuple[int, float]:
        """Multigrid.solve(mg, u, q, ws): (fmg! calls, residual RMS of the last check)."""
        it = C.c_int(0)
        eps = C.c_double(0.0)
        self.ctx.check(self.ctx.lib.mcs_poisson_mg_solve(self.h, C.byref(it), C.byref(eps)))
        return it.value, eps.value

    def solve_freebc(self) -> Tuple[int, int]:
        """solve_freebc!(u, q, grid, mg, ws): fmg! calls of its two solves."""
        it = (C.c_int * 2)()
        self.ctx.check(self.ctx.lib.mcs_poisson_solve_freebc(self.h, it))
        return it[0], it[1]

    def assemble(self) -> None:
        """q = Float32((qfixed + qpart) e) from the grid's cell charges."""
        self.ctx.check(self.ctx.lib.mcs_poisson_assemble(self.h))

    def fields(self, eb: float) -> None:
        """The grid's face fields er, ez from u (poisson.jl:47-57)."""
        self.ctx.check(self.ctx.lib.mcs_poisson_fields(self.h, float(eb)))

    def run(self, eb: float) -> Tuple[int, int]:
        """poisson! after density!: assemble, solve_freebc!, fields."""
        it = (C.c_int * 2)()
        self.ctx.check(self.ctx.lib.mcs_poisson_run(self.h, float(eb), it))
        return it[0], it[1]

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_poisson_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def poisson(solver: PoissonSolver, popl: Population, eb: float) -> Tuple[int, int]:
    """poisson!(fields, mpopl, eb, mg, ws, NullDenoiser(), t): the electrons' charge
    (weight -1 each, density! of poisson.jl:65-84) into fields.qpart, then the solve and the
    face fields the next push gathers."""
    solver.grid.zero(L.Q_PART)
    density(solver.grid, popl, -1.0)
    return solver.run(eb)


def freebc_coefficients(L_: float, R: float, N: int) -> np.ndarray:
    """f_n of solve_freebc! (freebc.jl:17-20), computed by the library on the host."""
    out = np.zeros(int(N))
    L.check(L.lib().mcs_freebc_coefficients(float(L_), float(R), int(N), L.dptr(out)))
    return out


def read_faces(grid: GridCyl) -> Tuple[np.ndarray, np.ndarray]:
    """The grid's (er, ez) face arrays, (M+3, N+3) each, indexed like calloc_faces."""
    nf = (grid.M + 3) * (grid.N + 3)
    out = np.zeros(2 * nf)
    grid.ctx.check(grid.ctx.lib.mcs_grid_read_efield(grid.h_, L.dptr(out)))
    er = out[:nf].reshape((grid.M + 3, grid.N + 3), order="F")
    ez = out[nf:].reshape((grid.M + 3, grid.N + 3), order="F")
    return er, ez
