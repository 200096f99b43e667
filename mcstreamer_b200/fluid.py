"""MCStreamer's electron fluid (MCStreamer/src/fluid.jl) on the device.

The fluid lives on a cylindrical grid beside the particles: setneedle! seeds it (and the
fixed charge), setdne! + euler! advance it through the face fields of the last poisson!
(main.jl:308-311), and poisson!'s charge subtracts it (poisson.jl:24), which
PoissonSolver.assemble does whenever the grid carries a fluid.

Arrays are Fortran-ordered numpy arrays: ne and dne are (M+4, N+4) with two ghost layers
(ne[i + 1, j + 1] is the reference's ne[i, j], i in -1..M+2, j in -1..N+2); qfd, the FP64
density part of qfixed, is (M+2, N+2).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib as L
from . import constants as co
from .streamer import GridCyl

MOBILITY = 1e24 / co.nair   # setdne!'s default (fluid.jl:44)


class Fluid:
    """ne, dne and the needle's share of qfixed of GridFields (gridfields.jl:24-27,67-68)."""

    def __init__(self, grid: GridCyl):
        self.grid, self.ctx, self.h = grid, grid.ctx, None
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_fluid_create(grid.h_, C.byref(h)))
        self.h = h
        self.M, self.N = grid.M, grid.N

    def set_needle(self, sigma_z: float, sigma_r: float, position_z: float, position_r: float, ne0: float) -> None:
        """setneedle!(fields, sigma_z, sigma_r, position_z, position_r, ne0) (fluid.jl:3-13)."""
        self.ctx.check(self.ctx.lib.mcs_fluid_set_needle(self.h, sigma_z, sigma_r, position_z, position_r, ne0))

    def derivatives(self, mobility: float = MOBILITY) -> None:
        """setdne!(fields, mobility) (fluid.jl:44-98), setnebc! included."""
        self.ctx.check(self.ctx.lib.mcs_fluid_derivatives(self.h, mobility))

    def euler(self, dt: float) -> None:
        """euler!(fields, dt) (fluid.jl:100-111)."""
        self.ctx.check(self.ctx.lib.mcs_fluid_euler(self.h, dt))

    def step(self, dt: float, mobility: float = MOBILITY) -> None:
        """setdne! then euler! (main.jl:308-311) in one kernel."""
        self.ctx.check(self.ctx.lib.mcs_fluid_step(self.h, mobility, dt))

    def upload(self, ne: Optional[np.ndarray] = None, qfd: Optional[np.ndarray] = None) -> None:
        a = self._flat(ne, (self.M + 4, self.N + 4))
        b = self._flat(qfd, (self.M + 2, self.N + 2))
        self.ctx.check(self.ctx.lib.mcs_fluid_upload(self.h, L.dptr(a) if a is not None else None,
                                                     L.dptr(b) if b is not None else None))

    def download(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(ne, dne, qfd)."""
        ne = np.zeros((self.M + 4) * (self.N + 4))
        dne = np.zeros_like(ne)
        qfd = np.zeros((self.M + 2) * (self.N + 2))
        self.ctx.check(self.ctx.lib.mcs_fluid_download(self.h, L.dptr(ne), L.dptr(dne), L.dptr(qfd)))
        shp = (self.M + 4, self.N + 4)
        return ne.reshape(shp, order="F"), dne.reshape(shp, order="F"), qfd.reshape((self.M + 2, self.N + 2), order="F")

    def launches(self) -> int:
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_fluid_launches(self.h, C.byref(n)))
        return n.value

    @staticmethod
    def _flat(a: Optional[np.ndarray], shape) -> Optional[np.ndarray]:
        if a is None:
            return None
        a = np.asarray(a, dtype=np.float64)
        if a.shape != shape:
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        return np.ascontiguousarray(a.ravel(order="F"))

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_fluid_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
