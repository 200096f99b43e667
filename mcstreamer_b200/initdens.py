"""Initial electrons from density files: MCStreamer/src/initdens.jl.

* `AMLoader(nefile, qfile)` and `AfivoLoader(nefile, qfile)` read the HDF5 init files
  (initdens.jl:23-55) into (ne, q, data_dr, data_dz), ne and q as (M, N) arrays.
* `NoiselessInitSampling(p)` and `PoissonInitSampling(p)` choose nsample (initdens.jl:
  109-142).
* `initfromfiles(method, grid, popl, loader, ...)` is initfromfiles! (initdens.jl:64-102) on
  the device: the electrons are appended to `popl` in the reference's cell order, qfixed's
  density part is set per cell, and cells above `fluid_threshold` go to the grid's fluid.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Tuple, Union

import numpy as np

from . import _lib as L
from . import constants as co
from . import h5
from .jumc import Population
from .streamer import GridCyl


@dataclass
class NoiselessInitSampling:
    p: int
    method: int = L.INIT_NOISELESS


@dataclass
class PoissonInitSampling:
    p: int
    method: int = L.INIT_POISSON


@dataclass
class AMLoader:
    """Files with `group1/electron_density`, `group1/charge_density` and the attributes
    `x.delta`, `y.delta` of `group1` (initdens.jl:23-37)."""
    nefile: str
    qfile: str

    def load(self):
        rn, rq = h5.Reader(self.nefile), h5.Reader(self.qfile)
        ne = rn["group1/electron_density"]
        q = rq["group1/charge_density"]
        att = rq.attrs("group1")
        return ne, q, float(np.ravel(att["x.delta"])[0]), float(np.ravel(att["y.delta"])[0])


@dataclass
class AfivoLoader:
    """Files with datasets `e`, `M_plus`, `M_min`, `r`, `z` (initdens.jl:40-55):
    q = e (M_plus - M_min - e)."""
    nefile: str
    qfile: str

    def load(self):
        rn, rq = h5.Reader(self.nefile), h5.Reader(self.qfile)
        ne = rn["e"]
        q = co.elementary_charge * (rq["M_plus"] - rq["M_min"] - rq["e"])
        if not (np.array_equal(rn["r"], rq["r"]) and np.array_equal(rn["z"], rq["z"])):
            raise ValueError("the ne and q files have different r or z coordinates")
        return ne, q, float(np.diff(rn["r"])[0]), float(np.diff(rn["z"])[0])


def loadinit(loader) -> Tuple[np.ndarray, np.ndarray, float, float]:
    return loader.load()


def initfromfiles(method: Union[NoiselessInitSampling, PoissonInitSampling], grid: GridCyl, popl: Population,
                  loader=None, ne: Optional[np.ndarray] = None, q: Optional[np.ndarray] = None,
                  fluid_threshold: float = math.inf, seed: int = 0) -> int:
    """initfromfiles!(method, fields, loader; fluid_threshold, maxp) with maxp the
    population's capacity.  Either a loader or the (M, N) arrays ne and q.  A finite
    fluid_threshold needs a Fluid on the grid.  Returns the electrons appended."""
    if loader is not None:
        ne, q, data_dr, data_dz = loadinit(loader)
        dr, dz = grid.R / grid.M, grid.L / grid.N
        if not (math.isclose(data_dr, dr, rel_tol=1.5e-8) and math.isclose(data_dz, dz, rel_tol=1.5e-8)):
            raise ValueError(f"file cell sizes ({data_dr}, {data_dz}) differ from the grid's ({dr}, {dz})")
    if ne is None or q is None:
        raise ValueError("a loader or the arrays ne and q are needed")
    ne = np.asarray(ne, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    if ne.shape != (grid.M, grid.N) or q.shape != (grid.M, grid.N):
        raise ValueError(f"Size {ne.shape} != (M={grid.M}, N={grid.N})")
    a = np.ascontiguousarray(ne.ravel(order="F"))
    b = np.ascontiguousarray(q.ravel(order="F"))
    added = C.c_int64()
    popl.ctx.check(popl.ctx.lib.mcs_init_from_density(popl.h, grid.h_, L.dptr(a), L.dptr(b), method.method,
                                                      int(method.p), float(fluid_threshold), int(seed),
                                                      C.byref(added)))
    return added.value
