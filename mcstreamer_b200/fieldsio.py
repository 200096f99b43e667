"""Grid fields on disk: `h5export` (MCStreamer/src/plot.jl:210-238) and its reader.

`h5export(path, grid, solver, fluid=None, p=None, wtotal=None)` writes what the reference's
h5export writes for a SavedGridFields (io.jl:9-50), in the same HDF5 layout (HDF5.jl's, the
Julia M x N arrays stored as N x M datasets):

    grid/R, grid/L, grid/M, grid/N          scalars
    grid/rc, grid/rf, grid/zc, grid/zf      cell centres and faces
    qfixed, qpart, q0, q, u, p, wtotal      [1:M, 1:N]
    er                                      [1:M+1, 1:N]
    ez                                      [1:M, 1:N+1]

qfixed and qpart are the grid's charge densities (the int64 deposits over dV, qfixed plus its
FP64 density part), q0 = (qfixed + qpart - ne) e, q the right-hand side poisson! left (the
Float32 copy plus the free-boundary term), u the potential, er and ez the face fields.  p and
wtotal are resample!'s per-cell counters; the resample kernel keeps them to itself, so they
are written as given, or zero.

`savefields` writes the same file.  The reference's savefields writes a JLD2 container of a
SavedGridFields (io.jl:56-58); this module writes the fields in h5export's HDF5 layout, which
the reference converts JLD2 files into for post-processing (`h5export(from, to)`).
`load_fields(path)` reads such a file back into a dict of (M, N)-shaped arrays.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from . import _lib as L
from . import constants as co
from . import h5
from .poisson import PoissonSolver, read_faces
from .streamer import GridCyl


def grid_coordinates(grid: GridCyl) -> Dict[str, np.ndarray]:
    """rc, rf, zc, zf with dr = R/M, dz = L/N (cell i spans [(i-1) dr, i dr])."""
    dr, dz = grid.R / grid.M, grid.L / grid.N
    return {"rf": np.arange(grid.M + 1) * dr, "zf": np.arange(grid.N + 1) * dz,
            "rc": (np.arange(grid.M) + 0.5) * dr, "zc": (np.arange(grid.N) + 0.5) * dz}


def saved_fields(grid: GridCyl, solver: PoissonSolver, fluid=None, p: Optional[np.ndarray] = None,
                 wtotal: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
    """The arrays of SavedGridFields(fields) (io.jl:42-54) from the device state."""
    M, N = grid.M, grid.N
    qfixed = grid.read_density(L.Q_FIXED) + grid.read_qfixed_density()
    qpart = grid.read_density(L.Q_PART)
    ne = np.zeros((M + 2, N + 2), order="F")
    if fluid is not None:
        ne[1:M + 1, 1:N + 1] = fluid.download()[0][2:M + 2, 2:N + 2]
    q0 = (qfixed + qpart - ne) * co.elementary_charge
    er, ez = read_faces(grid)
    out = {"qfixed": qfixed[1:M + 1, 1:N + 1], "qpart": qpart[1:M + 1, 1:N + 1], "q0": q0[1:M + 1, 1:N + 1],
           "q": solver.q[1:M + 1, 1:N + 1], "u": solver.u[1:M + 1, 1:N + 1],
           "er": er[1:M + 2, 1:N + 1], "ez": ez[1:M + 1, 1:N + 2],
           "p": np.zeros((M, N), np.int64) if p is None else np.asarray(p, np.int64),
           "wtotal": np.zeros((M, N)) if wtotal is None else np.asarray(wtotal, np.float64)}
    for k in ("p", "wtotal"):
        if out[k].shape != (M, N):
            raise ValueError(f"{k} must be (M, N)")
    return out


def h5export(path: str, grid: GridCyl, solver: PoissonSolver, fluid=None, p=None, wtotal=None) -> None:
    fields = saved_fields(grid, solver, fluid, p, wtotal)
    with h5.Writer(path) as w:
        w.create_group("grid")
        w.write("grid/R", float(grid.R))
        w.write("grid/L", float(grid.L))
        w.write("grid/M", np.int64(grid.M))
        w.write("grid/N", np.int64(grid.N))
        for k, v in grid_coordinates(grid).items():
            w.write(f"grid/{k}", v)
        for k in ("qfixed", "qpart", "q0", "q", "u", "er", "ez", "p", "wtotal"):
            w.write(k, np.asfortranarray(fields[k]))


savefields = h5export


def load_fields(path: str) -> Dict[str, object]:
    """An h5export file: the grid's scalars and coordinates under 'grid', the arrays with
    their Julia shapes."""
    r = h5.Reader(path)
    out: Dict[str, object] = {"grid": {k: r[f"grid/{k}"] for k in r.keys("grid")}}
    for k in r.keys("/"):
        if k != "grid":
            out[k] = r[k]
    return out
