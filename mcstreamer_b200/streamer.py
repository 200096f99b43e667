"""Python mirror of MCStreamer's particle-side call sites over the C ABI.

* Grid3D: the 3-D uniform node mesh of the streamer workloads (node field, CIC int64
  charge at 2^-32 e).  GridCyl: the reference's cylindrical Grid(R, L, M, N)
  (MCStreamer/src/grid.jl:4-42) with its staggered face field.
* FieldInterp(grid): the `efield` callable (gridfields.jl:89-190); CollisionTracker(grid):
  the tracker of gridfields.jl:198-224 (qfixed); density(grid, popl, val): density!
  (poisson.jl:65-84) into qpart.
* advance_deposit: advance! + density! of the post-step state in one kernel.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
from scipy.special import erf

from . import _lib as L
from . import constants as co
from .jumc import ParticleArrays, Context, Population


class DeviceArray:
    """A 1-D device buffer owned by the library, described by __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


class Grid3D:
    """nx*ny*nz cubic cells of side h with lower corner `origin`; nodes (nx+1)(ny+1)(nz+1)."""

    # the C handle is .h_ (.h is the cell size)
    def __init__(self, nx: int, ny: int, nz: int, h: float, origin: Sequence[float] = (0.0, 0.0, 0.0),
                 precision: str = "fp32", ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        self.nx, self.ny, self.nz, self.h = int(nx), int(ny), int(nz), float(h)
        self.origin = tuple(float(o) for o in origin)
        self.precision = precision
        hd = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_grid_create_cart3d(
            self.ctx.h, self.nx, self.ny, self.nz, self.h, *self.origin,
            L.FP32 if precision == "fp32" else L.FP64, C.byref(hd)))
        self.h_ = hd

    @property
    def nnodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    @property
    def shape_nodes(self):
        return (self.nz + 1, self.ny + 1, self.nx + 1)

    def node_coords(self, k0: int, k1: int):
        """Coordinates of nodes with z-plane index in [k0, k1), x fastest."""
        x = self.origin[0] + self.h * np.arange(self.nx + 1)
        y = self.origin[1] + self.h * np.arange(self.ny + 1)
        z = self.origin[2] + self.h * np.arange(k0, k1)
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        return X.ravel(), Y.ravel(), Z.ravel()

    def set_efield(self, e: np.ndarray) -> None:
        e = np.ascontiguousarray(e, dtype=np.float64).reshape(-1)
        assert e.size == 3 * self.nnodes
        self.ctx.check(self.ctx.lib.mcs_grid_set_efield(self.h_, L.dptr(e)))

    def set_efield_fn(self, fn, planes_per_chunk: int = 16) -> None:
        """Fill the node field plane by plane from fn(x, y, z) -> (n, 3)."""
        plane = (self.nx + 1) * (self.ny + 1)
        for k0 in range(0, self.nz + 1, planes_per_chunk):
            k1 = min(self.nz + 1, k0 + planes_per_chunk)
            x, y, z = self.node_coords(k0, k1)
            e = np.ascontiguousarray(fn(x, y, z), dtype=np.float64)
            self.ctx.check(self.ctx.lib.mcs_grid_set_efield_range(self.h_, k0 * plane, (k1 - k0) * plane,
                                                                  L.dptr(e)))

    def set_efield_gaussian(self, centre: Sequence[float], sigma: float, rho_peak_e: float,
                            e_bg: Sequence[float] = (0.0, 0.0, 0.0)) -> None:
        """The field of gaussian_charge_field(centre, sigma, rho_peak_e, e_bg), computed on the device."""
        self.ctx.check(self.ctx.lib.mcs_grid_set_efield_gaussian(self.h_, *map(float, centre), float(sigma),
                                                                 float(rho_peak_e), *map(float, e_bg)))

    def read_efield(self) -> np.ndarray:
        out = np.zeros((self.nnodes, 3))
        self.ctx.check(self.ctx.lib.mcs_grid_read_efield(self.h_, L.dptr(out)))
        return out

    def zero(self, which: int = L.Q_PART) -> None:
        self.ctx.check(self.ctx.lib.mcs_grid_zero(self.h_, which))

    def read_fixed(self, which: int = L.Q_PART) -> np.ndarray:
        out = np.zeros(self.nnodes, dtype=np.int64)
        self.ctx.check(self.ctx.lib.mcs_grid_read_fixed(self.h_, which, L.i64ptr(out)))
        return out

    def _box_planes(self, lo, hi, read_plane):
        """Nodes lo..hi (inclusive, (ix, iy, iz)) read z-plane by z-plane, x fastest."""
        plane = (self.nx + 1) * (self.ny + 1)
        out = []
        for k in range(lo[2], hi[2] + 1):
            a = read_plane(k * plane, plane).reshape(self.ny + 1, self.nx + 1, -1)
            out.append(a[lo[1]:hi[1] + 1, lo[0]:hi[0] + 1])
        return np.ascontiguousarray(np.stack(out))

    def read_efield_box(self, lo, hi) -> np.ndarray:
        """The node field of the box of nodes lo..hi (inclusive), (nodes, 3), x fastest."""
        def rd(node0, count):
            e = np.zeros((count, 3))
            self.ctx.check(self.ctx.lib.mcs_grid_read_efield_range(self.h_, node0, count, L.dptr(e)))
            return e
        return self._box_planes(lo, hi, rd).reshape(-1, 3)

    def read_fixed_box(self, which: int, lo, hi) -> np.ndarray:
        """The int64 charges of the box of nodes lo..hi (inclusive), x fastest."""
        def rd(node0, count):
            q = np.zeros(count, dtype=np.int64)
            self.ctx.check(self.ctx.lib.mcs_grid_read_fixed_range(self.h_, which, node0, count, L.i64ptr(q)))
            return q
        return self._box_planes(lo, hi, rd).reshape(-1)

    def read_fixed_planes(self, which: int, out: np.ndarray, filled=(0, 0)) -> tuple:
        """Bring a charge array into the full host array `out` moving only the z-planes that
        hold charge: the device finds their range, that slab is copied, and the planes of
        `filled` (the range an earlier call on the same `out` returned) outside it are zeroed on
        the host.  `out` must hold zeros outside `filled`.  Returns the new filled range; `out`
        then equals read_fixed(which) node for node."""
        plane = (self.nx + 1) * (self.ny + 1)
        z0, z1 = C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_grid_fixed_plane_range(self.h_, which, C.byref(z0), C.byref(z1)))
        z0, z1 = z0.value, z1.value
        if z1 > z0:
            view = out[z0 * plane:z1 * plane]
            self.ctx.check(self.ctx.lib.mcs_grid_read_fixed_range(self.h_, which, z0 * plane, (z1 - z0) * plane,
                                                                  L.i64ptr(view)))
        f0, f1 = filled
        if f1 > f0:   # planes of the earlier slab that are now empty
            if z1 <= z0:
                out[f0 * plane:f1 * plane] = 0
            else:
                if f0 < z0:
                    out[f0 * plane:min(f1, z0) * plane] = 0
                if f1 > z1:
                    out[max(f0, z1) * plane:f1 * plane] = 0
        return (z0, z1)

    def charge_array(self, which: int = L.Q_PART) -> "DeviceArray":
        """The device int64 charge array, exposed through __cuda_array_interface__ (so a
        collective library can sum it across processes in place)."""
        p = C.c_void_p()
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.mcs_grid_charge_ptr(self.h_, which, C.byref(p), C.byref(n)))
        return DeviceArray(p.value, n.value, "<i8")

    def cell_key(self, x: np.ndarray) -> np.ndarray:
        u = (np.asarray(x) - np.asarray(self.origin)) / self.h
        fl = np.floor(u).astype(np.int64)
        inside = np.all((fl >= 0) & (fl < np.array([self.nx, self.ny, self.nz])), axis=1)
        key = fl[:, 0] + self.nx * (fl[:, 1] + self.ny * fl[:, 2])
        return np.where(inside, key, np.iinfo(np.int64).max)

    def close(self) -> None:
        if self.h_:
            self.ctx.lib.mcs_grid_destroy(self.h_)
            self.h_ = None


class GridCyl:
    """Cylindrical Grid(R, L, M, N) (MCStreamer/src/grid.jl:4-42)."""

    def __init__(self, R: float, L_: float, M: int, N: int, ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        self.R, self.L, self.M, self.N = float(R), float(L_), int(M), int(N)
        hd = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_grid_create_cyl(self.ctx.h, self.R, self.L, self.M, self.N, C.byref(hd)))
        self.h_ = hd

    def set_efield(self, er: np.ndarray, ez: np.ndarray) -> None:
        """er, ez: (M+3, N+3) face arrays, index (i, j) from 0 (calloc_faces, grid.jl:71-72)."""
        e = np.concatenate([np.asarray(er, np.float64).T.ravel(), np.asarray(ez, np.float64).T.ravel()])
        self.ctx.check(self.ctx.lib.mcs_grid_set_efield(self.h_, L.dptr(np.ascontiguousarray(e))))

    def zero(self, which: int = L.Q_PART) -> None:
        self.ctx.check(self.ctx.lib.mcs_grid_zero(self.h_, which))

    def read_density(self, which: int = L.Q_PART) -> np.ndarray:
        out = np.zeros((self.M + 2) * (self.N + 2))
        self.ctx.check(self.ctx.lib.mcs_grid_read_density(self.h_, which, L.dptr(out)))
        return out.reshape(self.N + 2, self.M + 2).T   # (i, j) like calloc_centers

    def write_fixed(self, which: int, q: np.ndarray) -> None:
        """Overwrite the int64 cell charges (2^-32 e), flat, index i + j*(M+2)."""
        q = np.ascontiguousarray(q, dtype=np.int64)
        if q.size != (self.M + 2) * (self.N + 2):
            raise ValueError("charge array of the wrong size")
        self.ctx.check(self.ctx.lib.mcs_grid_write_fixed(self.h_, which, L.i64ptr(q)))

    def read_qfixed_density(self) -> np.ndarray:
        """qfixed's FP64 density part (setneedle!, initfromfiles!), (M+2, N+2) like
        calloc_centers."""
        out = np.zeros((self.M + 2) * (self.N + 2))
        self.ctx.check(self.ctx.lib.mcs_grid_read_qfixed_density(self.h_, L.dptr(out)))
        return out.reshape((self.M + 2, self.N + 2), order="F")

    def write_qfixed_density(self, a: np.ndarray) -> None:
        a = np.asarray(a, dtype=np.float64)
        if a.shape != (self.M + 2, self.N + 2):
            raise ValueError(f"expected shape {(self.M + 2, self.N + 2)}, got {a.shape}")
        flat = np.ascontiguousarray(a.ravel(order="F"))
        self.ctx.check(self.ctx.lib.mcs_grid_write_qfixed_density(self.h_, L.dptr(flat)))

    def read_fixed(self, which: int = L.Q_PART) -> np.ndarray:
        """The int64 cell charges (2^-32 e), flat, index i + j*(M+2)."""
        out = np.zeros((self.M + 2) * (self.N + 2), dtype=np.int64)
        self.ctx.check(self.ctx.lib.mcs_grid_read_fixed(self.h_, which, L.i64ptr(out)))
        return out

    def close(self) -> None:
        if self.h_:
            self.ctx.lib.mcs_grid_destroy(self.h_)
            self.h_ = None


def _handle(g):
    return g.h_ if g is not None else None


class FieldInterp:
    """FieldInterp (gridfields.jl:89-190): the field stored on a grid."""

    def __init__(self, grid):
        self.grid = grid
        self.ctx = grid.ctx
        hd = C.c_void_p()
        self.ctx.check(self.ctx.lib.mcs_field_from_grid(grid.h_, C.byref(hd)))
        self.h = hd

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_field_destroy(self.h)
            self.h = None


class CollisionTracker:
    """CollisionTracker (gridfields.jl:198-224): +w per ionization, -w per attachment."""

    def __init__(self, grid):
        self.grid = grid
        self.h = grid.h_


def density(grid, popl: Population, val: float = 1.0) -> None:
    """density!(grid, arr=qpart, mpopl, Electron, fields, val) (poisson.jl:65-84)."""
    popl.ctx.check(popl.ctx.lib.mcs_deposit(popl.h, grid.h_, float(val)))


def advance_deposit(popl: Population, efield: FieldInterp, dt: float, tracker: Optional[CollisionTracker],
                    grid: Grid3D, val: float = -1.0) -> None:
    """advance!(...) then density!(qpart, val) of the post-step particles, one kernel."""
    popl.ctx.check(popl.ctx.lib.mcs_advance_deposit(popl.h, popl.collisions.h, efield.h, dt,
                                                    tracker.h if tracker is not None else None, grid.h_,
                                                    float(val)))


def advance_deposit_host(work: Population, efield: FieldInterp, dt: float, tracker: Optional[CollisionTracker],
                         grid: Grid3D, host: ParticleArrays, n: int, val: float = -1.0, chunks: int = 4) -> int:
    """advance_deposit of a host-resident population (arrays of `host`, capacity len(host.w),
    first n in use): stepped and written back in place with the transfers pipelined over
    `chunks` pieces; `work` is the device workspace.  Returns the new particle count."""
    nn = C.c_int64(int(n))
    work.ctx.check(work.ctx.lib.mcs_advance_deposit_host(
        work.h, work.collisions.h, efield.h, dt, tracker.h if tracker is not None else None, grid.h_, float(val),
        L.dptr(host.x), L.dptr(host.v), L.dptr(host.w), L.dptr(host.s), L.u8ptr(host.active), C.byref(nn),
        len(host.w), int(chunks)))
    return nn.value


def host_step_bytes(work: Population) -> tuple:
    """(host -> device, device -> host) bytes that the last advance_deposit_host call with
    this workspace copied (mcs_pop_host_step_bytes)."""
    up, down = C.c_int64(), C.c_int64()
    work.ctx.check(work.ctx.lib.mcs_pop_host_step_bytes(work.h, C.byref(up), C.byref(down)))
    return up.value, down.value


def resample(popl: Population, grid, ntarget: int, nmax: int) -> None:
    """resample!(popl, fields, ntarget, nmax) (MCStreamer/src/resample.jl:7-77): the stable
    cell sort, then the per-cell roulette and splitting."""
    popl.ctx.check(popl.ctx.lib.mcs_resample_cells(popl.h, grid.h_, int(ntarget), int(nmax)))


def reserve_resample(popl: Population) -> None:
    """Allocate the device scratch of resample! (the cell sort's keys and second population
    arrays, the segment tables) for the population's capacity now, so that no later
    resample! allocates inside a time step."""
    popl.ctx.check(popl.ctx.lib.mcs_resample_reserve(popl.h))


def diagnostics(popl: Population, photons=None) -> dict:
    """The per-step diagnostics of nsteps (MCStreamer/src/main.jl:269-279): meanenergy and
    maxenergy of the electrons (J), their actives and weight, and the photons' actives and
    weight (zero without active photons).  Device reductions: FP64 sums in a fixed order."""
    m = popl.moments()
    ph = photons.moments() if photons is not None else np.zeros(2)
    with np.errstate(invalid="ignore", divide="ignore"):
        mean = np.float64(m[L.M_WE]) / np.float64(m[L.M_W])
    return {"mean_energy": float(mean), "max_energy": float(m[L.M_EMAX]),
            "active_superelectrons": int(m[L.M_COUNT]), "physical_electrons": float(m[L.M_W]),
            "active_superphotons": int(ph[0]), "physical_photons": float(ph[1]) if ph[0] > 0 else 0.0}


# ---------------------------------------------------------------------------------------
# Field of the streamer workloads: a uniform background plus a Gaussian charge cloud.
# ---------------------------------------------------------------------------------------
def gaussian_charge_field(centre: Sequence[float], sigma: float, rho_peak_e: float, e_bg=(0.0, 0.0, -15e6)):
    """E = e_bg + Q(r)/(4 pi eps0 r^2) r_hat for rho = e*rho_peak_e*exp(-r^2/2sigma^2):
    Q(r) = e*rho_peak_e*(2 pi sigma^2)^(3/2) [erf(r/(sqrt2 sigma)) - sqrt(2/pi)(r/sigma) exp(-r^2/2sigma^2)]."""
    cx, cy, cz = centre
    q0 = co.elementary_charge * rho_peak_e * (2 * np.pi * sigma ** 2) ** 1.5

    def fn(x, y, z):
        dx, dy, dz = x - cx, y - cy, z - cz
        r = np.sqrt(dx * dx + dy * dy + dz * dz)
        rs = r / sigma
        Q = q0 * (erf(rs / np.sqrt(2)) - np.sqrt(2 / np.pi) * rs * np.exp(-0.5 * rs * rs))
        with np.errstate(invalid="ignore", divide="ignore"):
            f = np.where(r > 0, Q / (4 * np.pi * co.epsilon_0 * r ** 3), 0.0)
        return np.stack([e_bg[0] + f * dx, e_bg[1] + f * dy, e_bg[2] + f * dz], axis=1)

    return fn
