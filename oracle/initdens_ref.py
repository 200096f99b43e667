"""CPU restatement of MCStreamer's initfromfiles! (MCStreamer/src/initdens.jl:64-159) --
TEST INFRASTRUCTURE (the checker, never the product).  The loop is orc_init_from_density in
oracle.cpp; this module is its numpy-facing wrapper."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import pyoracle

NOISELESS, POISSON = 0, 1
_pd = C.POINTER(C.c_double)
_ready = False


def _lib():
    global _ready
    L = pyoracle.lib()
    if not _ready:
        L.orc_init_from_density.restype = C.c_int64
        L.orc_init_from_density.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _pd, _pd, C.c_int, C.c_int64,
                                            C.c_double, C.c_uint64, C.c_int64, _pd, _pd, _pd, _pd, _pd]
        _ready = True
    return L


def initfromfiles(ne, q, R, L, M, N, method, p, fluid_threshold=np.inf, seed=0, cap=None, qfd=None, ne_fluid=None):
    """Returns (x (n, 3), w, s, qfd (M+2, N+2), ne_fluid (M+4, N+4)); n = -1 with empty arrays
    when more than cap electrons would be sampled.  ne, q: (M, N) arrays."""
    ne = np.ascontiguousarray(np.asarray(ne, dtype=np.float64).ravel(order="F"))
    q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel(order="F"))
    cap = int(cap if cap is not None else 4 * p * M * N + 16)
    x = np.zeros((cap, 3))
    w = np.zeros(cap)
    s = np.zeros(cap)
    qfd = np.zeros((M + 2, N + 2), order="F") if qfd is None else qfd
    ne_fluid = np.zeros((M + 4, N + 4), order="F") if ne_fluid is None else ne_fluid
    n = _lib().orc_init_from_density(M, N, R, L, ne.ctypes.data_as(_pd), q.ctypes.data_as(_pd), method, p,
                                     fluid_threshold, seed, cap, x.ctypes.data_as(_pd), w.ctypes.data_as(_pd),
                                     s.ctypes.data_as(_pd), qfd.ctypes.data_as(_pd), ne_fluid.ctypes.data_as(_pd))
    if n < 0:
        return -1, None, None, qfd, ne_fluid
    return x[:n], w[:n], s[:n], qfd, ne_fluid
