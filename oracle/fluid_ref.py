"""CPU restatement of MCStreamer's electron fluid (MCStreamer/src/fluid.jl) -- TEST
INFRASTRUCTURE (the checker, never the product).  The loops are fluid.cpp in liboracle.so;
this module holds the numpy-facing wrappers.

Arrays are Fortran-ordered numpy arrays: ne, dne (M+4)x(N+4) (calloc_centers with two ghost
layers: ne[i + 1, j + 1] is the reference's ne[i, j]); er, ez (M+3)x(N+3) faces; qfd
(M+2)x(N+2), the FP64 density part of qfixed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import pyoracle

NAIR = 2.6867811e+25                 # JuMC/src/constants.jl:149
MOBILITY = 1e24 / NAIR               # setdne!'s default (fluid.jl:44)

_pd = C.POINTER(C.c_double)
_ready = False


def _lib():
    global _ready
    L = pyoracle.lib()
    if not _ready:
        L.orc_fluid_needle.argtypes = [C.c_int, C.c_int] + [C.c_double] * 7 + [_pd, _pd]
        L.orc_fluid_setnebc.argtypes = [C.c_int, C.c_int, _pd]
        L.orc_fluid_setdne.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _pd, _pd, _pd, _pd]
        L.orc_fluid_euler.argtypes = [C.c_int, C.c_int, C.c_double, _pd, _pd]
        L.orc_fluid_koren.restype = C.c_double
        L.orc_fluid_koren.argtypes = [C.c_double]
        _ready = True
    return L


def _p(a):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_pd)


def centers(M, N):
    return np.zeros((M + 4, N + 4), order="F")


def setneedle(ne, qfd, R, L, M, N, sigma_z, sigma_r, position_z, position_r, ne0):
    _lib().orc_fluid_needle(M, N, R, L, sigma_z, sigma_r, position_z, position_r, ne0, _p(ne), _p(qfd))


def setnebc(ne, M, N):
    _lib().orc_fluid_setnebc(M, N, _p(ne))


def setdne(ne, dne, er, ez, R, L, M, N, mobility=MOBILITY):
    _lib().orc_fluid_setdne(M, N, R, L, mobility, _p(ne), _p(dne), _p(er), _p(ez))


def euler(ne, dne, dt, M, N):
    _lib().orc_fluid_euler(M, N, dt, _p(ne), _p(dne))


def koren(theta: float) -> float:
    return _lib().orc_fluid_koren(theta)
