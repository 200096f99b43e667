"""ctypes binding of libmcs_b200.so (the C ABI declared in include/mcs.h).

This is the same binding a Julia caller writes with ccall; the Python classes in
jumc.py / swarm.py / streamer.py sit on top of it.  Loading fails loudly: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmcs_b200.so"

# status codes (include/mcs.h)
OK, ERR_ARG, ERR_CUDA, ERR_CAPACITY, ERR_ENERGY_RANGE, ERR_FIELD_TOO_HIGH = 0, 1, 2, 3, 4, 5
ERR_NONFINITE, ERR_UNSUPPORTED, ERR_OVERFLOW, ERR_NOMEM, ERR_TIMEOUT, ERR_UNIFORMS = 6, 7, 8, 9, 10, 11
ERR_CHARGE_RANGE = 12
STATUS_NAMES = {
    0: "MCS_OK", 1: "MCS_ERR_ARG", 2: "MCS_ERR_CUDA", 3: "MCS_ERR_CAPACITY", 4: "MCS_ERR_ENERGY_RANGE",
    5: "MCS_ERR_FIELD_TOO_HIGH", 6: "MCS_ERR_NONFINITE", 7: "MCS_ERR_UNSUPPORTED", 8: "MCS_ERR_OVERFLOW",
    9: "MCS_ERR_NOMEM", 10: "MCS_ERR_TIMEOUT", 11: "MCS_ERR_UNIFORMS", 12: "MCS_ERR_CHARGE_RANGE",
}
UNIFORMS_PHILOX, UNIFORMS_INJECTED = 0, 1
# process kinds
NULL, ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, IONIZATION_UNIFORM, PHOTOEMISSION = 0, 1, 2, 3, 4, 5, 6
FP64, FP32 = 0, 1
FLAG_CLAMP_ENERGY = 1
Q_FIXED, Q_PART = 0, 1
PSN_U, PSN_B, PSN_BCOND, PSN_FREEBC_F = 0, 1, 2, 3
INIT_NOISELESS, INIT_POISSON = 0, 1
MOMENTS_BASE = 18
M_COUNT, M_W, M_X, M_X2, M_V, M_E, M_WE, M_EMAX, M_WX, M_WX2 = 0, 1, 2, 5, 8, 11, 12, 13, 14, 17
S_COUNT, S_W, S_X, S_X2, S_V, S_E, STEP_MOMENTS = 0, 1, 2, 5, 8, 11, 12
B_NU, B_NU2, BATCH_MOMENTS, BATCH_LOG, BATCH_VARIANTS = 12, 13, 14, 64, 22
OPT_MESH_SHAPE, MESH_SHAPES = 1, 8

vp = C.c_void_p
i32, i64, u32, u64, f64 = C.c_int, C.c_int64, C.c_uint32, C.c_uint64, C.c_double
pd = C.POINTER(C.c_double)
pi64 = C.POINTER(C.c_int64)
pu8 = C.POINTER(C.c_uint8)
pi32 = C.POINTER(C.c_int)
ph = C.POINTER(C.c_void_p)

SIGNATURES = {
    "mcs_version": (i32, []),
    "mcs_ctx_create": (i32, [i32, ph]),
    "mcs_ctx_destroy": (i32, [vp]),
    "mcs_last_error": (C.c_char_p, [vp]),
    "mcs_ctx_set_stream": (i32, [vp, vp]),
    "mcs_ctx_stream": (vp, [vp]),
    "mcs_ctx_set_flags": (i32, [vp, u32]),
    "mcs_sync": (i32, [vp]),
    "mcs_table_create": (i32, [vp, i32, i32, f64, f64, pd, pi32, pd, f64, ph]),
    "mcs_table_destroy": (i32, [vp]),
    "mcs_grid_create_cart3d": (i32, [vp, i32, i32, i32, f64, f64, f64, f64, i32, ph]),
    "mcs_grid_create_cyl": (i32, [vp, f64, f64, i32, i32, ph]),
    "mcs_grid_destroy": (i32, [vp]),
    "mcs_grid_set_efield": (i32, [vp, pd]),
    "mcs_grid_set_efield_range": (i32, [vp, i64, i64, pd]),
    "mcs_grid_zero": (i32, [vp, i32]),
    "mcs_grid_read_fixed": (i32, [vp, i32, pi64]),
    "mcs_grid_read_density": (i32, [vp, i32, pd]),
    "mcs_grid_read_efield_range": (i32, [vp, i64, i64, pd]),
    "mcs_grid_read_fixed_range": (i32, [vp, i32, i64, i64, pi64]),
    "mcs_grid_fixed_plane_range": (i32, [vp, i32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mcs_grid_charge_ptr": (i32, [vp, i32, ph, pi64]),
    "mcs_field_uniform": (i32, [vp, f64, f64, f64, ph]),
    "mcs_field_from_grid": (i32, [vp, ph]),
    "mcs_field_destroy": (i32, [vp]),
    "mcs_pop_create": (i32, [vp, i64, i32, vp, ph]),
    "mcs_pop_destroy": (i32, [vp]),
    "mcs_pop_set_seed": (i32, [vp, u64, u32]),
    "mcs_pop_get_step": (i32, [vp, C.POINTER(C.c_uint32)]),
    "mcs_pop_upload": (i32, [vp, pd, pd, pd, pd, pu8, i64]),
    "mcs_pop_download": (i32, [vp, pd, pd, pd, pd, pu8, i64, pi64]),
    "mcs_pop_nparticles": (i32, [vp, pi64]),
    "mcs_pop_copy": (i32, [vp, vp]),
    "mcs_advance": (i32, [vp, vp, vp, f64, vp]),
    "mcs_advance_deposit": (i32, [vp, vp, vp, f64, vp, vp, f64]),
    "mcs_advance_deposit_host": (i32, [vp, vp, vp, f64, vp, vp, f64, pd, pd, pd, pd, pu8, pi64, i64, i32]),
    "mcs_pop_host_step_bytes": (i32, [vp, pi64, pi64]),
    "mcs_collisions": (i32, [vp, vp, f64, vp]),
    "mcs_set_uniform_source": (i32, [vp, i32, pd, pi64, i64]),
    "mcs_deposit": (i32, [vp, vp, f64]),
    "mcs_repack": (i32, [vp]),
    "mcs_swarm_resample": (i32, [vp, i64, f64]),
    "mcs_sort_cells": (i32, [vp, vp]),
    "mcs_resample_cells": (i32, [vp, vp, i32, i32]),
    "mcs_resample_reserve": (i32, [vp]),
    "mcs_moments": (i32, [vp, vp, pd, i32]),
    "mcs_swarm_run": (i32, [vp, vp, vp, f64, i32, i64, f64, i32, pd]),
    "mcs_pop_step_log": (i32, [vp, i32]),
    "mcs_moments_noalloc": (i32, [i32, vp, i32, C.POINTER(C.c_void_p), pu8, i64, pd]),
    "mcs_ctx_set_option": (i32, [vp, i32, i32]),
    "mcs_diag_wait_timeout": (i32, [vp, u32]),
    "mcs_ctx_get_option": (i32, [vp, i32, pi32]),
    "mcs_mesh_shape": (i32, [i32, pi32, pi32, pi32]),
    "mcs_batch_create": (i32, [vp, i32, i64, ph]),
    "mcs_batch_destroy": (i32, [vp]),
    "mcs_batch_add": (i32, [vp, vp, f64, f64, f64, u64, i64, f64, i64, pd, pd, pd, pd, pu8, i64, pi32]),
    "mcs_batch_remove": (i32, [vp, i32]),
    "mcs_batch_add_maxwellian": (i32, [vp, vp, f64, f64, f64, u64, i64, f64, i64, i64, f64, pi32]),
    "mcs_batch_logs_enqueue": (i32, [vp, i32]),
    "mcs_batch_logs_wait": (i32, [vp, i32, C.POINTER(pd), C.POINTER(C.POINTER(C.c_uint32))]),
    "mcs_pop_init_maxwellian": (i32, [vp, i64, f64]),
    "mcs_pop_init_cloud": (i32, [vp, i64, f64, f64, f64, f64, f64, f64, f64]),
    "mcs_grid_set_efield_gaussian": (i32, [vp, f64, f64, f64, f64, f64, f64, f64, f64]),
    "mcs_grid_read_efield": (i32, [vp, pd]),
    "mcs_batch_step": (i32, [vp, f64, i32, i32]),
    "mcs_batch_sync": (i32, [vp]),
    "mcs_batch_state": (i32, [vp, pi64, C.POINTER(C.c_uint32)]),
    "mcs_batch_read_log": (i32, [vp, i32, pd, i32]),
    "mcs_batch_read_current": (i32, [vp, pd]),
    "mcs_batch_read_logs": (i32, [vp, pd, C.POINTER(C.c_uint32)]),
    "mcs_batch_download": (i32, [vp, i32, pd, pd, pd, pd, pu8, i64, pi64]),
    "mcs_batch_autotune": (i32, [vp, f64, i32, pi32, C.POINTER(C.c_float)]),
    "mcs_batch_profile": (i32, [vp, f64, i32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mcs_batch_set_variant": (i32, [vp, i32]),
    "mcs_batch_variant_shape": (i32, [i32, pi32, pi32]),
    "mcs_batch_variant_min_blocks": (i32, [i32, pi32]),
    "mcs_batch_variant_refill": (i32, [i32, pi32]),
    "mcs_pop_read_step_log": (i32, [vp, pd, i32]),
    "mcs_poisson_create": (i32, [vp, i32, i32, i32, i32, f64, f64, C.POINTER(C.c_void_p)]),
    "mcs_poisson_destroy": (i32, [vp]),
    "mcs_poisson_upload": (i32, [vp, i32, pd]),
    "mcs_poisson_download": (i32, [vp, i32, pd]),
    "mcs_poisson_mg_solve": (i32, [vp, pi32, pd]),
    "mcs_poisson_solve_freebc": (i32, [vp, pi32]),
    "mcs_poisson_assemble": (i32, [vp]),
    "mcs_poisson_fields": (i32, [vp, f64]),
    "mcs_poisson_run": (i32, [vp, f64, pi32]),
    "mcs_freebc_coefficients": (i32, [f64, f64, i32, pd]),
    "mcs_poisson_zero": (i32, [vp, i32]),
    "mcs_poisson_launches": (i32, [vp, pi64]),
    "mcs_poisson_profile": (i32, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mcs_grid_write_fixed": (i32, [vp, i32, pi64]),
    "mcs_fluid_create": (i32, [vp, C.POINTER(C.c_void_p)]),
    "mcs_fluid_destroy": (i32, [vp]),
    "mcs_fluid_upload": (i32, [vp, pd, pd]),
    "mcs_fluid_download": (i32, [vp, pd, pd, pd]),
    "mcs_fluid_set_needle": (i32, [vp, f64, f64, f64, f64, f64]),
    "mcs_fluid_derivatives": (i32, [vp, f64]),
    "mcs_fluid_euler": (i32, [vp, f64]),
    "mcs_fluid_step": (i32, [vp, f64, f64]),
    "mcs_fluid_launches": (i32, [vp, pi64]),
    "mcs_init_from_density": (i32, [vp, vp, pd, pd, i32, i64, f64, C.c_uint64, pi64]),
    "mcs_grid_read_qfixed_density": (i32, [vp, pd]),
    "mcs_grid_write_qfixed_density": (i32, [vp, pd]),
    "mcs_init_from_density_device": (i32, [vp, vp, vp, vp, i32, i64, f64, C.c_uint64, pi64]),
    "mcs_table_set_photoemission": (i32, [vp, pd, pd, f64, f64]),
    "mcs_photons_create": (i32, [vp, i64, f64, C.c_uint64, C.POINTER(C.c_void_p)]),
    "mcs_photons_destroy": (i32, [vp]),
    "mcs_photons_moments": (i32, [vp, pd]),
    "mcs_photons_repack": (i32, [vp]),
    "mcs_photons_upload": (i32, [vp, pd, pd, pd, pd, pd, pu8, i64]),
    "mcs_photons_download": (i32, [vp, pd, pd, pd, pd, pd, pu8, i64, pi64]),
    "mcs_photons_count": (i32, [vp, pi64]),
    "mcs_photons_copy": (i32, [vp, vp]),
    "mcs_photons_last_timing": (i32, [vp, C.POINTER(C.c_float), pi64, C.POINTER(C.c_float), pi64]),
    "mcs_advance_mixed": (i32, [vp, vp, vp, vp, f64, vp]),
    "mcs_photon_advance": (i32, [vp, vp, f64, vp]),
}

_lib = None


class MCSError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load libmcs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mcstreamer_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, ctx=None) -> None:
    if code != OK:
        msg = ""
        if ctx is not None:
            raw = lib().mcs_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise MCSError(code, msg)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(pd)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(pu8)


def i64ptr(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(pi64)


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(pi32)
