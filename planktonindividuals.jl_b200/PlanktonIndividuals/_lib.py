"""Loads libpib200.so, the CUDA (sm_100a) implementation behind this package.

There is no CPU fallback: if the library is missing or no CUDA device can be used, model
construction raises. Build it with `python planktonindividuals.jl_b200/build.py`."""
import ctypes as ct
import os

from . import _abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpib200.so")
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libpib200.so not found at {LIB_PATH}; build it with "
                          f"`python planktonindividuals.jl_b200/build.py` (the package has no CPU fallback)")
    lib = ct.CDLL(LIB_PATH)
    _abi.declare(lib, "pi_")
    P = ct.c_void_p
    dp = ct.POINTER(ct.c_double)
    lib.pi_sim_create.restype = ct.c_int32
    lib.pi_sim_create.argtypes = [P, ct.c_double, ct.c_int64, dp, dp, dp, ct.c_int64, ct.c_double,
                                  dp, ct.c_int64, ct.c_double, dp, ct.c_int64, ct.c_double,
                                  ct.POINTER(P)]
    lib.pi_sim_update.restype = ct.c_int32
    lib.pi_sim_update.argtypes = [P, ct.c_int32, ct.c_int32]
    lib.pi_sim_destroy.restype = ct.c_int32
    lib.pi_sim_destroy.argtypes = [P]
    lib.pi_synchronize.restype = ct.c_int32
    lib.pi_synchronize.argtypes = [P]
    lib.pi_reset_diags.restype = ct.c_int32
    lib.pi_reset_diags.argtypes = [P]
    lib.pi_get_stream.restype = ct.c_int32
    lib.pi_get_stream.argtypes = [P, ct.POINTER(ct.c_void_p)]
    lib.pi_profile_enable.restype = ct.c_int32
    lib.pi_profile_enable.argtypes = [P, ct.c_int32]
    lib.pi_profile_read.restype = ct.c_int32
    lib.pi_profile_read.argtypes = [P, ct.c_int32, ct.c_char_p, ct.c_size_t, ct.POINTER(ct.c_int64),
                                    dp, ct.POINTER(ct.c_int32)]
    lib.pi_status_string.restype = ct.c_char_p
    lib.pi_status_string.argtypes = [ct.c_int32]
    _declare_batch(lib)
    _lib = lib
    return lib


def _declare_batch(lib):
    P = ct.c_void_p
    dp = ct.POINTER(ct.c_double)
    i32, i64 = ct.c_int32, ct.c_int64
    pind = ct.POINTER(_abi.pi_individuals)
    protos = {
        "pi_batch_create": [ct.POINTER(_abi.pi_member), i32, i32, ct.POINTER(P)],
        "pi_batch_destroy": [P],
        "pi_batch_set_individuals": [P, i32, i32, pind],
        "pi_batch_get_individuals": [P, i32, i32, pind],
        "pi_batch_set_tracer": [P, i32, i32, dp],
        "pi_batch_get_tracer": [P, i32, i32, dp],
        "pi_batch_set_velocity": [P, i32, dp, dp, dp],
        "pi_batch_set_velocity0": [P, i32, dp, dp, dp],
        "pi_batch_set_PARF": [P, i32, dp],
        "pi_batch_set_temp": [P, i32, dp],
        "pi_batch_set_flux_bc": [P, i32, i32, i32, i32, dp, i64],
        "pi_batch_set_series": [P, i32, dp, dp, dp, i64, ct.c_double, dp, i64, ct.c_double, dp, i64,
                                ct.c_double, i32],
        "pi_batch_set_time_offset": [P, i32, i32],
        "pi_batch_clear_series": [P, i32],
        "pi_batch_step": [P, ct.c_double, i64, i32],
        "pi_batch_synchronize": [P],
        "pi_batch_get_time": [P, ct.POINTER(i64), dp],
        "pi_batch_set_time": [P, i64, ct.c_double],
        "pi_batch_count_active": [P, i32, i32, ct.POINTER(i64)],
        "pi_batch_get_diag": [P, i32, i32, i32, dp],
        "pi_batch_reset_diags": [P],
        "pi_batch_budget": [P, i32, dp],
        "pi_batch_autotune": [P, ct.c_double, i32, ct.c_char_p, ct.c_size_t],
        "pi_batch_get_stream": [P, ct.POINTER(P)],
        "pi_batch_profile_enable": [P, i32],
        "pi_batch_profile_read": [P, i32, ct.c_char_p, ct.c_size_t, ct.POINTER(i64), dp, ct.POINTER(i32)],
        "pi_batch_last_error": [P, ct.c_char_p, ct.c_size_t],
    }
    for name, args in protos.items():
        fn = getattr(lib, name)
        fn.restype = ct.c_int32
        fn.argtypes = args


# Exported entry points of include/pib200.h (checked by the CPU test suite).
EXPORTS = ("pi_create", "pi_destroy", "pi_set_individuals", "pi_get_individuals", "pi_set_tracer",
           "pi_get_tracer", "pi_set_velocity", "pi_set_velocity0", "pi_set_PARF", "pi_set_temp", "pi_set_flux_bc",
           "pi_time_step", "pi_get_time", "pi_set_time", "pi_count_active", "pi_get_diag",
           "pi_reset_diags", "pi_sim_create", "pi_sim_update", "pi_sim_destroy", "pi_synchronize",
           "pi_last_error", "pi_status_string", "pi_get_stream", "pi_profile_enable", "pi_profile_read",
           "pi_tracer_advection_noalloc", "pi_noalloc_last_error",
           "pi_batch_create", "pi_batch_destroy", "pi_batch_set_individuals", "pi_batch_get_individuals",
           "pi_batch_set_tracer", "pi_batch_get_tracer", "pi_batch_set_velocity", "pi_batch_set_velocity0",
           "pi_batch_set_PARF", "pi_batch_set_temp", "pi_batch_set_flux_bc", "pi_batch_set_series",
           "pi_batch_set_time_offset", "pi_batch_clear_series", "pi_batch_step", "pi_batch_synchronize",
           "pi_batch_get_time", "pi_batch_set_time", "pi_batch_count_active", "pi_batch_get_diag",
           "pi_batch_reset_diags", "pi_batch_budget", "pi_batch_autotune", "pi_batch_get_stream",
           "pi_batch_profile_enable", "pi_batch_profile_read", "pi_batch_last_error",
           "pi_batch_set_sort_interval", "pi_check_finite", "pi_batch_check_finite",
           "pi_set_velocity_f32", "pi_set_PARF_f32", "pi_set_temp_f32", "pi_time_step_async",
           "pi_count_active_async", "pi_batch_set_velocity_f32", "pi_batch_set_PARF_f32", "pi_batch_set_temp_f32",
           "pi_batch_count_active_async", "pi_batch_guard_stats",
           "pi_set_diags", "pi_batch_set_diags", "pi_sim_update_steps", "pi_batch_step_from", "pi_get_budget", "pi_batch_set_tracer_kernel", "pi_selftest_bounded_wait", "pi_batch_set_option")
