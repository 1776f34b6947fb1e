"""ctypes binding of librigidfibers.so (the C ABI declared in include/rigidfibers.h).

The library is the product path: there is no CPU fallback.  Importing this
module without the built library raises ImportError with the build command.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librigidfibers.so")

RF_OK, RF_E_INPUT, RF_E_CUDA, RF_E_OOM, RF_E_NOCONV, RF_E_NAN, RF_E_TIMEOUT, RF_E_UNSUPPORTED, RF_E_STATE, \
    RF_E_SINGULAR = range(10)
SOLVERS = {"gmres": 0, "bicgstab": 1, "direct": 2, "magma": 2}
INTEGRATIONS = {"numerical": 0, "analytical": 1}
PRECISIONS = {"fp32": 0, "mixed_fp16": 1, "mixed_bf16": 2, "matrix_free": 3,
              "mixed_fp16_recompute": 4, "mixed_bf16_recompute": 5}


class rf_config(ctypes.Structure):
    _fields_ = [
        ("number_of_timesteps", ctypes.c_int),
        ("state_save_interval", ctypes.c_int),
        ("velocity_save_interval", ctypes.c_int),
        ("timestep", ctypes.c_double),
        ("slenderness", ctypes.c_double),
        ("number_of_terms_in_force_expansion", ctypes.c_int),
        ("number_of_quadrature_intervals", ctypes.c_int),
        ("number_of_quadrature_points_per_interval", ctypes.c_int),
        ("gmres_restart", ctypes.c_int),
        ("gmres_max_iterations", ctypes.c_int),
        ("gmres_tolerance", ctypes.c_double),
        ("bicgstab_max_iterations", ctypes.c_int),
        ("bicgstab_tolerance", ctypes.c_double),
        ("solver", ctypes.c_int),
        ("integration", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("velocity_integration", ctypes.c_int),
        ("refinement_tolerance", ctypes.c_double),
        ("refinement_max_iterations", ctypes.c_int),
        ("refinement_restart", ctypes.c_int),
    ]


class rf_stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("restarts", ctypes.c_int),
        ("refinement_steps", ctypes.c_int),
        ("relative_residual", ctypes.c_double),
        ("ms_assemble_system", ctypes.c_double),
        ("ms_solve_system", ctypes.c_double),
        ("ms_update_velocities", ctypes.c_double),
        ("ms_update_fibers", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int),
        ("graph_replays", ctypes.c_int),
        ("factorizations", ctypes.c_int),
        ("pivoted", ctypes.c_int),
        ("max_multiplier", ctypes.c_double),
        ("ms_step", ctypes.c_double),
    ]


class rf_tune_report(ctypes.Structure):
    _fields_ = [
        ("matvec_variant", ctypes.c_int),
        ("matvec_ms", ctypes.c_double * 2),
        ("gemv_ctas_per_sm", ctypes.c_int),
        ("gemv_ms", ctypes.c_double * 4),
        ("cached", ctypes.c_int),
        ("panel_blocks", ctypes.c_int),
        ("panel_ms", ctypes.c_double * 3),
        ("asm_variant", ctypes.c_int),
        ("asm_ms", ctypes.c_double * 2),
    ]


RF_REQ_QUEUED, RF_REQ_RUNNING, RF_REQ_DONE, RF_REQ_FAILED, RF_REQ_CANCELLED = range(5)


class rf_server_config(ctypes.Structure):
    _fields_ = [("max_active", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_int64), ("use_cuda_graphs", ctypes.c_int),
                ("pack_max_fibers", ctypes.c_int), ("pack_max_members", ctypes.c_int),
                ("reserve_bytes", ctypes.c_int64)]


class rf_request_stats(ctypes.Structure):
    _fields_ = [
        ("steps_done", ctypes.c_int),
        ("queue_ms", ctypes.c_double),
        ("run_ms", ctypes.c_double),
        ("mean_step_ms", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
        ("setup_ms", ctypes.c_double),
    ]


class rf_server_stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64),
        ("p50_step_ms", ctypes.c_double),
        ("p99_step_ms", ctypes.c_double),
        ("fiber_steps", ctypes.c_int64),
        ("elapsed_s", ctypes.c_double),
        ("peak_active", ctypes.c_int),
        ("peak_bytes", ctypes.c_int64),
        ("completed", ctypes.c_int),
        ("failed", ctypes.c_int),
        ("queued", ctypes.c_int),
        ("active", ctypes.c_int),
        ("pack_steps", ctypes.c_int64),
        ("pack_p50_ms", ctypes.c_double),
        ("pack_p99_ms", ctypes.c_double),
        ("pack_max_ms", ctypes.c_double),
        ("pack_mean_members", ctypes.c_double),
        ("p50_setup_ms", ctypes.c_double), ("p99_setup_ms", ctypes.c_double),
    ]


# name -> (restype, argtypes); every entry point declared in include/rigidfibers.h
_P = ctypes.c_void_p
_H = ctypes.c_void_p
_S = ctypes.c_void_p
SIGNATURES = {
    "rf_config_default": (ctypes.c_int, [ctypes.POINTER(rf_config)]),
    "rf_create": (ctypes.c_int, [ctypes.POINTER(rf_config), ctypes.c_int, _P, _P, ctypes.POINTER(_H)]),
    "rf_destroy": (ctypes.c_int, [_H]),
    "rf_assemble": (ctypes.c_int, [_H]),
    "rf_solve": (ctypes.c_int, [_H]),
    "rf_update_velocities": (ctypes.c_int, [_H]),
    "rf_update_fibers": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_step": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_run": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int]),
    "rf_solve_packed": (ctypes.c_int, [ctypes.POINTER(_H), ctypes.c_int]),
    "rf_step_packed": (ctypes.c_int, [ctypes.POINTER(_H), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]),
    "rf_get_state": (ctypes.c_int, [_H, _P, _P]),
    "rf_set_state": (ctypes.c_int, [_H, _P, _P]),
    "rf_get_velocities": (ctypes.c_int, [_H, _P, _P]),
    "rf_get_system": (ctypes.c_int, [_H, _P, _P]),
    "rf_get_solution": (ctypes.c_int, [_H, _P]),
    "rf_last_stats": (ctypes.c_int, [_H, ctypes.POINTER(rf_stats)]),
    "rf_get_config": (ctypes.c_int, [_H, ctypes.POINTER(rf_config)]),
    "rf_number_of_fibers": (ctypes.c_int, [_H]),
    "rf_dense_matvec": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    "rf_dense_lu_solve": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, ctypes.c_double, _P]),
    "rf_dense_matvec_noalloc": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    "rf_operator_apply": (ctypes.c_int, [_H, _P, _P, ctypes.c_int]),
    "rf_get_stream": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_void_p)]),
    "rf_set_profiling": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_set_cuda_graphs": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_set_near_field_preconditioner": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_set_assembly_variant": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_prepare_step_graphs": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_set_host_wait": (ctypes.c_int, [_H, ctypes.c_int]),
    "rf_autotune": (ctypes.c_int, [_H, ctypes.POINTER(rf_tune_report)]),
    "rf_matvec_profile": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "rf_checkpoint_bytes": (ctypes.c_int64, [_H]),
    "rf_checkpoint_save": (ctypes.c_int, [_H, _P, ctypes.c_int64]),
    "rf_checkpoint_load": (ctypes.c_int, [_H, _P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "rf_device_bytes_estimate": (ctypes.c_int64, [ctypes.POINTER(rf_config), ctypes.c_int]),
    "rf_server_config_default": (ctypes.c_int, [ctypes.POINTER(rf_server_config)]),
    "rf_server_create": (ctypes.c_int, [ctypes.POINTER(rf_server_config), ctypes.POINTER(_S)]),
    "rf_server_submit": (ctypes.c_int, [_S, ctypes.POINTER(rf_config), ctypes.c_int, _P, _P, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int64)]),
    "rf_server_poll": (ctypes.c_int, [_S, ctypes.c_int64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "rf_server_cancel": (ctypes.c_int, [_S, ctypes.c_int64]),
    "rf_server_wait": (ctypes.c_int, [_S, ctypes.c_int64, ctypes.c_double]),
    "rf_server_drain": (ctypes.c_int, [_S, ctypes.c_double]),
    "rf_server_result": (ctypes.c_int, [_S, ctypes.c_int64, _P, _P, _P, _P, ctypes.POINTER(rf_request_stats)]),
    "rf_server_get_stats": (ctypes.c_int, [_S, ctypes.POINTER(rf_server_stats)]),
    "rf_server_step_times": (ctypes.c_int, [_S, ctypes.c_int64, _P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "rf_server_destroy": (ctypes.c_int, [_S]),
    "rf_debug_set_device_wait_limit": (ctypes.c_int, [ctypes.c_int64]),
    "rf_debug_fail_allocation_after": (ctypes.c_int, [ctypes.c_int]),
    "rf_debug_noalloc_plan": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int64)]),
    "rf_debug_pack_plan": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]),
    "rf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rf_last_error": (ctypes.c_char_p, []),
}

_lib = None


def load():
    """Load the library (once).  Raises ImportError if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("librigidfibers.so not built: run `python -m rigidfibers_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class RigidFibersError(RuntimeError):
    def __init__(self, status, where):
        lib = load()
        msg = lib.rf_status_string(status).decode()
        detail = lib.rf_last_error().decode()
        super().__init__("%s: %s (%d)%s" % (where, msg, status, ": " + detail if detail else ""))
        self.status = status


def check(status, where, allow=()):
    if status != RF_OK and status not in allow:
        raise RigidFibersError(status, where)
    return status


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def f64(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.size != n:
        raise ValueError("expected %d values, got %d" % (n, a.size))
    return a
