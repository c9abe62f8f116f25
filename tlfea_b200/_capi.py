"""ctypes binding of the C ABI declared in include/tlfea_b200.h.

The shared library is built in-tree (``tlfea_b200/libtlfea_b200.so``) by
``tlfea_b200.build``; loading fails loudly when it is missing -- there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libtlfea_b200.so"

OK = 0
INVALID_ARG = 1
NOT_SETUP = 2
SIZE_MISMATCH = 3
CUDA_ERROR = 4
NO_CONVERGENCE = 5
BUDGET_EXCEEDED = 6
NONFINITE = 7
UNSUPPORTED = 8
ALREADY_SETUP = 9
NO_CUDA_DEVICE = 10

STATUS_NAMES = {
    OK: "OK", INVALID_ARG: "INVALID_ARG", NOT_SETUP: "NOT_SETUP", SIZE_MISMATCH: "SIZE_MISMATCH",
    CUDA_ERROR: "CUDA_ERROR", NO_CONVERGENCE: "NO_CONVERGENCE", BUDGET_EXCEEDED: "BUDGET_EXCEEDED",
    NONFINITE: "NONFINITE", UNSUPPORTED: "UNSUPPORTED", ALREADY_SETUP: "ALREADY_SETUP",
    NO_CUDA_DEVICE: "NO_CUDA_DEVICE",
}

TYPE_T10 = 2
TYPE_T4 = 3
PRECISION_FP64 = 0
PRECISION_FP32 = 1


class TLFEAError(RuntimeError):
    """A C-ABI call returned a non-OK status."""

    def __init__(self, status: int, func: str, message: str):
        self.status = status
        super().__init__(f"{func}: {STATUS_NAMES.get(status, status)}: {message}")


class NesterovParams(C.Structure):
    """tlfea_nesterov_params == SyncedNesterovParams (SyncedNesterov.cuh:31-35)."""
    _fields_ = [("alpha", C.c_double), ("rho", C.c_double), ("inner_tol", C.c_double), ("outer_tol", C.c_double),
                ("max_outer", C.c_int), ("max_inner", C.c_int), ("time_step", C.c_double)]


class AdamWParams(C.Structure):
    """tlfea_adamw_params == SyncedAdamWParams (SyncedAdamW.cuh:32-39)."""
    _fields_ = [("lr", C.c_double), ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_double),
                ("weight_decay", C.c_double), ("lr_decay", C.c_double), ("inner_tol", C.c_double),
                ("outer_tol", C.c_double), ("rho", C.c_double), ("max_outer", C.c_int), ("max_inner", C.c_int),
                ("time_step", C.c_double), ("convergence_check_interval", C.c_int), ("inner_rtol", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("outer_iters", C.c_int), ("inner_iters_total", C.c_int), ("last_inner_iters", C.c_int),
                ("status", C.c_int), ("last_norm_g", C.c_double), ("kernel_ms", C.c_double),
                ("rel_residual", C.c_double), ("stop_rule_met", C.c_int)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_LL = C.c_longlong

# name -> argtypes (all return int status unless listed in _RESTYPES)
_SIGS = {
    "tlfea_last_error": [],
    "tlfea_launch_count": [],
    "tlfea_version": [],
    "tlfea_element_create": [C.c_int, C.c_int, C.c_int, C.POINTER(_P)],
    "tlfea_element_destroy": [_P],
    "tlfea_element_set_stream": [_P, _P],
    "tlfea_element_get_stream": [_P, C.POINTER(_P)],
    "tlfea_element_get_counts": [_P, _I, _I, _I],
    "tlfea_element_set_blocking": [_P, C.c_int],
    "tlfea_element_reset_positions": [_P],
    "tlfea_element_setup": [_P, _D, _D, _D, _D, C.c_int, _D, _D, _D, _I],
    "tlfea_element_set_density": [_P, C.c_double],
    "tlfea_element_set_damping": [_P, C.c_double, C.c_double],
    "tlfea_element_set_svk_default": [_P],
    "tlfea_element_set_svk": [_P, C.c_double, C.c_double],
    "tlfea_element_set_mooney_rivlin": [_P, C.c_double, C.c_double, C.c_double],
    "tlfea_element_set_external_force": [_P, _D, C.c_int],
    "tlfea_element_add_gravity": [_P, C.c_double, C.c_double, C.c_double],
    "tlfea_element_set_nodal_fixed": [_P, _I, C.c_int],
    "tlfea_element_update_nodal_fixed": [_P, _I, C.c_int],
    "tlfea_element_update_positions": [_P, _D, _D, _D, C.c_int],
    "tlfea_element_update_constraint_targets": [_P, _D, _D, _D, C.c_int],
    "tlfea_element_calc_dndu_pre": [_P],
    "tlfea_element_calc_mass_matrix": [_P],
    "tlfea_element_calc_p": [_P],
    "tlfea_element_calc_internal_force": [_P],
    "tlfea_element_calc_constraint_data": [_P],
    "tlfea_element_build_constraint_jact_csr": [_P],
    "tlfea_element_build_constraint_jac_csr": [_P],
    "tlfea_element_compute_internal_force": [_P, _P],
    "tlfea_element_set_force_precision": [_P, C.c_int],
    "tlfea_element_set_launch_config": [_P, C.c_int, C.c_int],
    "tlfea_element_compute_internal_force_noalloc": [_P, _P, _P],
    "tlfea_element_get_mass_nnz": [_P, C.POINTER(_LL)],
    "tlfea_element_retrieve_mass_csr": [_P, _I, _I, _D],
    "tlfea_element_retrieve_internal_force": [_P, _D, C.c_int],
    "tlfea_element_retrieve_external_force": [_P, _D, C.c_int],
    "tlfea_element_retrieve_positions": [_P, _D, _D, _D, C.c_int],
    "tlfea_element_retrieve_p": [_P, _D, _LL],
    "tlfea_element_retrieve_dndu_pre": [_P, _D, _LL],
    "tlfea_element_retrieve_detj": [_P, _D, _LL],
    "tlfea_element_retrieve_connectivity": [_P, _I, _LL],
    "tlfea_element_retrieve_constraint": [_P, _D, C.c_int],
    "tlfea_element_retrieve_constraint_jac_csr": [_P, C.c_int, _I, _I, _D],
    "tlfea_element_write_vtk": [_P, C.c_char_p],
    "tlfea_element_device_ptrs": [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)],
    "tlfea_nesterov_create": [_P, C.c_int, C.POINTER(_P)],
    "tlfea_adamw_create": [_P, C.c_int, C.POINTER(_P)],
    "tlfea_adamw_nocoop_create": [_P, C.c_int, C.POINTER(_P)],
    "tlfea_linear_static_create": [_P, C.c_double, C.c_int, C.POINTER(_P)],
    "tlfea_solver_destroy": [_P],
    "tlfea_solver_setup": [_P],
    "tlfea_solver_set_parameters": [_P, _P],
    "tlfea_solver_solve": [_P],
    "tlfea_linear_static_last": [_P, _I, _D],
    "tlfea_linear_static_set_operator": [_P, C.c_int],
    "tlfea_linear_static_set_preconditioner": [_P, C.c_int],
    "tlfea_linear_static_retrieve_k": [_P, C.POINTER(_LL), _I, _I, _D],
    "tlfea_linear_static_apply": [_P, _P, _P],
    "tlfea_solver_get_velocity": [_P, _D, _D, C.c_int],
    "tlfea_solver_set_velocity": [_P, _D, _D, C.c_int],
    "tlfea_solver_get_multipliers": [_P, _D, C.c_int],
    "tlfea_solver_get_stats": [_P, C.POINTER(SolveStats)],
    "tlfea_solver_set_stop_rule": [_P, C.c_double],
    "tlfea_solver_set_mode": [_P, C.c_int],
    "tlfea_solver_run_steps": [_P, C.c_int, C.c_double, _D, C.c_double, C.c_double, C.c_double, _I],
    "tlfea_batch_create": [C.c_int, C.c_int, _I, _I, _D, _D, _D, _D, C.c_int, _D, _D, _D, _I, C.POINTER(_P)],
    "tlfea_batch_create_shared": [C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, _D, _D, C.c_int, _D, _D, _D, _I,
                                  C.POINTER(_P)],
    "tlfea_batch_destroy": [_P],
    "tlfea_dynbatch_create": [_P, C.c_int, C.POINTER(_P)],
    "tlfea_dynbatch_destroy": [_P],
    "tlfea_dynbatch_set_material": [_P, _D, _D],
    "tlfea_dynbatch_set_parameters": [_P, _P, C.c_double],
    "tlfea_dynbatch_set_step_sizes": [_P, _D],
    "tlfea_dynbatch_set_load": [_P, _D, C.c_int, C.c_double, C.c_double, C.c_double],
    "tlfea_dynbatch_set_chunk": [_P, C.c_int],
    "tlfea_dynbatch_set_restart": [_P, C.c_int],
    "tlfea_dynbatch_reset": [_P],
    "tlfea_dynbatch_step": [_P, C.c_int, _P, _I, _D, _I],
    "tlfea_dynbatch_device_ptrs": [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)],
    "tlfea_dynbatch_retrieve_positions": [_P, C.c_int, _D, _D, _D],
    "tlfea_dynbatch_retrieve_velocity": [_P, C.c_int, _D],
    "tlfea_batch_get_counts": [_P, _I, _I, _I, _I],
    "tlfea_batch_get_stream": [_P, C.POINTER(_P)],
    "tlfea_batch_set_material": [_P, _D, _D],
    "tlfea_batch_set_fixed": [_P, _I, C.c_int],
    "tlfea_batch_set_external_force": [_P, _P, _LL, C.c_int],
    "tlfea_batch_set_initial_guess": [_P, _P, _LL, C.c_int],
    "tlfea_batch_set_precision": [_P, C.c_int],
    "tlfea_batch_set_launch": [_P, C.c_int, C.c_int],
    "tlfea_batch_set_mode": [_P, C.c_int],
    "tlfea_batch_get_launch": [_P, _I, _I, _I],
    "tlfea_batch_autotune": [_P, C.c_int, _I, _I, C.POINTER(C.c_float)],
    "tlfea_batch_solve": [_P, C.c_double, C.c_int],
    "tlfea_batch_get_results": [_P, _I, _D, _I],
    "tlfea_batch_retrieve_displacement": [_P, _D, _LL],
    "tlfea_batch_device_ptrs": [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)],
    "tlfea_batch_apply": [_P, _P, _P],
    "tlfea_mlp_create": [C.c_int, _I, C.c_int, C.c_ulonglong, C.POINTER(_P)],
    "tlfea_mlp_destroy": [_P],
    "tlfea_mlp_get_stream": [_P, C.POINTER(_P)],
    "tlfea_mlp_param_count": [_P, C.POINTER(_LL)],
    "tlfea_mlp_set_params": [_P, _F, _LL],
    "tlfea_mlp_get_params": [_P, _F, _LL],
    "tlfea_mlp_get_grads": [_P, _F, _LL],
    "tlfea_mlp_forward": [_P, _P, C.c_int, _P],
    "tlfea_mlp_loss_grad": [_P, _P, _P, C.c_int, _F],
    "tlfea_mlp_adamw_step": [_P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float],
    "tlfea_mlp_train_step": [_P, _P, _P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _F],
    "tlfea_mlp_sync": [_P],
    "tlfea_mlp_gemm_bf16": [C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, C.c_int, _P, _P, C.c_int, _P],
    "tlfea_mlp_gemm_bf16_async": [C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, C.c_int, _P, _P, C.c_int, _P, _P],
}
_RESTYPES = {"tlfea_last_error": C.c_char_p, "tlfea_launch_count": C.c_longlong, "tlfea_version": C.c_char_p}

_lib = None


def lib():
    """Load the sm_100a library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run python -m tlfea_b200.build (or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_GLOBAL if hasattr(os, "RTLD_GLOBAL") else 0)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def call(name: str, *args):
    """Call a C-ABI function; raise TLFEAError on a non-OK status."""
    st = getattr(lib(), name)(*args)
    if st != OK:
        msg = lib().tlfea_last_error().decode(errors="replace")
        raise TLFEAError(st, name, msg)
    return st


def last_error() -> str:
    return lib().tlfea_last_error().decode(errors="replace")


def launch_count() -> int:
    return int(lib().tlfea_launch_count())


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)
