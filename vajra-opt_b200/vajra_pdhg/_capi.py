"""ctypes declarations of libvajra_pdhg.so (include/vajra_pdhg.h).

The library is built in-tree (vajra-opt_b200/csrc/Makefile -> vajra_pdhg/lib/).  Loading
fails loudly when it is missing: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libvajra_pdhg.so")

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)

ABI_VERSION = 8   # VAJRA_ABI_VERSION of include/vajra_pdhg.h these declarations follow

# vajra_status
OK, ERR_INVALID_ARGUMENT, ERR_NO_DEVICE, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_WAIT_TIMEOUT, ERR_INTERNAL = range(7)
ALGO_REFERENCE, ALGO_HALPERN = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2   # PREC_FP32: vajra_pdhg_unrolled only


class VajraLp(C.Structure):
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("nnz", C.c_int64),
                ("col_ptr", _i64p), ("row_idx", _i32p), ("values", _dp), ("c", _dp),
                ("col_lower", _dp), ("col_upper", _dp), ("row_lower", _dp), ("row_upper", _dp),
                ("sense", C.c_int32), ("objective_offset", C.c_double)]


class VajraOpts(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("precision", C.c_int32), ("tolerance", C.c_double),
                ("gap_tolerance", C.c_double), ("time_limit", C.c_double),
                ("iteration_limit", C.c_int64), ("check_frequency", C.c_int32),
                ("enable_scaling", C.c_int32), ("pock_chambolle", C.c_int32),
                ("ruiz_iterations", C.c_int32), ("reflection", C.c_double),
                ("mixed_switch_tolerance", C.c_double), ("device", C.c_int32),
                ("autotune", C.c_int32), ("verbose", C.c_int32), ("mixed_stall_checks", C.c_int32),
                ("restart_sufficient", C.c_double), ("restart_necessary", C.c_double),
                ("restart_artificial", C.c_double), ("primal_weight_smoothing", C.c_double),
                ("step_safety", C.c_double), ("restart_metric", C.c_int32),
                ("spmv_shape_a", C.c_int32), ("spmv_shape_at", C.c_int32),
                ("mixed_reflection", C.c_double), ("degree_order", C.c_int32), ("pow2_scaling", C.c_int32),
                ("fp64_value_storage", C.c_int32), ("handover_mode", C.c_int32), ("max_violation", C.c_double),
                ("max_abs_violation", C.c_double)]


class VajraResult(C.Structure):
    _fields_ = [("col_value", _dp), ("row_value", _dp), ("row_dual", _dp), ("col_dual", _dp),
                ("status", C.c_int32), ("iterations", C.c_int64), ("objective_value", C.c_double),
                ("dual_objective", C.c_double), ("restart_count", C.c_int32),
                ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("duality_gap", C.c_double), ("spectral_norm_estimate", C.c_double),
                ("tau", C.c_double), ("sigma", C.c_double), ("converged", C.c_int32),
                ("rel_primal", C.c_double), ("rel_dual", C.c_double), ("rel_gap", C.c_double),
                ("rel_kkt", C.c_double), ("primal_weight", C.c_double),
                ("fp32_iterations", C.c_int64), ("fp64_iterations", C.c_int64),
                ("upload_time_sec", C.c_double), ("setup_time_sec", C.c_double),
                ("iteration_time_sec", C.c_double), ("download_time_sec", C.c_double),
                ("total_time_sec", C.c_double), ("host_device_transfers", C.c_int64),
                ("spmv_group_a", C.c_int32), ("spmv_group_at", C.c_int32),
                ("primal_kernel_us", C.c_double), ("dual_kernel_us", C.c_double),
                ("primal_kernel_bytes", C.c_double), ("dual_kernel_bytes", C.c_double),
                ("kernel_samples", C.c_int64), ("kernel_launches", C.c_int64),
                ("device_time_sec", C.c_double), ("status_message", C.c_char * 256)]


class VajraDeviceInfo(C.Structure):
    _fields_ = [("available", C.c_int32), ("device_name", C.c_char * 256),
                ("total_vram_bytes", C.c_uint64), ("free_vram_bytes", C.c_uint64),
                ("compute_capability_major", C.c_int32), ("compute_capability_minor", C.c_int32),
                ("multi_processor_count", C.c_int32)]


class VajraTiming(C.Structure):
    _fields_ = [("upload_time_sec", C.c_double), ("iteration_time_sec", C.c_double),
                ("download_time_sec", C.c_double), ("total_time_sec", C.c_double),
                ("host_device_transfers", C.c_int64), ("iterations", C.c_int64),
                ("device_name", C.c_char * 256), ("kernel_mode", C.c_char * 64)]


class VajraDeviceDiagnostics(C.Structure):
    _fields_ = [("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("objective", C.c_double), ("duality_gap", C.c_double),
                ("converged", C.c_int32), ("numerical_error", C.c_int32)]


# (name, restype, argtypes) of every exported symbol declared in include/vajra_pdhg.h
SIGNATURES = [
    ("vajra_default_opts", None, [C.POINTER(VajraOpts)]),
    ("vajra_pdhg_solve", C.c_int32, [C.POINTER(VajraLp), C.POINTER(VajraOpts), C.POINTER(VajraResult)]),
    ("vajra_pdhg_create", C.c_int32, [C.POINTER(VajraLp), C.POINTER(VajraOpts), C.POINTER(C.c_void_p)]),
    ("vajra_pdhg_solve_batch", C.c_int32, [C.c_int32, C.POINTER(VajraLp), C.POINTER(VajraOpts), C.POINTER(VajraResult)]),
    ("vajra_pdhg_run", C.c_int32, [C.c_void_p, C.POINTER(VajraResult)]),
    ("vajra_pdhg_destroy", C.c_int32, [C.c_void_p]),
    ("vajra_probe_device", C.c_int32, [C.c_int32, C.POINTER(VajraDeviceInfo)]),
    ("vajra_is_cuda_available", C.c_int32, []),
    ("vajra_last_timing", None, [C.POINTER(VajraTiming)]),
    ("vajra_status_string", C.c_char_p, [C.c_int32]),
    ("vajra_abi_version", C.c_int32, []),
    ("vajra_default_unrolled_opts", None, [C.c_void_p]),
    ("vajra_pdhg_unrolled", C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_csr_spmv_f64", C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_csr_spmv_f32", C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_csc_spmv_transpose_f64", C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_csc_spmv_transpose_f32", C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_dual_prox_f64", C.c_int32, [C.c_int32, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vajra_primal_prox_f64", C.c_int32, [C.c_int32, C.c_double] + [C.c_void_p] * 7),
    ("vajra_device_diagnostics_f64", C.c_int32, [C.c_int32, C.c_int32] + [C.c_void_p] * 11),
    ("vajra_pdhg_step_f64", C.c_int32, [C.c_int32, C.c_int32] + [C.c_void_p] * 11 + [C.c_double, C.c_double] + [C.c_void_p] * 6),
    ("vajra_relative_kkt_noalloc_f64", C.c_int32, [C.c_int32, C.c_int32] + [C.c_void_p] * 13
     + [C.c_int32, C.c_double, C.c_void_p, C.c_void_p]),
    ("vajra_scale_lp", C.c_int32, [C.POINTER(VajraLp), C.POINTER(VajraOpts)] + [C.c_void_p] * 8),
    ("vajra_release_cached_memory", C.c_int64, [C.c_int32]),
    ("vajra_gather_probe_f32", C.c_int32, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
]

_lib = None


def lib():
    """Load libvajra_pdhg.so once; raise if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C vajra-opt_b200/csrc` "
                "(or __graft_entry__.build()); this package has no CPU fallback")
        handle = C.CDLL(LIB_PATH)
        handle.vajra_abi_version.restype = C.c_int32
        handle.vajra_abi_version.argtypes = []
        got = handle.vajra_abi_version()
        if got != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {got}, these bindings expect {ABI_VERSION}: rebuild")
        for name, res, args in SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, what: str = "") -> None:
    if status != OK:
        msg = lib().vajra_status_string(status).decode()
        raise RuntimeError(f"{what}: vajra status {status} ({msg})")
