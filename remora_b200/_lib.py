"""ctypes binding of libremora_cuda.so, the C-ABI declared in include/remora_cuda.h.

This is the Python view of the same entry points a C++ host (the ``remora/cuda.hpp``
headers) binds. Loading fails loudly when the library has not been built: there is no
fallback path.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_uint32, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libremora_cuda.so"

RC_SUCCESS = 0
RC_PREC_TF32 = 0
RC_PREC_BF16 = 1
RC_PREC_EMU64 = 2


class MixedOptions(ctypes.Structure):
    _fields_ = [("tol", c_double), ("max_iter", c_int), ("outer", c_int), ("shift_factor", c_double)]


class RefineInfo(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("residuals", c_int), ("converged", c_int), ("backward_error", c_double),
                ("factor_ms", c_double), ("refine_ms", c_double), ("shift", c_double)]
STATUS_NAMES = {0: "RC_SUCCESS", 1: "RC_ERR_INVALID_ARGUMENT", 2: "RC_ERR_CUDA", 3: "RC_ERR_ALLOC",
                4: "RC_ERR_NOT_SUPPORTED", 5: "RC_ERR_TIMEOUT", 6: "RC_ERR_NOT_CONVERGED", 7: "RC_ERR_SIZE_LIMIT"}

_U4 = POINTER(c_uint32)
_I = c_int
_Z = c_size_t
_P = c_void_p

# name -> argument types (restype is int for every entry point unless listed in _RESTYPES)
SIGNATURES: dict[str, list] = {
    "rc_version": [],
    "rc_error_string": [_I],
    "rc_release_workspaces": [],
    "rc_launch_count": [],
    "rc_allocation_count": [],
    "rc_device_count": [_P],
    "rc_set_device": [_I],
    "rc_get_device": [_P],
    "rc_malloc": [_P, _Z],
    "rc_free": [_P],
    "rc_memcpy2d": [_P, _Z, _P, _Z, _Z, _Z, _I, _P],
    "rc_host_alloc": [_P, _Z],
    "rc_host_free": [_P],
    "rc_event_create": [_P],
    "rc_event_record": [_P, _P],
    "rc_event_synchronize": [_P],
    "rc_event_destroy": [_P],
    "rc_stream_create": [_P],
    "rc_stream_destroy": [_P],
    "rc_stream_synchronize": [_P],
    "rc_rng_bits_u32": [_U4, _Z, _Z, _P, _Z, _I, _P],
    "rc_rng_uniform_f32": [_U4, _Z, _Z, _P, _Z, _I, c_float, c_float, _P],
    "rc_rng_normal_f32": [_U4, _Z, _Z, _P, _Z, _I, c_float, c_float, _P],
    "rc_rng_discrete_f32": [_U4, _Z, _Z, _P, _Z, _I, _I, _I, _P],
    "rc_rng_discrete_i32": [_U4, _Z, _Z, _P, _Z, _I, _I, _I, _P],
    "rc_gemm_f64": [_I, _I, _Z, _Z, _Z, c_double, _P, _Z, _P, _Z, c_double, _P, _Z, _P],
    "rc_gemm_f32": [_I, _I, _Z, _Z, _Z, c_float, _P, _Z, _P, _Z, c_float, _P, _Z, _P],
    "rc_gemm_f64_sliced": [_Z, _Z, _Z, c_double, _P, _Z, _P, _Z, c_double, _P, _Z, _P],
    "rc_gemm_tf32": [_I, _I, _Z, _Z, _Z, c_float, _P, _Z, _P, _Z, c_float, _P, _Z, _P],
    "rc_gemm_bf16": [_I, _I, _Z, _Z, _Z, c_float, _P, _Z, _P, _Z, c_float, _P, _Z, _P],
    "rc_set_wait_limit_ns": [ctypes.c_uint64],
    "rc_device_status": [_P],
    "rc_device_error_site": [_P, _P],
    "rc_selftest_wait_timeout": [ctypes.c_uint64, _P],
    "rc_syrk_f64": [_I, _I, _Z, _Z, c_double, _P, _Z, c_double, _P, _Z, _P],
    "rc_syrk_f32": [_I, _I, _Z, _Z, c_float, _P, _Z, c_float, _P, _Z, _P],
    "rc_trsm_f64": [_I, _I, _I, _I, _Z, _Z, c_double, _P, _Z, _P, _Z, _P, _P],
    "rc_trsm_f32": [_I, _I, _I, _I, _Z, _Z, c_float, _P, _Z, _P, _Z, _P, _P],
    "rc_gemv_f64": [_I, _Z, _Z, c_double, _P, _Z, _P, _Z, c_double, _P, _Z, _P],
    "rc_gemv_f32": [_I, _Z, _Z, c_float, _P, _Z, _P, _Z, c_float, _P, _Z, _P],
    "rc_trsv_f64": [_I, _I, _I, _Z, _P, _Z, _P, _Z, _P],
    "rc_trsv_f32": [_I, _I, _I, _Z, _P, _Z, _P, _Z, _P],
    "rc_trmm_f64": [_I, _I, _I, _I, _Z, _Z, _P, _Z, _P, _Z, _P],
    "rc_trmm_f32": [_I, _I, _I, _I, _Z, _Z, _P, _Z, _P, _Z, _P],
    "rc_trmv_f64": [_I, _I, _I, _Z, _P, _Z, _P, _Z, _P],
    "rc_trmv_f32": [_I, _I, _I, _Z, _P, _Z, _P, _Z, _P],
    "rc_axpby_f64": [_Z, c_double, _P, _Z, c_double, _P, _Z, _P],
    "rc_axpby_f32": [_Z, c_float, _P, _Z, c_float, _P, _Z, _P],
    "rc_potrf_f64": [_I, _Z, _P, _Z, _P, _P],
    "rc_getrf_f64": [_I, _Z, _P, _Z, _P, _P, _P],
    "rc_getrf_f32": [_I, _Z, _P, _Z, _P, _P, _P],
    "rc_pstrf_f64": [_I, _Z, _P, _Z, _P, _P, _P],
    "rc_pstrf_f32": [_I, _Z, _P, _Z, _P, _P, _P],
    "rc_potrf_f32": [_I, _Z, _P, _Z, _P, _P],
    "rc_spd_solve_f64": [_Z, _Z, _P, _Z, _P, _Z, _P, _P],
    "rc_spd_solve_f64_noalloc": [_Z, _Z, _P, _Z, _P, _Z, _P, _P],
    "rc_potrf_trsm_batched_f64": [_Z, _P, _P, _P, _P, _I, _P],
    "rc_potrf_trsm_batched_f32": [_Z, _P, _P, _P, _P, _I, _P],
    "rc_batched_release_plans": [],
    "rc_spd_solve_mixed": [_I, _Z, _Z, _P, _Z, _P, _Z, _P, _Z, _P, _P, _P, _P],
    "rc_spd_solve_mixed_workspace": [_I, _Z, _Z, _P, _P],
    "rc_syrk_tc": [_I, _Z, _Z, c_float, _P, _Z, c_float, _P, _Z, _P],
    "rc_syrk_tc_ex": [_I, _Z, _Z, c_float, _P, _Z, c_float, _P, _Z, _I, _P],
    "rc_syrk_emu64": [_Z, _Z, c_double, _P, _Z, c_double, _P, _Z, _P],
    "rc_potrf_backward_f64": [_Z, _P, _Z, _P, _Z, _P, _Z, _P],
    "rc_trsm_backward_f64": [_I, _Z, _Z, _P, _Z, _P, _Z, _P, _Z, _P, _Z, _P],
    "rc_rbf_kernel_f64": [_Z, _I, _P, _P, c_double, _P, _Z, _P],
    "rc_rbf_lengthscale_grad_f64": [_Z, _I, _P, _P, _P, _Z, _P, _P],
    "rc_copy2d_f64": [_I, _Z, _Z, c_double, _P, _Z, _P, _Z, _P],
    "rc_copy2d_f32": [_I, _Z, _Z, c_float, _P, _Z, _P, _Z, _P],
    "rc_fill_f64": [_Z, _Z, c_double, _P, _Z, _P],
    "rc_gather_rows_f64": [_Z, _Z, _P, _P, ctypes.c_ssize_t, ctypes.c_ssize_t, _P, ctypes.c_ssize_t,
                           ctypes.c_ssize_t, _P],
    "rc_gather_rows_f32": [_Z, _Z, _P, _P, ctypes.c_ssize_t, ctypes.c_ssize_t, _P, ctypes.c_ssize_t,
                           ctypes.c_ssize_t, _P],
    "rc_fill_f32": [_Z, _Z, c_float, _P, _Z, _P],
}
_RESTYPES = {"rc_error_string": ctypes.c_char_p, "rc_launch_count": ctypes.c_ulonglong,
             "rc_allocation_count": ctypes.c_ulonglong}

_lib = None


class RemoraCudaError(RuntimeError):
    def __init__(self, name: str, status: int):
        self.status = status
        super().__init__(f"{name} returned {STATUS_NAMES.get(status, status)}: {error_string(status)}")


def lib() -> ctypes.CDLL:
    """Load libremora_cuda.so once (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m remora_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, c_int)
        _lib = handle
    return _lib


def error_string(status: int) -> str:
    return lib().rc_error_string(status).decode()


def call(name: str, *args) -> None:
    """Call an entry point and raise RemoraCudaError on a non-zero status."""
    status = getattr(lib(), name)(*args)
    if status != RC_SUCCESS:
        raise RemoraCudaError(name, status)


def key_array(key) -> ctypes.Array:
    return (c_uint32 * 4)(*[int(k) & 0xFFFFFFFF for k in key])
