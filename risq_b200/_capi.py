"""ctypes binding of librisqgpu.so (include/risqgpu.h).

The shared library is the only compute path: importing this module does not
require a GPU, but every call that does device work goes through the library,
and loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librisqgpu.so")

OK = 0
ERR_INVALID = 1
ERR_OOM = 2
ERR_CUDA = 3
ERR_NOT_CONVERGED = 4
ERR_NO_DEVICE = 5
ERR_CAPACITY = 6

FP64, FP32, MIXED, COLS, FP64_UPPER, FP32_UPPER, MIXED_UPPER, MATRIX_FREE = 0, 1, 2, 3, 4, 5, 6, 7
BUILDER_AUTO, BUILDER_FAST, BUILDER_LEGACY = 0, 1, 2
MODE_FP64, MODE_MIXED, MODE_FP32 = 0, 1, 2
PRECOND_DPR, PRECOND_LEARNED = 0, 1

STATUS_NAMES = {
    OK: "ok", ERR_INVALID: "invalid argument", ERR_OOM: "out of device memory", ERR_CUDA: "CUDA error",
    ERR_NOT_CONVERGED: "Davidson did not converge", ERR_NO_DEVICE: "no CUDA device",
    ERR_CAPACITY: "output buffer too small",
}


class HStats(C.Structure):
    _fields_ = [("n_dets", C.c_uint64), ("nnz_upper", C.c_uint64), ("nnz_full", C.c_uint64),
                ("candidates", C.c_uint64), ("ms_setup", C.c_double), ("ms_count", C.c_double),
                ("ms_fill", C.c_double), ("ms_total", C.c_double), ("bytes_csr", C.c_uint64),
                ("gpu_ms_count", C.c_double), ("gpu_ms_fill", C.c_double), ("n_tiles", C.c_uint64),
                ("nnz_dense", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DStats(C.Structure):
    _fields_ = [("iters", C.c_int), ("n_sigma", C.c_int), ("n_sigma_fp64", C.c_int), ("converged", C.c_int),
                ("reason", C.c_int), ("learned_fallbacks", C.c_int), ("ms_total", C.c_double),
                ("ms_sigma", C.c_double), ("residual", C.c_double * 8)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "residual"}
        d["residual"] = list(self.residual)
        return d


class VarIter(C.Structure):
    _fields_ = [("eps", C.c_double), ("n_dets", C.c_uint64), ("n_new", C.c_uint64), ("candidates", C.c_uint64),
                ("nnz_upper", C.c_uint64), ("energy", C.c_double), ("dav_iters", C.c_int),
                ("dav_converged", C.c_int), ("ms_select", C.c_double), ("ms_build", C.c_double),
                ("ms_davidson", C.c_double), ("storage", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# risqgpu_allreduce_fn: int (*)(void* buf_dev, size_t count, void* stream, void* user)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_handle = C.c_void_p

# (name, restype, argtypes) for every entry point declared in include/risqgpu.h
SIGNATURES = [
    ("risqgpu_version", C.c_char_p, []),
    ("risqgpu_device_count", C.c_int, []),
    ("risqgpu_create", C.c_int, [C.c_int, _dp, C.c_size_t, _dp, C.c_size_t, C.c_double, C.c_int, C.POINTER(_handle)]),
    ("risqgpu_destroy", None, [_handle]),
    ("risqgpu_last_error", C.c_char_p, [_handle]),
    ("risqgpu_set_dets", C.c_int, [_handle, _u64p, C.c_size_t, C.c_size_t, _dp]),
    ("risqgpu_build_h", C.c_int, [_handle, C.c_int, C.c_int, C.POINTER(HStats)]),
    ("risqgpu_nnz", C.c_int, [_handle, _u64p, _u64p]),
    ("risqgpu_export_upper", C.c_int, [_handle, _i64p, _i64p, _dp, C.c_size_t, _dp]),
    ("risqgpu_export_rows", C.c_int, [_handle, _i64p, C.c_size_t, _i64p, _i64p, _dp, C.c_size_t,
                                      C.POINTER(C.c_size_t)]),
    ("risqgpu_sigma", C.c_int, [_handle, _dp, _dp, C.c_int]),
    ("risqgpu_sigma_device", C.c_int, [_handle, C.c_void_p, C.c_void_p, C.c_int]),
    ("risqgpu_davidson", C.c_int, [_handle, C.c_int, _dp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                   _dp, _dp, C.POINTER(DStats)]),
    ("risqgpu_sparse_optimize", C.c_int, [_handle, _dp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                          _dp, _dp, C.POINTER(HStats), C.POINTER(DStats)]),
    ("risqgpu_set_subspace", C.c_int, [_handle, C.c_int, C.c_int]),
    ("risqgpu_set_reproducible", C.c_int, [_handle, C.c_int]),
    ("risqgpu_set_partition", C.c_int, [_handle, C.c_int, C.c_int, ALLREDUCE_FN, C.c_void_p]),
    ("risqgpu_set_memory_limit", C.c_int, [_handle, C.c_size_t]),
    ("risqgpu_memory_used", C.c_int, [_handle, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("risqgpu_set_stream", C.c_int, [_handle, C.c_void_p]),
    ("risqgpu_sigma_noalloc", C.c_int, [_handle, C.c_void_p, C.c_void_p]),
    ("risqgpu_ham_diag", C.c_int, [_handle, _u64p, C.c_size_t, _dp]),
    ("risqgpu_ham_off_diag", C.c_int, [_handle, _u64p, _u64p, C.c_size_t, _dp]),
    ("risqgpu_set_precond_mlp", C.c_int, [_handle, C.c_int, C.c_int, _fp, _fp, _fp, _fp, _fp, _fp, _fp]),
    ("risqgpu_precond_factors", C.c_int, [_handle, C.c_double, _fp]),
    ("risqgpu_self_energy", C.c_int, [_handle, C.c_double, C.c_double, _dp]),
    ("risqgpu_mlp_grad", C.c_int, [C.c_int, C.c_int, C.c_int, _fp, _fp, _fp, _fp, C.c_int64, _fp, _fp]),
    ("risqgpu_mlp_train", C.c_int, [C.c_int, C.c_int, C.c_int, _fp, _fp, _fp, _fp, C.c_int64, C.c_int, C.c_int,
                                    C.c_float, C.c_uint64, _fp]),
    ("risqgpu_find_new_dets", C.c_int, [_handle, _dp, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    ("risqgpu_get_new_dets", C.c_int, [_handle, _u64p, _dp, C.c_size_t]),
    ("risqgpu_variational", C.c_int, [_handle, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, _dp, _u64p]),
    ("risqgpu_get_wf", C.c_int, [_handle, _u64p, _dp, _dp, C.c_size_t]),
    ("risqgpu_var_log", C.c_int, [_handle, C.POINTER(VarIter), C.c_int, C.POINTER(C.c_int)]),
]

_lib = None


class RisqGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load librisqgpu.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C {_HERE}` or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, handle=None):
    if code != OK:
        msg = lib().risqgpu_last_error(handle).decode() if handle else ""
        raise RisqGpuError(code, msg)


def ptr(a, t):
    return a.ctypes.data_as(t)
