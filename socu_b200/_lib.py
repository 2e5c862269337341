"""ctypes binding of the native library ``socu_b200/lib/libsocu_b200.so``.

The library is the only compute path: there is no CPU or PyTorch fallback.
If it is missing, every solver entry point raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import threading

LIB_DIR = pathlib.Path(__file__).resolve().parent / "lib"
LIB_PATH = LIB_DIR / "libsocu_b200.so"

SOCU_OK = 0
STATUS_TEXT = {
    0: "ok",
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "unsupported problem size",
    -4: "device wait timed out",
    -5: "problem needs more scratch than the fixed no-allocation array holds",
}

FLOAT32 = 0
FLOAT64 = 1

OP_FACTOR = 0
OP_FACTOR_AND_SOLVE = 1
OP_FORWARD = 2
OP_BACKWARD = 3
OP_SOLVE = 4
OP_FACTOR_INV = 5
OP_FORWARD_INV = 6
OP_BACKWARD_INV = 7
OP_SOLVE_INV = 8

KIND_NAMES = ("node", "update", "pull", "forward", "backward", "refine_setup", "refine_update", "residual",
              "refine_check", "ragged")
KIND_COUNT = len(KIND_NAMES)


class Tuning(ctypes.Structure):
    """socu_tuning: launch settings, 0 = not set (include/socu_b200.h)."""
    _fields_ = [("node_threads", ctypes.c_int32), ("update_threads", ctypes.c_int32),
                ("sweep_threads", ctypes.c_int32), ("sweep_tensor_cores", ctypes.c_int32),
                ("update_tile", ctypes.c_int32), ("ragged_units", ctypes.c_int32),
                ("update_tensor_cores", ctypes.c_int32), ("node_tensor_cores", ctypes.c_int32)]

    FIELDS = ("node_threads", "update_threads", "sweep_threads", "sweep_tensor_cores", "update_tile",
              "ragged_units", "update_tensor_cores", "node_tensor_cores")

    @classmethod
    def from_dict(cls, d):
        return cls(**{k: int(d.get(k, 0) or 0) for k in cls.FIELDS})

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in self.FIELDS}


_lock = threading.Lock()
_lib = None

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_u8p = ctypes.c_void_p

_SIGNATURES = {
    "socu_version": (ctypes.c_char_p, []),
    "socu_status_string": (ctypes.c_char_p, [_int]),
    "socu_last_cuda_error": (_int, []),
    "socu_last_cuda_error_line": (_int, []),
    "socu_recursive_iterations": (_i64, [_i64]),
    "socu_off_diag_storage_len": (_i64, [_i64]),
    "socu_max_block_size": (_i64, [_int, _i64]),
    "socu_cholesky_factor": (_int, [_int, _vp, _vp, _u8p, _i64, _i64, _i64, _vp]),
    "socu_cholesky_factor_and_solve": (_int, [_int, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _vp]),
    "socu_cholesky_forward_substitution": (_int, [_int, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _vp]),
    "socu_cholesky_backward_substitution": (_int, [_int, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _vp]),
    "socu_cholesky_solve": (_int, [_int, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _vp]),
    "socu_cholesky_run": (_int, [_int, _int, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _vp]),
    "socu_launch_create": (_int, [ctypes.POINTER(_vp), _int, _int, _vp, _vp, _vp, _u8p,
                                  _i64, _i64, _i64, _i64, _int, _vp]),
    "socu_launch_run": (_int, [_vp, _vp]),
    "socu_launch_create_tuned": (_int, [ctypes.POINTER(_vp), _int, _int, _vp, _vp, _vp, _u8p,
                                        _i64, _i64, _i64, _i64, _int, _vp, _vp]),
    "socu_launch_create_ex": (_int, [ctypes.POINTER(_vp), _int, _int, _vp, _vp, _vp, _u8p, _vp,
                                     _i64, _i64, _i64, _i64, _int, _vp, _vp]),
    "socu_cholesky_run_info": (_int, [_int, _int, _vp, _vp, _vp, _u8p, _vp, _i64, _i64, _i64, _i64, _vp]),
    "socu_tuning_set": (_int, [_int, _i64, _i64, _vp]),
    "socu_tuning_get": (_int, [_int, _i64, _i64, _vp]),
    "socu_tuning_clear": (_int, []),
    "socu_launch_profile": (_int, [_vp, _vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i64)]),
    "socu_profile_error": (_int, [ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "socu_launch_kernel_count": (_i64, [_vp]),
    "socu_launch_round_kernel_count": (_i64, [_vp]),
    "socu_launch_destroy": (_int, [_vp]),
    "socu_refine_workspace_bytes": (ctypes.c_size_t, [_i64, _i64, _i64, _i64]),
    "socu_refine_solve": (_int, [_vp, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _int, ctypes.c_double,
                                 _vp, ctypes.c_size_t, _vp, _vp, _vp]),
    "socu_refine_launch_create": (_int, [ctypes.POINTER(_vp), _vp, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64,
                                         _int, ctypes.c_double, _vp, ctypes.c_size_t, _vp, _vp, _int, _vp]),
    "socu_refine_fallback_workspace_bytes": (ctypes.c_size_t, [_i64, _i64, _i64, _i64]),
    "socu_refine_fallback_launch_create": (_int, [ctypes.POINTER(_vp), _vp, _vp, _vp, _vp, _u8p, _i64, _i64, _i64,
                                                  _i64, _int, ctypes.c_double, _vp, ctypes.c_size_t, _vp, _vp, _vp,
                                                  _vp]),
    "socu_block_tridiag_residual": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "socu_copy_lower_blocks_async": (_int, [_vp, _vp, _i64, _i64, _i64, _vp]),
    "socu_lower_blocks_bytes": (_i64, [_i64, _i64, _i64]),
    "socu_block_tridiag_grad": (_int, [_int, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp]),
    "socu_refine_solve_noalloc": (_int, [_vp, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _int, ctypes.c_double,
                                         _vp, _vp, _vp]),
    "socu_ragged_layout": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp]),
    "socu_ragged_create": (_int, [ctypes.POINTER(_vp), _int, _int, _vp, _vp, _vp, _i64, _int]),
    "socu_ragged_factor_and_solve": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "socu_ragged_refine_solve": (_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _vp, _vp]),
    "socu_ragged_launch_create": (_int, [ctypes.POINTER(_vp), _vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _vp,
                                         _int, _vp]),
    "socu_ragged_error": (_int, [_vp, ctypes.POINTER(_int)]),
    "socu_ragged_grid": (_i64, [_vp]),
    "socu_ragged_set_wait_limit": (_int, [_vp, _i64]),
    "socu_ragged_withhold_instance": (_int, [_vp, _i64]),
    "socu_tc_selftest": (_int, [_vp, _vp, _vp, _i64, _i64, _i64, _vp, _vp]),
    "socu_tc_error": (_int, [ctypes.POINTER(_int), _int]),
    "socu_dmma_peak_launch": (_int, [_i64, _int, _int, _vp, _vp, ctypes.POINTER(ctypes.c_double)]),
    "socu_ragged_destroy": (_int, [_vp]),
}


def exported_symbols():
    """Names the C ABI declares (include/socu_b200.h)."""
    return list(_SIGNATURES)


def load():
    """Load (once) and return the native library; raise RuntimeError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = os.environ.get("SOCU_B200_LIB", str(LIB_PATH))
        if not os.path.exists(path):
            raise RuntimeError(
                f"socu_b200 native library not found at {path}; build it with "
                "`python -m socu_b200.build` (nvcc, sm_100a)")
        lib = ctypes.CDLL(path)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int, what: str):
    if status != SOCU_OK:
        lib = load()
        detail = STATUS_TEXT.get(status, "unknown status")
        cuda = lib.socu_last_cuda_error()
        extra = f" (cudaError {cuda} at capi.cu:{lib.socu_last_cuda_error_line()})" if status == -2 else ""
        raise RuntimeError(f"{what} failed: {detail}{extra}")
