"""ctypes binding of libdsht_b200.so (the C ABI declared in include/dsht.h).

The library is built in-tree by ``python -m directsht_b200.build``.  There is no CPU
fallback: if the library is missing, or no CUDA device is present, calls fail loudly.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdsht_b200.so")

DSHT_OK = 0
DSHT_ERR_INVALID = 1
DSHT_ERR_CUDA = 2
DSHT_ERR_NOMEM = 3
DSHT_ERR_THETA_RANGE = 4
DSHT_ERR_EMPTY = 5
DSHT_ERR_POLAR_RANGE = 6

DSHT_MODE_CALL = 0
DSHT_MODE_BASIC = 1

DSHT_W_F64 = 0
DSHT_W_F32 = 1

DSHT_PLAN_DEFAULT = 0
DSHT_PLAN_F32_TABLES = 1

DSHT_TUNE_PIECE_MAX = 1
DSHT_TUNE_MAPS_PER_PASS = 2
DSHT_TUNE_BIN_SUMS = 3

DSHT_BIN_SUMS_AUTO = 0
DSHT_BIN_SUMS_NUFFT = 1
DSHT_BIN_SUMS_TC = 2
DSHT_BIN_SUMS_FP64 = 3

DSHT_PREC_FP64 = 0
DSHT_PREC_MIXED = 1
DSHT_PREC_MIXED_F64_TABLES = 2

STAGES = ("points", "bin_sums", "fold", "contract", "rotate")

# Every symbol include/dsht.h declares, with (restype, argtypes).
_dp = ct.POINTER(ct.c_double)
_vp = ct.c_void_p
SIGNATURES = {
    "dsht_plan_create": (ct.c_int, [ct.c_int, ct.c_int, ct.c_double, ct.c_int, ct.POINTER(ct.c_void_p)]),
    "dsht_plan_destroy": (ct.c_int, [_vp]),
    "dsht_plan_info": (ct.c_int, [_vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_double),
                                  ct.POINTER(ct.c_int64)]),
    "dsht_index": (ct.c_int64, [ct.c_int, ct.c_int, ct.c_int]),
    "dsht_workspace_size": (ct.c_int, [_vp, ct.c_int64, ct.POINTER(ct.c_size_t)]),
    "dsht_execute": (ct.c_int, [_vp, _vp, _vp, _vp, ct.c_int64, ct.c_int, _vp, _vp, ct.c_size_t, _vp]),
    "dsht_plan_tune": (ct.c_int, [_vp, ct.c_int, ct.c_int]),
    "dsht_plan_get_tune": (ct.c_int, [_vp, ct.c_int, ct.POINTER(ct.c_int)]),
    "dsht_workspace_size_maps": (ct.c_int, [_vp, ct.c_int64, ct.c_int, ct.POINTER(ct.c_size_t)]),
    "dsht_execute_maps": (ct.c_int, [_vp, _vp, _vp, _vp, ct.c_int, ct.c_int64, ct.c_int, ct.c_int64, ct.c_int, _vp,
                                     _vp, ct.c_size_t, _vp]),
    "dsht_enqueue_maps": (ct.c_int, [_vp, _vp, _vp, _vp, ct.c_int, ct.c_int64, ct.c_int, ct.c_int64, ct.c_int, _vp,
                                     _vp, _vp, ct.c_size_t, _vp]),
    "dsht_status": (ct.c_int, [ct.c_uint, ct.c_int]),
    "dsht_workspace_size_batch": (ct.c_int, [_vp, ct.c_int64, ct.c_int, ct.POINTER(ct.c_size_t)]),
    "dsht_execute_batch": (ct.c_int, [_vp, ct.c_int, _vp, _vp, _vp, _vp, ct.c_int, _vp, _vp, ct.c_size_t, _vp]),
    "dsht_enqueue_batch": (ct.c_int, [_vp, ct.c_int, _vp, _vp, _vp, _vp, ct.c_int, _vp, _vp, _vp, ct.c_size_t,
                                      _vp]),
    "dsht_execute_noalloc": (ct.c_int, [_vp, _vp, _vp, _vp, ct.c_int64, ct.c_int, _vp, _vp]),
    "dsht_noalloc_scratch_bytes": (ct.c_size_t, []),
    "dsht_execute_host": (ct.c_int, [_vp, _dp, _dp, _dp, ct.c_int64, ct.c_int, _dp]),
    "dsht_rotate_back": (ct.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "dsht_get_row": (ct.c_int, [_vp, ct.c_int, ct.c_int, ct.c_int, _dp]),
    "dsht_get_table": (ct.c_int, [_vp, ct.c_int, _dp]),
    "dsht_get_table_mlayout": (ct.c_int, [_vp, ct.c_int, _vp, ct.c_int, _vp]),
    "dsht_alm2cl": (ct.c_int, [ct.c_int, _dp, _dp]),
    "dsht_alm2cl_device": (ct.c_int, [ct.c_int, ct.c_int, _vp, ct.c_int64, _vp, _vp]),
    "dsht_mode_coupling": (ct.c_int, [ct.c_int, _vp, ct.c_int, _vp, _vp]),
    "dsht_make_table": (ct.c_int, [ct.c_int, ct.c_int, ct.c_double, _dp, _dp]),
    "dsht_do_transform": (ct.c_int, [ct.c_int, ct.c_int, ct.c_double, _dp, _dp, ct.c_int, _dp, _dp, _dp, _dp,
                                     _dp]),
    "dsht_set_precision": (ct.c_int, [_vp, ct.c_int]),
    "dsht_get_precision": (ct.c_int, [_vp, ct.POINTER(ct.c_int)]),
    "dsht_profile_enable": (ct.c_int, [_vp, ct.c_int]),
    "dsht_profile_read": (ct.c_int, [_vp, _dp, ct.POINTER(ct.c_int64), ct.c_int]),
    "dsht_launch_count": (ct.c_int64, []),
    "dsht_test_stall_next_contraction": (ct.c_int, []),
    "dsht_test_point_keys": (ct.c_int, [_vp, _vp, _vp, ct.c_int64, ct.c_int, _vp, _vp, _vp]),
    "dsht_test_nufft_tables": (ct.c_int, [ct.c_int, ct.POINTER(ct.c_int), _dp, _dp]),
    "dsht_mixed_min_points": (ct.c_int64, []),
    "dsht_last_error": (ct.c_char_p, []),
    "dsht_version": (ct.c_char_p, []),
}

_lock = threading.Lock()
_lib = None


class DSHTError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dsht error {code}: {msg}")
        self.code = code
        self.msg = msg


def load() -> ct.CDLL:
    """Load the library once (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m directsht_b200.build`")
        lib = ct.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    return load().dsht_last_error().decode()


def check(code: int) -> None:
    if code != DSHT_OK:
        raise DSHTError(code, last_error())


def ptr(a) -> ct.c_void_p:
    """Raw address of a numpy array or torch tensor as c_void_p."""
    if hasattr(a, "data_ptr"):
        return ct.c_void_p(a.data_ptr())
    return ct.c_void_p(a.ctypes.data)


def dptr(a):
    return a.ctypes.data_as(_dp)
