"""ctypes binding of the C ABI in include/lqg.h (``liteqg_b200/_lib/liblqg.so``).

Loading fails loudly when the library has not been built: there is no
fallback implementation of the search anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "liblqg.so")

LQG_OK = 0
LQG_NO_ID = 0xFFFFFFFF
STATUS_NAMES = {
    0: "LQG_OK", 1: "LQG_ERR_ARG", 2: "LQG_ERR_IO", 3: "LQG_ERR_CUDA",
    4: "LQG_ERR_NOMEM", 5: "LQG_ERR_STATE", 6: "LQG_ERR_CAPACITY", 7: "LQG_ERR_CORRUPT",
}

# Every symbol include/lqg.h declares, with its ctypes signature.
_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)
_vp = C.c_void_p
SIGNATURES = {
    "lqg_last_error": (C.c_char_p, []),
    "lqg_create": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_int,
                             C.POINTER(_vp)]),
    "lqg_free": (None, [_vp]),
    "lqg_load": (C.c_int, [_vp, C.c_char_p]),
    "lqg_save": (C.c_int, [_vp, C.c_char_p]),
    "lqg_set_arrays": (C.c_int, [_vp, C.c_uint32, _vp, _vp, _vp, _vp]),
    "lqg_get_arrays": (C.c_int, [_vp, _u32p, _vp, _vp, _vp, _vp]),
    "lqg_set_ef": (C.c_int, [_vp, C.c_uint32]),
    "lqg_build": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32]),
    "lqg_build_ex": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                               C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, _vp]),
    "lqg_search": (C.c_int, [_vp, _vp, C.c_uint32, _vp]),
    "lqg_search_batch_device": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp, C.c_uint32,
                                          _vp, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp]),
    "lqg_stream_status": (C.c_int, [_vp, _vp]),
    "lqg_search_batch": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp, C.c_uint32,
                                   _vp, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp]),
    "lqg_search_exact_device": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp, C.c_uint32,
                                          _vp, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp]),
    "lqg_search_exact_noalloc": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp, C.c_uint32,
                                           _vp, C.c_uint32, _vp, _vp, C.c_uint32, _vp, _vp]),
    "lqg_set_kernel_events": (C.c_int, [_vp, _vp, _vp]),
    "lqg_server_start": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "lqg_server_submit": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)]),
    "lqg_server_wait": (C.c_int, [_vp, C.c_uint64, _vp, C.c_int64, C.POINTER(C.c_double)]),
    "lqg_server_replay": (C.c_int, [_vp, _vp, C.c_int64, _vp, _vp, _vp, _vp, C.c_uint32, _vp]),
    "lqg_server_stats": (C.c_int, [_vp, _vp]),
    "lqg_server_reset_stats": (C.c_int, [_vp]),
    "lqg_server_stop": (C.c_int, [_vp]),
    "lqg_set_tuning": (C.c_int, [_vp, _vp]),
    "lqg_get_tuning": (C.c_int, [_vp, _vp]),
    "lqg_info": (C.c_int, [_vp, C.POINTER(C.c_uint64), _u32p, _u32p, _u32p, _u32p]),
    "lqg_device_arrays": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), _u32p]),
    "lqg_fs_build": (C.c_int, [_vp, C.c_uint64]),
    "lqg_fs_set_arrays": (C.c_int, [_vp, _vp, _vp, _vp]),
    "lqg_fs_get_arrays": (C.c_int, [_vp, _u32p, _vp, _vp, _vp]),
    "lqg_fs_search_batch_device": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp,
                                             C.c_uint32, _vp, C.c_uint32, _vp, _vp]),
    "lqg_fs_stream_status": (C.c_int, [_vp, _vp]),
    "lqg_fs_search_batch": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_uint32, _vp, C.c_uint32,
                                      _vp, C.c_uint32, _vp, _vp]),
    "lqg_fs_search": (C.c_int, [_vp, _vp, C.c_uint32, _vp]),
    "lqg_selftest_bounded_wait": (C.c_int, [C.c_int, C.c_uint32, _u32p]),
}


class Tuning(C.Structure):
    _fields_ = [
        ("lanes_per_cand", C.c_uint32),
        ("visited_bits", C.c_uint32),
        ("warps_per_block", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("mode", C.c_uint32),
        ("heap_warps", C.c_uint32),
        ("heap_scap", C.c_uint32),
        ("replay_warps", C.c_uint32),
        ("replay_all", C.c_uint32),
        ("small_batch", C.c_uint32),
    ]


SMALL_BATCH_AUTO = 0xFFFFFFFE
SMALL_BATCH_OFF = 0xFFFFFFFF


class BuildReport(C.Structure):
    _fields_ = [
        ("prune_ms", C.c_double),
        ("build_ms", C.c_double),
        ("rechecks", C.c_uint64),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("streams", C.c_uint32),
        ("max_batch", C.c_uint32),
        ("state_budget", C.c_uint64),
        ("max_k", C.c_uint32),
        ("max_ef", C.c_uint32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_uint64),
        ("batches", C.c_uint64),
        ("mean_batch", C.c_double),
        ("p50_us", C.c_double),
        ("p99_us", C.c_double),
        ("qps", C.c_double),
        ("max_batch", C.c_uint32),
        ("streams", C.c_uint32),
    ]


class LqgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """The loaded C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(
                f"{_LIB_PATH} is missing: build it with `python -m liteqg_b200._build` "
                "(or __graft_entry__.build())")
        L = C.CDLL(_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def library_path() -> str:
    return _LIB_PATH


def check(status: int) -> None:
    if status != LQG_OK:
        raise LqgError(status, lib().lqg_last_error().decode(errors="replace"))
