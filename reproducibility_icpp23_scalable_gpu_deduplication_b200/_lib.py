"""ctypes bindings for libb200dedup.so (the C ABI in include/b200dedup.h).

The library is loaded from this package directory only.  There is no fallback: if the
shared library is missing or a call fails, an exception is raised.
"""
import ctypes
import os

from . import _build

_lib = None

B2D_OK = 0
STATUS = {
    0: "B2D_OK", -1: "B2D_ERR_ARG", -2: "B2D_ERR_CUDA", -3: "B2D_ERR_NOMEM", -4: "B2D_ERR_FORMAT",
    -5: "B2D_ERR_IO", -6: "B2D_ERR_MAP_FULL", -7: "B2D_ERR_TIMEOUT", -8: "B2D_ERR_INTERNAL",
    -9: "B2D_ERR_RESTART_RANGE", -10: "B2D_ERR_LEN_CHANGED", -11: "B2D_ERR_UNSUPPORTED",
}
HASH_MURMUR3 = 0
HASH_MD5 = 1

# every symbol include/b200dedup.h declares: (name, restype, argtypes)
_vp, _u32, _u64, _int, _cc = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_char_p
_u8pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8))
SIGNATURES = [
    ("b2d_create", _int, [_u32, _int, ctypes.POINTER(_vp)]),
    ("b2d_create_list", _int, [_u32, _int, ctypes.POINTER(_vp)]),
    ("b2d_destroy", _int, [_vp]),
    ("b2d_set_stream", _int, [_vp, _vp]),
    ("b2d_set_param", _int, [_vp, _cc, ctypes.c_int64]),
    ("b2d_checkpoint_device", _int, [_vp, _vp, _u64, _int, _int, ctypes.POINTER(_u64)]),
    ("b2d_diff_device", _int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_u64)]),
    ("b2d_copy_diff", _int, [_vp, _vp, _u64]),
    ("b2d_copy_diff_async", _int, [_vp, _vp, _u64, _vp]),
    ("b2d_write_chkpt_log", _int, [_vp, ctypes.c_char_p]),
    ("b2d_write_chkpt_log_host", _int, [_vp, _vp, _vp, _u64, _cc]),
    ("b2d_write_restart_log", _int, [_vp, _u32, _cc]),
    ("b2d_checkpoint", _int, [_vp, _vp, _u64, _int, _u8pp, ctypes.POINTER(_u64)]),
    ("b2d_checkpoint_log", _int, [_vp, _vp, _u64, _cc, _int, _u8pp, ctypes.POINTER(_u64)]),
    ("b2d_checkpoint_file", _int, [_vp, _vp, _u64, _cc, _cc, _int]),
    ("b2d_restart", _int, [_vp, _vp, _u64, ctypes.POINTER(_vp), ctypes.POINTER(_u64), _u32, _u32, _cc]),
    ("b2d_restart_files", _int, [_vp, _vp, _u64, ctypes.POINTER(_cc), _u32, _u32, _cc]),
    ("b2d_restart_device", _int, [_vp, _vp, _u64, ctypes.POINTER(_vp), ctypes.POINTER(_u64), _u32, _u32]),
    ("b2d_restart_noalloc", _int, [_vp, _u64, ctypes.POINTER(_vp), ctypes.POINTER(_u64), _u32, _u32, _vp]),
    ("b2d_num_first_ocur", _int, [_vp, ctypes.POINTER(_u64)]),
    ("b2d_num_shift_dupl", _int, [_vp, ctypes.POINTER(_u64)]),
    ("b2d_current_id", _int, [_vp, ctypes.POINTER(_u32)]),
    ("b2d_baseline_id", _int, [_vp, ctypes.POINTER(_u32)]),
    ("b2d_timers", _int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("b2d_restart_timers", _int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("b2d_datasizes", _int, [_vp, ctypes.POINTER(_u64)]),
    ("b2d_phase_times", _int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_int)]),
    ("b2d_last_launch_count", _int, [_vp, ctypes.POINTER(_u32)]),
    ("b2d_debug_tree", _int, [_vp, _vp, _u64]),
    ("b2d_debug_labels", _int, [_vp, _vp, _u64]),
    ("b2d_hash_chunks", _int, [_int, _vp, _u64, _u32, _vp, _vp]),
    ("b2d_pool_reserve", _int, [_u64]),
    ("b2d_memory", _int, [_vp, ctypes.POINTER(_u64)]),
    ("b2d_map_stats", _int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("b2d_estimate_memory", _int, [_u64, _u32, _int, ctypes.POINTER(_u64)]),
    ("b2d_batch_create", _int, [ctypes.POINTER(_vp)]),
    ("b2d_batch_destroy", _int, [_vp]),
    ("b2d_batch_set_stream", _int, [_vp, _vp]),
    ("b2d_batch_set_param", _int, [_vp, _cc, ctypes.c_int64]),
    ("b2d_batch_get_param", _int, [_vp, _cc, ctypes.POINTER(ctypes.c_int64)]),
    ("b2d_batch_checkpoint", _int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_u64),
                                    ctypes.POINTER(_int), _u32, ctypes.POINTER(_int)]),
    ("b2d_batch_launch", _int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_u64),
                                ctypes.POINTER(_int), _u32, ctypes.POINTER(_int)]),
    ("b2d_batch_query", _int, [_vp, ctypes.POINTER(_int)]),
    ("b2d_batch_wait", _int, [_vp, ctypes.POINTER(_int)]),
    ("b2d_batch_times", _int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("b2d_batch_launch_count", _int, [_vp, ctypes.POINTER(_u32)]),
    ("b2d_hash_host", _int, [_int, _vp, _u64, _vp]),
    ("b2d_strerror", ctypes.c_char_p, [_int]),
]


class B2DError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        msg = lib().b2d_strerror(code).decode() if _lib is not None else ""
        super().__init__(f"{what} failed: {STATUS.get(code, code)} ({msg})")


def lib_path():
    return _build.LIB_PATH


def lib():
    """Load the in-tree library; builds it first when nvcc is available and it is missing."""
    global _lib
    if _lib is None:
        path = _build.LIB_PATH
        if not os.path.exists(path):
            _build.build()
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run `python -m {__package__}._build`")
        L = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, what):
    if code != B2D_OK:
        raise B2DError(code, what)
    return code
