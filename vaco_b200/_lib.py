"""Loads libvaco_av1_gpu.so (the sm_100a CUDA library) and declares its C ABI.

There is no CPU fallback: if the library is missing this raises, and every
entry point returns VACO_AV1_DEVICE_ERROR when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libvaco_av1_gpu.so"

# (name, restype, argtypes) for every symbol of include/vaco_av1_gpu.h
_vp, _i32, _u64 = C.c_void_p, C.c_int32, C.c_uint64
_pi32 = C.POINTER(C.c_int32)
SIGNATURES = [
    ("vaco_av1_message", C.c_char_p, [_i32]),
    ("vaco_av1_ctx_create", _i32, [_i32, C.POINTER(_vp)]),
    ("vaco_av1_ctx_destroy", None, [_vp]),
    ("vaco_av1_ctx_last_cuda_error", _i32, [_vp]),
    ("vaco_av1_ctx_launch_count", _u64, [_vp]),
    ("vaco_av1_postfilter_frame_host_submit", _i32, [_vp, _vp, _vp, _vp]),
    ("vaco_av1_postfilter_frame_host_wait", _i32, [_vp, _u64, _vp]),
    ("vaco_av1_emit_frame_dev", _i32, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("vaco_av1_emit_frame_host", _i32, [_vp, _vp, _vp, _vp, _vp]),
    ("vaco_av1_postfilter_frame_emit_host", _i32, [_vp, _vp, _vp, _vp]),
    ("vaco_av1_ctx_set_deferred_status", _i32, [_vp, _i32]),
    ("vaco_av1_ctx_flush", _i32, [_vp, _vp, _vp]),
    ("vaco_av1_ctx_set_stage_timing", _i32, [_vp, _i32]),
    ("vaco_av1_ctx_stage_ms", _i32, [_vp, _vp, _vp]),
    ("vaco_av1_cdef_find_direction_dev", _i32, [_vp, _vp, _vp, _i32, _i32, _vp, _vp, _pi32]),
    ("vaco_av1_cdef_find_direction_host", _i32, [_vp, _vp, _i32, _i32, _vp, _vp, _pi32]),
    ("vaco_av1_cdef_filter_block_dev", _i32, [_vp, _vp, _vp, _vp, _i32, _vp, _pi32]),
    ("vaco_av1_cdef_filter_block_host", _i32, [_vp, _vp, _vp, _i32, _vp, _pi32]),
    ("vaco_av1_cdef_picture_dev", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _pi32]),
    ("vaco_av1_cdef_picture_host", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _pi32]),
    ("vaco_av1_superres_upscale_plane_dev", _i32,
     [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _vp, _i32, _pi32]),
    ("vaco_av1_superres_upscale_plane_host", _i32, [_vp, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _vp, _pi32]),
    ("vaco_av1_superres_upscale_picture_dev", _i32, [_vp, _vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_superres_upscale_picture_host", _i32, [_vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_restore_plane_dev", _i32,
     [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _i32, _i32, _i32, _vp, _vp, _i32, _vp, _i32, _pi32]),
    ("vaco_av1_restore_plane_host", _i32, [_vp, _vp, _i32, _i32, _vp, _i32, _i32, _vp, _vp, _i32, _vp, _pi32]),
    ("vaco_av1_deblock_picture_dev", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_deblock_picture_host", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_postfilter_frame_dev", _i32, [_vp, _vp, _vp, _pi32]),
    ("vaco_av1_postfilter_frame_host", _i32, [_vp, _vp, _pi32]),
    ("vaco_av1_ctx_set_tuning", _i32, [_vp, _vp]),
    ("vaco_av1_ctx_get_tuning", _i32, [_vp, _vp]),
    ("vaco_av1_postfilter_batch_dev", _i32, [_vp, _vp, _vp, _i32, _vp, _vp]),
    ("vaco_av1_postfilter_frame_noalloc", _i32, [_vp, _vp, _pi32]),
    ("vaco_av1_film_grain_dev", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_film_grain_host", _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _pi32]),
    ("vaco_av1_server_create", _i32, [_vp, _vp]),
    ("vaco_av1_server_destroy", None, [_vp]),
    ("vaco_av1_server_open_stream", _i32, [_vp, _vp, _vp, _i32, _vp, _vp]),
    ("vaco_av1_server_close_stream", _i32, [_vp, _i32]),
    ("vaco_av1_server_slot", _i32, [_vp, _i32, _i32, _vp]),
    ("vaco_av1_server_submit", _i32, [_vp, _i32, _i32, _vp, _vp]),
    ("vaco_av1_server_submit_host", _i32, [_vp, _i32, _i32, _vp, _vp]),
    ("vaco_av1_server_wait", _i32, [_vp, C.c_uint64, _i32, _vp, _vp]),
    ("vaco_av1_server_get_stats", _i32, [_vp, _vp]),
    ("vaco_av1_server_upload", _i32, [_vp, _i32, _i32, _vp]),
    ("vaco_av1_server_download", _i32, [_vp, _i32, _i32, _vp]),
    ("vaco_av1_server_submit_many", _i32, [_vp, _i32, _vp, _vp, _vp, _vp]),
    ("vaco_av1_server_wait_many", _i32, [_vp, _i32, _vp, _i32, _vp, _vp, _vp]),
]

_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m vaco_b200.build` "
                "(the CUDA path has no CPU fallback)")
        l = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def exported_symbols():
    return [s[0] for s in SIGNATURES]
