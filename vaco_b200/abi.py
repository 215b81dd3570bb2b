"""ctypes mirror of include/vaco_av1_gpu.h: structs, status codes, messages.

The struct layouts here must match the C header field for field; the
`test_abi_layout` CPU test checks sizes and offsets against the compiled
library's own `sizeof`/`offsetof` report.
"""
from __future__ import annotations

import ctypes as C

# vaco_av1_status (mirrors vaco_core::Error, crates/core/vaco-core/src/error.rs:14-54)
OK = 0
INVALID_DATA = 1
UNSUPPORTED = 2
LIMIT_EXCEEDED = 3
DEVICE_ERROR = 4
TIMEOUT = 5

# vaco_av1_msg -> vaco's own &'static str where vaco has one
MESSAGES = {
    0: "",
    1: "CDEF bit depth must be 8, 10, or 12",
    2: "CDEF sample exceeds bit depth",
    3: "invalid CDEF block parameters",
    4: "CDEF strength index exceeds table",
    5: "AV1 superres bit depth must be 8, 10, or 12",
    6: "invalid AV1 superres plane geometry",
    7: "AV1 superres sample exceeds bit depth",
    8: "AV1 restoration plane geometry or bit depth",
    9: "AV1 restoration unit count",
    10: "AV1 restoration coefficient out of range",
    11: "AV1 restoration sample exceeds bit depth",
    12: "AV1 active restoration has no unit size",
    13: "invalid AV1 deblocking parameters",
    14: "AV1 deblocking sample exceeds bit depth",
    15: "AV1 frame geometry does not match its pictures",
    16: "required argument is NULL",
    17: "CUDA runtime error",
    18: "request exceeds the fixed scratch size",
    19: "job admission refused: queue or memory budget full",
    20: "bounded device wait timed out",
    21: "vaco-codec-av1: unsupported pixel format",
    22: "invalid AV1 film grain parameters",
    23: "AV1 film grain sample exceeds bit depth",
    24: "AV1 superres missing U plane",
    25: "AV1 superres missing V plane",
}
MSG = {
    "NONE": 0, "CDEF_BIT_DEPTH": 1, "CDEF_SAMPLE": 2, "CDEF_BLOCK_PARAMS": 3,
    "CDEF_STRENGTH_INDEX": 4, "SR_BIT_DEPTH": 5, "SR_GEOMETRY": 6, "SR_SAMPLE": 7,
    "LR_GEOMETRY": 8, "LR_UNIT_COUNT": 9, "LR_COEFFICIENT": 10, "LR_SAMPLE": 11,
    "LR_NO_UNIT_SIZE": 12, "DB_PARAMS": 13, "DB_SAMPLE": 14, "FRAME_GEOMETRY": 15,
    "NULL_ARGUMENT": 16, "CUDA": 17, "SCRATCH_LIMIT": 18, "QUEUE_FULL": 19, "TIMEOUT": 20,
    "PIXEL_FORMAT": 21, "FG_PARAMS": 22, "FG_SAMPLE": 23, "SR_MISSING_U": 24, "SR_MISSING_V": 25,
}

LR_NONE, LR_WIENER, LR_SGRPROJ = 0, 1, 2
FRAME_LR_NONE, FRAME_LR_SWITCHABLE, FRAME_LR_WIENER, FRAME_LR_SGRPROJ = 0, 1, 2, 3

u16p = C.POINTER(C.c_uint16)


class Picture(C.Structure):
    _fields_ = [
        ("planes", C.c_void_p * 3),
        ("width", C.c_int32 * 3),
        ("height", C.c_int32 * 3),
        ("stride", C.c_int32 * 3),
    ]


class FrameInfo(C.Structure):
    _fields_ = [
        ("bit_depth", C.c_int32),
        ("subsampling_x", C.c_int32),
        ("subsampling_y", C.c_int32),
        ("monochrome", C.c_int32),
        ("mi_rows", C.c_int32),
        ("mi_cols", C.c_int32),
        ("coded_width", C.c_int32),
        ("coded_height", C.c_int32),
        ("upscaled_width", C.c_int32),
    ]


class CdefParams(C.Structure):
    _fields_ = [
        ("enabled", C.c_uint8),
        ("damping", C.c_uint8),
        ("y_primary", C.c_uint8 * 8),
        ("y_secondary", C.c_uint8 * 8),
        ("uv_primary", C.c_uint8 * 8),
        ("uv_secondary", C.c_uint8 * 8),
    ]


class CdefFilterParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint8),
        ("height", C.c_uint8),
        ("edges", C.c_uint8),
        ("bit_depth", C.c_uint8),
        ("direction", C.c_uint8),
        ("damping", C.c_uint8),
        ("primary", C.c_uint16),
        ("secondary", C.c_uint16),
    ]


class LrUnit(C.Structure):
    _fields_ = [
        ("type", C.c_int16),
        ("set", C.c_int16),
        ("vertical", C.c_int16 * 3),
        ("horizontal", C.c_int16 * 3),
        ("xqd", C.c_int16 * 2),
    ]


class LrPlaneConfig(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("bit_depth", C.c_int32),
        ("unit_size", C.c_int32),
        ("subsampling_y", C.c_int32),
    ]


class SuperresPictureConfig(C.Structure):
    """vaco_av1_superres_picture_config: superres::PictureConfig (src/superres.rs:107-122)."""

    _fields_ = [
        ("coded_width", C.c_int32),
        ("upscaled_width", C.c_int32),
        ("coded_height", C.c_int32),
        ("subsampling_x", C.c_int32),
        ("subsampling_y", C.c_int32),
        ("monochrome", C.c_int32),
        ("bit_depth", C.c_int32),
    ]


class DeblockParams(C.Structure):
    _fields_ = [
        ("levels", C.c_uint8 * 4),
        ("sharpness", C.c_uint8),
        ("reserved", C.c_uint8 * 3),
    ]


class FrameJob(C.Structure):
    _fields_ = [
        ("info", FrameInfo),
        ("src", Picture),
        ("dst", Picture),
        ("tx_luma", C.c_void_p),
        ("tx_chroma", C.c_void_p),
        ("lvl_map", C.c_void_p),
        ("skip", C.c_void_p),
        ("cdef_idx", C.c_void_p),
        ("cdef_stride", C.c_int32),
        ("cdef_count", C.c_int32),
        ("deblock", DeblockParams),
        ("cdef", CdefParams),
        ("lr_type", C.c_int32 * 3),
        ("lr_unit_size", C.c_int32 * 3),
        ("lr_units", C.c_void_p * 3),
        ("lr_unit_count", C.c_int32 * 3),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("dbcdef_ctas_per_sm", C.c_int32),
        ("lr_ctas_per_sm", C.c_int32),
        ("use_graphs", C.c_int32),
        ("largest_first", C.c_int32),
        ("dbcdef_threads", C.c_int32),
        ("stage_fusion", C.c_int32),
    ]


class FrameBuffer(C.Structure):
    _fields_ = [
        ("planes", C.c_void_p * 3),
        ("linesize", C.c_int64 * 3),
    ]


class FilmGrainParams(C.Structure):
    """vaco_av1_film_grain_params: film_grain_params() of AV1 5.9.30."""
    _fields_ = [
        ("apply_grain", C.c_uint8),
        ("num_y_points", C.c_uint8),
        ("grain_seed", C.c_uint16),
        ("point_y_value", C.c_uint8 * 14),
        ("point_y_scaling", C.c_uint8 * 14),
        ("chroma_scaling_from_luma", C.c_uint8),
        ("num_cb_points", C.c_uint8),
        ("point_cb_value", C.c_uint8 * 10),
        ("point_cb_scaling", C.c_uint8 * 10),
        ("num_cr_points", C.c_uint8),
        ("point_cr_value", C.c_uint8 * 10),
        ("point_cr_scaling", C.c_uint8 * 10),
        ("grain_scaling_minus_8", C.c_uint8),
        ("ar_coeff_lag", C.c_uint8),
        ("ar_coeffs_y_plus_128", C.c_uint8 * 24),
        ("ar_coeffs_cb_plus_128", C.c_uint8 * 25),
        ("ar_coeffs_cr_plus_128", C.c_uint8 * 25),
        ("ar_coeff_shift_minus_6", C.c_uint8),
        ("grain_scale_shift", C.c_uint8),
        ("cb_mult", C.c_uint8),
        ("cb_luma_mult", C.c_uint8),
        ("cb_offset", C.c_uint16),
        ("cr_mult", C.c_uint8),
        ("cr_luma_mult", C.c_uint8),
        ("cr_offset", C.c_uint16),
        ("overlap_flag", C.c_uint8),
        ("clip_to_restricted_range", C.c_uint8),
        ("mc_identity", C.c_uint8),
    ]


# numpy structured dtype with the vaco_av1_lr_unit layout (20 bytes)
def lr_unit_dtype():
    import numpy as np

    return np.dtype([
        ("type", "<i2"), ("set", "<i2"), ("vertical", "<i2", (3,)),
        ("horizontal", "<i2", (3,)), ("xqd", "<i2", (2,)),
    ])


def cdef_filter_params_dtype():
    import numpy as np

    return np.dtype([
        ("width", "u1"), ("height", "u1"), ("edges", "u1"), ("bit_depth", "u1"),
        ("direction", "u1"), ("damping", "u1"), ("primary", "<u2"), ("secondary", "<u2"),
    ])


STRUCT_SIZES = {
    "vaco_av1_picture": C.sizeof(Picture),
    "vaco_av1_frame_info": C.sizeof(FrameInfo),
    "vaco_av1_cdef_params": C.sizeof(CdefParams),
    "vaco_av1_cdef_filter_params": C.sizeof(CdefFilterParams),
    "vaco_av1_lr_unit": C.sizeof(LrUnit),
    "vaco_av1_lr_plane_config": C.sizeof(LrPlaneConfig),
    "vaco_av1_deblock_params": C.sizeof(DeblockParams),
    "vaco_av1_frame_job": C.sizeof(FrameJob),
    "vaco_av1_tuning": C.sizeof(Tuning),
    "vaco_av1_frame_buffer": C.sizeof(FrameBuffer),
    "vaco_av1_film_grain_params": C.sizeof(FilmGrainParams),
    "vaco_av1_superres_picture_config": C.sizeof(SuperresPictureConfig),
}
