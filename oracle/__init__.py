"""CPU oracle for the AV1 post-filter path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/libvaco_oracle.so, the C++ restatement of vaco's
scalar filters (oracle/vaco_oracle.cpp).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module, and only as the checker or
the timed CPU baseline; the CUDA library never calls it.

Every function returns (result, msg) where msg is the vaco_av1_msg id (0 = ok)
the restated vaco function would have failed with.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

from vaco_b200 import abi
from vaco_b200.frame import FrameInputs, alloc_outputs, host_job, picture_struct, ptr

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libvaco_oracle.so"
_lib = None


def build(force: bool = False) -> pathlib.Path:
    """Compile the oracle with its Makefile (g++ -O2)."""
    deps = [HERE / "vaco_oracle.cpp", HERE.parent / "include" / "vaco_av1_gpu.h"]
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        l = C.CDLL(str(LIB_PATH))
        vp, i32 = C.c_void_p, C.c_int
        l.vo_find_direction.argtypes = [vp, i32, i32, vp, vp]
        l.vo_filter_block.argtypes = [vp, vp, i32, vp]
        l.vo_adjust_strength.argtypes = [i32, C.c_uint32]
        l.vo_chroma_direction.argtypes = [i32, i32, i32]
        l.vo_cdef_picture.argtypes = [vp, vp, vp, vp, vp, i32, i32, vp, i32]
        l.vo_upscale_plane.argtypes = [vp, i32, i32, i32, i32, i32, i32, i32, vp, i32, i32]
        l.vo_restore_plane.argtypes = [vp, i32, i32, i32, vp, i32, i32, i32, vp, vp, i32, vp, i32, i32]
        l.vo_deblock_picture.argtypes = [vp, vp, vp, vp, vp, vp, vp, i32]
        l.vo_postfilter_frame.argtypes = [vp, i32]
        l.vo_emit_frame.argtypes = [vp, vp, vp]
        l.vo_film_grain.argtypes = [vp, vp, vp, vp, vp]
        l.vo_upscale_picture.argtypes = [vp, vp, vp, i32]
        l.vo_deblock_lines.argtypes = [vp, i32, i32, i32, vp, i32, i32, vp]
        _lib = l
    return _lib


def _u16(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint16)


def default_threads() -> int:
    return int(os.environ.get("VACO_ORACLE_THREADS", "1"))


# ---------------------------------------------------------------- CDEF
def find_direction(blocks: np.ndarray, bit_depth: int):
    """cdef::find_direction (src/cdef.rs:79) over blocks of shape (n, 64)."""
    blocks = _u16(blocks).reshape(-1, 64)
    n = blocks.shape[0]
    dirs = np.zeros(n, np.uint8)
    var = np.zeros(n, np.uint32)
    m = lib().vo_find_direction(ptr(blocks), n, bit_depth, ptr(dirs), ptr(var))
    return (dirs, var), m


def filter_block(inputs: np.ndarray, params: np.ndarray):
    """cdef::filter_block (src/cdef.rs:142) over (n, 144) inputs and a
    structured params array (abi.cdef_filter_params_dtype())."""
    inputs = _u16(inputs).reshape(-1, 144)
    params = np.ascontiguousarray(params, dtype=abi.cdef_filter_params_dtype())
    out = np.zeros((inputs.shape[0], 64), np.uint16)
    m = lib().vo_filter_block(ptr(inputs), ptr(params), inputs.shape[0], ptr(out))
    return out, m


def adjust_strength(primary: int, variance: int) -> int:
    return lib().vo_adjust_strength(primary, variance)


def chroma_direction(direction: int, sub_x: bool, sub_y: bool) -> int:
    return lib().vo_chroma_direction(direction, int(sub_x), int(sub_y))


def cdef_picture(f: FrameInputs, planes=None, threads: int | None = None):
    """apply_cdef (src/decode.rs:739) on f.planes (or `planes`)."""
    planes = [_u16(p) for p in (planes if planes is not None else f.planes)]
    outs = [np.zeros_like(p) for p in planes]
    shapes = [p.shape for p in planes]
    src = picture_struct([ptr(p) for p in planes], shapes)
    dst = picture_struct([ptr(o) for o in outs], shapes)
    info = f.info()
    skip = np.ascontiguousarray(f.skip, np.uint8)
    idx = np.ascontiguousarray(f.cdef_idx, np.int32)
    params = f.cdef.to_c()
    m = lib().vo_cdef_picture(C.byref(src), C.byref(dst), C.byref(info), ptr(skip), ptr(idx),
                              idx.shape[1], idx.size, C.byref(params),
                              threads or default_threads())
    return outs, m


# ---------------------------------------------------------------- superres
def upscale_plane(plane: np.ndarray, visible_width: int, output_width: int, height: int,
                  bit_depth: int, threads: int | None = None):
    """superres::upscale_plane (src/superres.rs:163)."""
    plane = _u16(plane)
    out = np.zeros((max(height, 0), max(output_width, 0)), np.uint16)
    m = lib().vo_upscale_plane(ptr(plane), plane.shape[1], plane.shape[0], plane.shape[1],
                               visible_width, output_width, height, bit_depth,
                               ptr(out) if out.size else None, max(output_width, 1),
                               threads or default_threads())
    return out, m


def upscale_picture(planes, config: abi.SuperresPictureConfig, threads: int | None = None):
    """superres::upscale_picture (src/superres.rs:226-274) over `planes`
    (Mi-padded; None for an absent chroma plane); returns (output planes, msg)."""
    np_ = 1 if config.monochrome else 3
    ins = [None if p is None else _u16(p) for p in planes]
    outs = []
    for k in range(np_):
        sx = config.subsampling_x if k else 0
        sy = config.subsampling_y if k else 0
        w = -(-config.upscaled_width // (1 << sx))
        h = -(-config.coded_height // (1 << sy))
        outs.append(np.zeros((max(h, 0), max(w, 0)), np.uint16))
    pin = abi.Picture()
    pout = abi.Picture()
    for k in range(np_):
        if ins[k] is not None:
            pin.planes[k] = ins[k].ctypes.data
            pin.height[k], pin.width[k] = ins[k].shape
            pin.stride[k] = ins[k].shape[1]
        pout.planes[k] = outs[k].ctypes.data if outs[k].size else None
        pout.height[k], pout.width[k] = outs[k].shape
        pout.stride[k] = max(outs[k].shape[1], 1)
    m = lib().vo_upscale_picture(C.byref(pin), C.byref(pout), C.byref(config), threads or default_threads())
    return outs, m


# ---------------------------------------------------------------- restoration
def restore_plane(before: np.ndarray, after: np.ndarray, width: int, height: int,
                  bit_depth: int, unit_size: int, subsampling_y: bool, units: np.ndarray,
                  threads: int | None = None):
    """restoration::restore_plane (src/restoration.rs:178)."""
    before, after = _u16(before), _u16(after)
    units = np.ascontiguousarray(units, dtype=abi.lr_unit_dtype())
    cfg = abi.LrPlaneConfig(width, height, bit_depth, unit_size, int(subsampling_y))
    out = np.zeros((max(height, 0), max(width, 0)), np.uint16)
    m = lib().vo_restore_plane(ptr(before), before.shape[1], before.shape[0], before.shape[1],
                               ptr(after), after.shape[1], after.shape[0], after.shape[1],
                               C.byref(cfg), ptr(units) if len(units) else None, len(units),
                               ptr(out) if out.size else None, max(width, 1),
                               threads or default_threads())
    return out, m


# ---------------------------------------------------------------- deblocking
def deblock_picture(f: FrameInputs, threads: int | None = None):
    """AV1 7.14 loop filter (spec restatement; no vaco counterpart)."""
    planes = [_u16(p) for p in f.planes[: f.num_planes]]
    outs = [np.zeros_like(p) for p in planes]
    shapes = [p.shape for p in planes]
    src = picture_struct([ptr(p) for p in planes], shapes)
    dst = picture_struct([ptr(o) for o in outs], shapes)
    info = f.info()
    params = f.deblock_c()
    lvl = None if f.lvl_map is None else np.ascontiguousarray(f.lvl_map, np.uint8)
    m = lib().vo_deblock_picture(C.byref(src), C.byref(dst), C.byref(info),
                                 ptr(np.ascontiguousarray(f.tx_luma, np.uint8)),
                                 ptr(np.ascontiguousarray(f.tx_chroma, np.uint8)),
                                 ptr(lvl), C.byref(params), threads or default_threads())
    return outs, m


def deblock_lines(lines, plane: int, filter_size: int, levels, sharpness: int, bit_depth: int) -> np.ndarray:
    """Lines of 16 samples across an edge (sample k past the edge at index
    8 + k), shape (n, 16), each at its own level, through the oracle's 7.14.6
    sample filter; returns the filtered lines."""
    lines = _u16(lines).reshape(-1, 16)
    lv = np.ascontiguousarray(levels, np.uint8).reshape(-1)
    assert lv.size == lines.shape[0]
    out = np.zeros_like(lines)
    lib().vo_deblock_lines(ptr(lines), lines.shape[0], plane, filter_size, ptr(lv), sharpness, bit_depth, ptr(out))
    return out


# ---------------------------------------------------------------- whole chain
def postfilter_frame(f: FrameInputs, threads: int | None = None):
    """deblock -> CDEF -> superres -> restoration (decode.rs:553-559 order)."""
    outs = alloc_outputs(f)
    job = host_job(f, outs)
    m = lib().vo_postfilter_frame(C.byref(job), threads or default_threads())
    return outs, m


# ---------------------------------------------------------------- frame emission
def emit_frame(planes, info: abi.FrameInfo, frame):
    """pic_to_frame / blit (decode.rs:3795-3891) into `frame`, a list of
    uint8 arrays (rows x linesize) as frame_layout() makes them; returns
    (frame, msg)."""
    planes = [_u16(p) for p in planes]  # alive through the call
    pic = picture_struct([ptr(p) for p in planes], [p.shape for p in planes])
    out = abi.FrameBuffer()
    for k, b in enumerate(frame):
        out.planes[k] = b.ctypes.data
        out.linesize[k] = b.shape[1]
    m = lib().vo_emit_frame(C.byref(pic), C.byref(info), C.byref(out))
    return frame, m


def film_grain(planes, info: abi.FrameInfo, params: abi.FilmGrainParams, gauss):
    """Film grain synthesis (AV1 7.18.3) of u16 `planes` with the Gaussian
    table `gauss` (2048 int16); returns (output planes, msg)."""
    planes = [_u16(p) for p in planes]
    outs = [np.zeros_like(p) for p in planes]
    g = np.ascontiguousarray(gauss, np.int16)
    pin = picture_struct([ptr(p) for p in planes], [p.shape for p in planes])
    pout = picture_struct([ptr(o) for o in outs], [o.shape for o in outs])
    m = lib().vo_film_grain(C.byref(pin), C.byref(pout), C.byref(info), C.byref(params), g.ctypes.data)
    return outs, m
