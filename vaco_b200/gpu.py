"""Thin Python binding of the C ABI: one `Context` per CUDA device/thread.

Host-array calls (`*_host`) take and return numpy arrays; device calls take
torch CUDA tensors (torch is used only for device memory and streams).
Errors raise `VacoError` carrying the C status and vaco's message text.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from ._lib import lib
from .frame import (FrameInputs, alloc_outputs, build_job, frame_buffer, frame_layout, host_job, picture_struct,
                    ptr)


class VacoError(Exception):
    """Mirrors vaco_core::Error: `status` is the vaco_av1_status, `msg` the id."""

    def __init__(self, status: int, msg: int, detail: str = ""):
        self.status, self.msg = status, msg
        text = abi.MESSAGES.get(msg, "")
        kind = {1: "InvalidData", 2: "Unsupported", 3: "LimitExceeded", 4: "DeviceError", 5: "Timeout"}.get(status, "Error")
        super().__init__(f"{kind}({text!r}){(' ' + detail) if detail else ''}")


def _check(ctx: "Context", status: int, msg: C.c_int32):
    if status != abi.OK:
        detail = ""
        if status == abi.DEVICE_ERROR:
            detail = f"cudaError={lib().vaco_av1_ctx_last_cuda_error(ctx.handle)}"
        raise VacoError(status, msg.value, detail)


class Context:
    """vaco_av1_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().vaco_av1_ctx_create(device, C.byref(h))
        if st != abi.OK:
            raise VacoError(st, abi.MSG["CUDA"], f"vaco_av1_ctx_create(device={device})")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().vaco_av1_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(lib().vaco_av1_ctx_launch_count(self.handle))

    # ------------------------------------------------------------ CDEF block API
    def find_direction(self, blocks: np.ndarray, bit_depth: int):
        blocks = np.ascontiguousarray(blocks, np.uint16).reshape(-1, 64)
        n = blocks.shape[0]
        dirs = np.zeros(n, np.uint8)
        var = np.zeros(n, np.uint32)
        m = C.c_int32()
        st = lib().vaco_av1_cdef_find_direction_host(self.handle, ptr(blocks), n, bit_depth, ptr(dirs), ptr(var),
                                                     C.byref(m))
        _check(self, st, m)
        return dirs, var

    def filter_block(self, inputs: np.ndarray, params: np.ndarray) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, np.uint16).reshape(-1, 144)
        params = np.ascontiguousarray(params, abi.cdef_filter_params_dtype())
        out = np.zeros((inputs.shape[0], 64), np.uint16)
        m = C.c_int32()
        st = lib().vaco_av1_cdef_filter_block_host(self.handle, ptr(inputs), ptr(params), inputs.shape[0], ptr(out),
                                                   C.byref(m))
        _check(self, st, m)
        return out

    # ------------------------------------------------------------ frame-level (host arrays)
    def cdef_picture(self, f: FrameInputs, planes: Optional[Sequence[np.ndarray]] = None) -> List[np.ndarray]:
        planes = [np.ascontiguousarray(p, np.uint16) for p in (planes if planes is not None else f.planes)]
        outs = [np.zeros_like(p) for p in planes]
        shapes = [p.shape for p in planes]
        src = picture_struct([ptr(p) for p in planes], shapes)
        dst = picture_struct([ptr(o) for o in outs], shapes)
        info = f.info()
        skip = np.ascontiguousarray(f.skip, np.uint8)
        idx = np.ascontiguousarray(f.cdef_idx, np.int32)
        params = f.cdef.to_c()
        m = C.c_int32()
        st = lib().vaco_av1_cdef_picture_host(self.handle, C.byref(src), C.byref(dst), C.byref(info), ptr(skip),
                                              ptr(idx), idx.shape[1], idx.size, C.byref(params), C.byref(m))
        _check(self, st, m)
        return outs

    def upscale_plane(self, plane: np.ndarray, visible_width: int, output_width: int, height: int,
                      bit_depth: int) -> np.ndarray:
        plane = np.ascontiguousarray(plane, np.uint16)
        out = np.zeros((max(height, 0), max(output_width, 0)), np.uint16)
        m = C.c_int32()
        st = lib().vaco_av1_superres_upscale_plane_host(self.handle, ptr(plane), plane.shape[1], plane.shape[0],
                                                        visible_width, output_width, height, bit_depth,
                                                        ptr(out) if out.size else None, C.byref(m))
        _check(self, st, m)
        return out

    def upscale_picture(self, planes, config: abi.SuperresPictureConfig) -> List[np.ndarray]:
        """superres::upscale_picture through the host entry point: Mi-padded
        planes (None for an absent chroma plane) in, upscaled planes out."""
        n = 1 if config.monochrome else 3
        ins = [None if p is None else np.ascontiguousarray(p, np.uint16) for p in planes]
        outs = []
        for k in range(n):
            sx = config.subsampling_x if k else 0
            sy = config.subsampling_y if k else 0
            w = -(-config.upscaled_width // (1 << sx))
            h = -(-config.coded_height // (1 << sy))
            outs.append(np.zeros((max(h, 0), max(w, 0)), np.uint16))
        pin, pout = abi.Picture(), abi.Picture()
        for k in range(n):
            if ins[k] is not None:
                pin.planes[k] = ins[k].ctypes.data
                pin.height[k], pin.width[k] = ins[k].shape
                pin.stride[k] = ins[k].shape[1]
            pout.planes[k] = outs[k].ctypes.data if outs[k].size else None
            pout.height[k], pout.width[k] = outs[k].shape
            pout.stride[k] = max(outs[k].shape[1], 1)
        m = C.c_int32()
        st = lib().vaco_av1_superres_upscale_picture_host(self.handle, C.byref(pin), C.byref(pout), C.byref(config),
                                                          C.byref(m))
        _check(self, st, m)
        return outs

    def restore_plane(self, before: np.ndarray, after: np.ndarray, width: int, height: int, bit_depth: int,
                      unit_size: int, subsampling_y: bool, units: np.ndarray) -> np.ndarray:
        before = np.ascontiguousarray(before, np.uint16)
        after = np.ascontiguousarray(after, np.uint16)
        units = np.ascontiguousarray(units, abi.lr_unit_dtype())
        cfg = abi.LrPlaneConfig(width, height, bit_depth, unit_size, int(bool(subsampling_y)))
        out = np.zeros((max(height, 0), max(width, 0)), np.uint16)
        m = C.c_int32()
        st = lib().vaco_av1_restore_plane_host(self.handle, ptr(before), before.shape[1], before.shape[0],
                                               ptr(after), after.shape[1], after.shape[0], C.byref(cfg),
                                               ptr(units) if len(units) else None, len(units),
                                               ptr(out) if out.size else None, C.byref(m))
        _check(self, st, m)
        return out

    def deblock_picture(self, f: FrameInputs) -> List[np.ndarray]:
        planes = [np.ascontiguousarray(p, np.uint16) for p in f.planes[: f.num_planes]]
        outs = [np.zeros_like(p) for p in planes]
        shapes = [p.shape for p in planes]
        src = picture_struct([ptr(p) for p in planes], shapes)
        dst = picture_struct([ptr(o) for o in outs], shapes)
        info = f.info()
        params = f.deblock_c()
        lvl = None if f.lvl_map is None else np.ascontiguousarray(f.lvl_map, np.uint8)
        txl = np.ascontiguousarray(f.tx_luma, np.uint8)
        txc = np.ascontiguousarray(f.tx_chroma, np.uint8)
        m = C.c_int32()
        st = lib().vaco_av1_deblock_picture_host(self.handle, C.byref(src), C.byref(dst), C.byref(info), ptr(txl),
                                                 ptr(txc), ptr(lvl), C.byref(params), C.byref(m))
        _check(self, st, m)
        return outs

    def emit_frame(self, planes: Sequence[np.ndarray], info: abi.FrameInfo, fill: int = 0) -> List[np.ndarray]:
        """pic_to_frame through the host entry point: u16 planes -> packed
        frame planes (uint8 rows x linesize, vaco's layout)."""
        frame = frame_layout(info, fill)
        planes = [np.ascontiguousarray(p, np.uint16) for p in planes]  # alive through the call
        pic = picture_struct([ptr(p) for p in planes], [p.shape for p in planes])
        m = C.c_int32()
        st = lib().vaco_av1_emit_frame_host(self.handle, C.byref(pic), C.byref(info), C.byref(frame_buffer(frame)),
                                            C.byref(m))
        _check(self, st, m)
        return frame

    def film_grain(self, planes: Sequence[np.ndarray], info: abi.FrameInfo, params: abi.FilmGrainParams,
                   gauss: np.ndarray) -> List[np.ndarray]:
        """Film grain synthesis through the host entry point: u16 planes in,
        grained u16 planes out; `gauss` is the 2048-entry Gaussian table."""
        planes = [np.ascontiguousarray(p, np.uint16) for p in planes]  # alive through the call
        outs = [np.zeros_like(p) for p in planes]
        g = np.ascontiguousarray(gauss, np.int16)
        pin = picture_struct([ptr(p) for p in planes], [p.shape for p in planes])
        pout = picture_struct([ptr(o) for o in outs], [o.shape for o in outs])
        m = C.c_int32()
        st = lib().vaco_av1_film_grain_host(self.handle, C.byref(pin), C.byref(pout), C.byref(info),
                                            C.byref(params), g.ctypes.data, C.byref(m))
        _check(self, st, m)
        return outs

    def postfilter_frame_emit(self, f: FrameInputs, fill: int = 0) -> List[np.ndarray]:
        """The chain then pic_to_frame, host arrays in, packed frame out."""
        info = f.info()
        frame = frame_layout(info, fill)
        job = host_job(f, [np.zeros((1, 1), np.uint16)] * f.num_planes)
        m = C.c_int32()
        st = lib().vaco_av1_postfilter_frame_emit_host(self.handle, C.byref(job), C.byref(frame_buffer(frame)),
                                                       C.byref(m))
        _check(self, st, m)
        return frame

    def postfilter_frame(self, f: FrameInputs) -> List[np.ndarray]:
        """deblock -> CDEF -> superres -> restoration through the host entry point."""
        outs = alloc_outputs(f)
        job = host_job(f, outs)
        m = C.c_int32()
        st = lib().vaco_av1_postfilter_frame_host(self.handle, C.byref(job), C.byref(m))
        _check(self, st, m)
        return outs

    # ------------------------------------------------------------ device-resident frames
    def postfilter_frame_dev(self, dev: "DeviceFrame", stream=None) -> None:
        m = C.c_int32()
        st = lib().vaco_av1_postfilter_frame_dev(self.handle, stream, C.byref(dev.job), C.byref(m))
        _check(self, st, m)

    def set_deferred_status(self, enable: bool) -> None:
        """postfilter_frame_dev enqueues without a host sync; flush() reports errors."""
        if lib().vaco_av1_ctx_set_deferred_status(self.handle, 1 if enable else 0) != abi.OK:
            raise VacoError(abi.DEVICE_ERROR, abi.MSG["CUDA"], "could not switch deferred status")

    def flush(self, stream=None) -> None:
        """Synchronize `stream` and raise the earliest error of the frames since the last flush."""
        m = C.c_int32()
        st = lib().vaco_av1_ctx_flush(self.handle, stream, C.byref(m))
        _check(self, st, m)

    # ------------------------------------------------------------ batched form
    @property
    def tuning(self) -> abi.Tuning:
        t = abi.Tuning()
        lib().vaco_av1_ctx_get_tuning(self.handle, C.byref(t))
        return t

    def set_tuning(self, dbcdef_ctas_per_sm=None, lr_ctas_per_sm=None, use_graphs=None, largest_first=None,
                   dbcdef_threads=None, stage_fusion=None):
        t = self.tuning
        for name, v in (("dbcdef_ctas_per_sm", dbcdef_ctas_per_sm), ("lr_ctas_per_sm", lr_ctas_per_sm),
                        ("use_graphs", use_graphs), ("largest_first", largest_first),
                        ("dbcdef_threads", dbcdef_threads), ("stage_fusion", stage_fusion)):
            if v is not None:
                setattr(t, name, int(v))
        st = lib().vaco_av1_ctx_set_tuning(self.handle, C.byref(t))
        if st != abi.OK:
            raise VacoError(st, 0, "invalid tuning")

    def batch_jobs(self, frames: Sequence["DeviceFrame"]):
        arr = (abi.FrameJob * len(frames))()
        for i, d in enumerate(frames):
            arr[i] = d.job
        return arr

    def postfilter_batch_dev(self, frames: Sequence["DeviceFrame"], stream=None, jobs=None):
        """The chain over many device-resident frames in one launch set;
        returns per-frame (status, msg) lists."""
        n = len(frames)
        jobs = jobs if jobs is not None else self.batch_jobs(frames)
        st = (C.c_int32 * n)()
        ms = (C.c_int32 * n)()
        rc = lib().vaco_av1_postfilter_batch_dev(self.handle, stream, jobs, n, st, ms)
        if rc == abi.DEVICE_ERROR:
            raise VacoError(rc, abi.MSG["CUDA"], f"cudaError={lib().vaco_av1_ctx_last_cuda_error(self.handle)}")
        return list(st), list(ms)


class DeviceFrame:
    """A FrameInputs uploaded to device memory (torch tensors) with its output
    planes allocated, packed as a device-pointer vaco_av1_frame_job."""

    def __init__(self, f: FrameInputs, device: int = 0):
        import torch

        self.f = f
        dev = torch.device("cuda", device)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.planes = [t(p.view(np.int16)) for p in f.planes[: f.num_planes]]
        self.outputs = [torch.zeros(f.output_shape(k), dtype=torch.int16, device=dev) for k in range(f.num_planes)]
        self.side = {k: (t(v) if v is not None else None) for k, v in f.side_arrays().items()}
        self.units = [t(f.lr_units[k].view(np.uint8)) if (k < len(f.lr_units) and f.lr_units[k] is not None) else None
                      for k in range(3)]
        side_ptrs = {k: (v.data_ptr() if v is not None else None) for k, v in self.side.items()}
        unit_ptrs = [u.data_ptr() if u is not None else None for u in self.units]
        self.job = build_job(f, [p.data_ptr() for p in self.planes], [o.data_ptr() for o in self.outputs],
                             side_ptrs, unit_ptrs)

    def outputs_numpy(self) -> List[np.ndarray]:
        return [o.cpu().numpy().view(np.uint16) for o in self.outputs]
