"""Host-side description of one frame's post-filter inputs.

`FrameInputs` carries exactly what vaco's decode_frame hands its post-filter
stages (crates/codec/vaco-codec-av1/src/decode.rs:553-559), plus the
deblocking side information vaco parses but cannot use:

  planes        Mi-padded reconstruction planes, uint16 (framebuf.rs:16-20)
  tx_luma       per 4x4 luma cell TX_SIZE (MiCell.tx_size, decode.rs:107-114)
  tx_chroma     per 4x4 chroma cell TX_SIZE (get_tx_size, decode.rs:2438-2468)
  lvl_map       optional per-cell final loop-filter levels (Yv, Yh, U, V)
  skip          per 4x4 luma cell skip flag (MiCell.skip)
  cdef_idx      per-64x64 CDEF strength index, -1 = absent (FrameCtx.cdef_idx)
  deblock/cdef/lr parameters from the frame header

`job()` packs host or device pointers into the C ABI's vaco_av1_frame_job.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import abi


@dataclass
class CdefSettings:
    """src/cdef.rs:24-33 CdefParams."""

    enabled: bool = True
    damping: int = 3
    y_primary: Sequence[int] = (0,) * 8
    y_secondary: Sequence[int] = (0,) * 8
    uv_primary: Sequence[int] = (0,) * 8
    uv_secondary: Sequence[int] = (0,) * 8

    def to_c(self) -> abi.CdefParams:
        p = abi.CdefParams()
        p.enabled = 1 if self.enabled else 0
        p.damping = self.damping
        for k in range(8):
            p.y_primary[k] = self.y_primary[k]
            p.y_secondary[k] = self.y_secondary[k]
            p.uv_primary[k] = self.uv_primary[k]
            p.uv_secondary[k] = self.uv_secondary[k]
        return p


@dataclass
class FrameInputs:
    bit_depth: int
    coded_width: int
    coded_height: int
    upscaled_width: int
    planes: List[np.ndarray]
    tx_luma: np.ndarray
    tx_chroma: np.ndarray
    skip: np.ndarray
    cdef_idx: np.ndarray
    subsampling_x: int = 1
    subsampling_y: int = 1
    monochrome: bool = False
    lvl_map: Optional[np.ndarray] = None
    deblock_levels: Sequence[int] = (0, 0, 0, 0)
    sharpness: int = 0
    cdef: CdefSettings = field(default_factory=CdefSettings)
    lr_type: Sequence[int] = (0, 0, 0)
    lr_unit_size: Sequence[int] = (64, 64, 64)
    lr_units: List[np.ndarray] = field(default_factory=list)

    # ------------------------------------------------------------ geometry
    @property
    def num_planes(self) -> int:
        return 1 if self.monochrome else 3

    @property
    def mi_cols(self) -> int:
        # decode.rs:511-512: mi_cols = 2 * ((coded_width + 7) >> 3)
        return 2 * ((self.coded_width + 7) >> 3)

    @property
    def mi_rows(self) -> int:
        return 2 * ((self.coded_height + 7) >> 3)

    def plane_sub(self, k: int):
        return (self.subsampling_x, self.subsampling_y) if k else (0, 0)

    def padded_shape(self, k: int):
        sx, sy = self.plane_sub(k)
        return ((self.mi_rows * 4) >> sy, (self.mi_cols * 4) >> sx)

    def output_shape(self, k: int):
        """Visible output plane (rows, cols): restoration_plane_config, decode.rs:587-610."""
        sx, sy = self.plane_sub(k)
        return (self.coded_height >> sy, self.upscaled_width >> sx)

    def lr_active(self) -> bool:
        return any(t != abi.FRAME_LR_NONE for t in self.lr_type[: self.num_planes])

    @property
    def output_pixels(self) -> int:
        """Output luma pixels: the Mpixel/s unit."""
        return self.upscaled_width * self.coded_height

    def info(self) -> abi.FrameInfo:
        i = abi.FrameInfo()
        i.bit_depth = self.bit_depth
        i.subsampling_x = self.subsampling_x
        i.subsampling_y = self.subsampling_y
        i.monochrome = 1 if self.monochrome else 0
        i.mi_rows = self.mi_rows
        i.mi_cols = self.mi_cols
        i.coded_width = self.coded_width
        i.coded_height = self.coded_height
        i.upscaled_width = self.upscaled_width
        return i

    def deblock_c(self) -> abi.DeblockParams:
        d = abi.DeblockParams()
        for k in range(4):
            d.levels[k] = self.deblock_levels[k]
        d.sharpness = self.sharpness
        return d

    def side_arrays(self):
        """The side-information arrays in the order the job struct names them."""
        return {
            "tx_luma": self.tx_luma,
            "tx_chroma": self.tx_chroma,
            "lvl_map": self.lvl_map,
            "skip": self.skip,
            "cdef_idx": self.cdef_idx,
        }

    def validate_shapes(self) -> None:
        for k in range(self.num_planes):
            if self.planes[k].shape != self.padded_shape(k) or self.planes[k].dtype != np.uint16:
                raise ValueError(f"plane {k} must be uint16 {self.padded_shape(k)}")
        if self.tx_luma.shape != (self.mi_rows, self.mi_cols):
            raise ValueError("tx_luma shape")
        if self.skip.shape != (self.mi_rows, self.mi_cols):
            raise ValueError("skip shape")


def picture_struct(ptrs: Sequence[int], shapes, strides=None) -> abi.Picture:
    """vaco_av1_picture from plane pointers and (rows, cols) shapes."""
    p = abi.Picture()
    for k in range(3):
        if k < len(ptrs) and ptrs[k]:
            p.planes[k] = ptrs[k]
            p.height[k], p.width[k] = shapes[k]
            p.stride[k] = strides[k] if strides else shapes[k][1]
        else:
            p.planes[k] = None
    return p


def build_job(f: FrameInputs, src_ptrs, dst_ptrs, side_ptrs: dict, unit_ptrs) -> abi.FrameJob:
    """vaco_av1_frame_job from pointers (host or device, as the callee expects)."""
    j = abi.FrameJob()
    j.info = f.info()
    np_ = f.num_planes
    j.src = picture_struct(src_ptrs[:np_], [f.padded_shape(k) for k in range(np_)])
    j.dst = picture_struct(dst_ptrs[:np_], [f.output_shape(k) for k in range(np_)])
    j.tx_luma = side_ptrs.get("tx_luma") or None
    j.tx_chroma = side_ptrs.get("tx_chroma") or None
    j.lvl_map = side_ptrs.get("lvl_map") or None
    j.skip = side_ptrs.get("skip") or None
    j.cdef_idx = side_ptrs.get("cdef_idx") or None
    j.cdef_stride = f.cdef_idx.shape[1]
    j.cdef_count = f.cdef_idx.size
    j.deblock = f.deblock_c()
    j.cdef = f.cdef.to_c()
    for k in range(3):
        j.lr_type[k] = f.lr_type[k] if k < np_ else 0
        j.lr_unit_size[k] = f.lr_unit_size[k]
        if k < np_ and k < len(f.lr_units) and f.lr_units[k] is not None:
            j.lr_units[k] = unit_ptrs[k] or None
            j.lr_unit_count[k] = len(f.lr_units[k])
        else:
            j.lr_units[k] = None
            j.lr_unit_count[k] = 0
    return j


def ptr(a: Optional[np.ndarray]) -> Optional[int]:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def host_job(f: FrameInputs, outputs: List[np.ndarray]) -> abi.FrameJob:
    """A job over host numpy arrays (for the `_host` entry points and the oracle)."""
    side = {k: ptr(v) for k, v in f.side_arrays().items()}
    units = [ptr(f.lr_units[k]) if k < len(f.lr_units) else None for k in range(3)]
    return build_job(f, [ptr(p) for p in f.planes], [ptr(o) for o in outputs], side, units)


def alloc_outputs(f: FrameInputs) -> List[np.ndarray]:
    return [np.zeros(f.output_shape(k), np.uint16) for k in range(f.num_planes)]


def pinned_copy(f: FrameInputs):
    """f with every host array in page-locked memory, plus pinned output
    planes: the best case for the `_host` entry points, whose copies then
    run at full PCIe/C2C speed.  Returns (frame, outputs, job)."""
    import dataclasses

    import torch

    def pin(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    pf = dataclasses.replace(f)
    pf.planes = [pin(p) for p in f.planes]
    pf.tx_luma, pf.tx_chroma, pf.skip = pin(f.tx_luma), pin(f.tx_chroma), pin(f.skip)
    pf.cdef_idx = pin(f.cdef_idx)
    pf.lvl_map = None if f.lvl_map is None else pin(f.lvl_map)
    pf.lr_units = [pin(u.view(np.uint8)).view(u.dtype) for u in f.lr_units]
    outs = [pin(o) for o in alloc_outputs(pf)]
    return pf, outs, host_job(pf, outs)


def frame_layout(info: "abi.FrameInfo", fill: int = 0) -> List[np.ndarray]:
    """Host planes of an emitted frame in vaco's layout (vaco-pixfmt
    plane_layout with vaco-pool's 64-byte row alignment): rows of
    ceil(samples * bytes per sample / 64) * 64 bytes, chroma extents rounded
    up.  `fill` marks the bytes the emission must leave alone."""
    bps = 2 if info.bit_depth > 8 else 1
    out = []
    for k in range(1 if info.monochrome else 3):
        sx = info.subsampling_x if k else 0
        sy = info.subsampling_y if k else 0
        w = (info.upscaled_width + (1 << sx) - 1) >> sx
        h = (info.coded_height + (1 << sy) - 1) >> sy
        line = (w * bps + 63) // 64 * 64
        out.append(np.full((h, line), fill, np.uint8))
    return out


def frame_buffer(planes: Sequence[np.ndarray]) -> "abi.FrameBuffer":
    """A vaco_av1_frame_buffer over host uint8 planes (rows x linesize)."""
    fb = abi.FrameBuffer()
    for k, b in enumerate(planes):
        fb.planes[k] = b.ctypes.data
        fb.linesize[k] = b.shape[1]
    return fb
