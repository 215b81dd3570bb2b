"""Seeded synthetic frames for the five post-filter workloads.

No public corpus is involved: every frame is generated here from numpy's
PCG64 with seed 0xA1F0 + 1000*config + frame_index, so the CPU oracle, the
CUDA library and the benchmark all see identical bytes.

Content model (per plane, at the plane's own resolution):
  128 + sum of 3 sinusoids A*sin(2*pi*(u*x + v*y)/P + phi), P ~ U[32, 512] px,
  random orientation, amplitudes splitting a +-112 swing (so [16, 240]),
  plus N(0, 4) noise, clipped to 0..255.  10-bit frames compute the same in
  8-bit float units, scale by 1023/255, round and clip to 0..1023.

Side information:
  deblocking  64x64 superblocks split recursively (square 64..8 plus the
              64x32/32x64/32x16/16x32/16x8/8x16 halves), each block carrying a
              transform size 4x4..64x64 (depth 0-2 below its largest
              rectangular size); chroma sizes follow get_tx_size
              (vaco src/decode.rs:2438-2468).  All blocks intra.  Frame levels
              [Yv, Yh, U, V] ~ U{0..63}, U/V forced to 0 when both Y levels are
              0 (AV1 loop_filter_params syntax).
  CDEF        cdef_bits = 3: 8 presets with primary ~ U{0..15} and secondary
              ~ U{0,1,2,4} drawn separately for luma and chroma, damping
              ~ U{3..6}, per-64x64 index ~ U{0..7}, 20% of 8x8 blocks skipped.
  restoration unit size 64 on every plane; each unit Wiener / self-guided /
              none with probability 1/3 each.  Wiener taps uniform over the
              coded ranges [-5,10], [-23,8], [-17,46] (chroma outer tap 0);
              self-guided set ~ U{0..15} with coefficients from [-96,31] and
              [-32,95], an unused pass's coefficient derived as
              read_sgrproj_unit does (vaco src/decode.rs:1261-1291).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import abi
from .frame import CdefSettings, FrameInputs

# AV1 TX_SIZE enum: (width, height) -> value
TX_BY_DIMS = {
    (4, 4): 0, (8, 8): 1, (16, 16): 2, (32, 32): 3, (64, 64): 4, (4, 8): 5, (8, 4): 6,
    (8, 16): 7, (16, 8): 8, (16, 32): 9, (32, 16): 10, (32, 64): 11, (64, 32): 12,
    (4, 16): 13, (16, 4): 14, (8, 32): 15, (32, 8): 16, (16, 64): 17, (64, 16): 18,
}
# Sgr_Params radii (radius of pass 0, pass 1) per set, AV1 7.17.3
SGR_RADII = [(2, 1)] * 10 + [(0, 1)] * 4 + [(2, 0)] * 2


@dataclass
class Workload:
    """One named configuration."""

    name: str
    width: int           # coded luma width
    height: int
    bit_depth: int
    upscaled_width: int  # == width without superres
    chain: bool          # deblock + CDEF + LR (False: CDEF only)


# The five configurations (config index -> workload or frame mix)
CONFIG0 = Workload("cdef_1080p_8bit", 1920, 1080, 8, 1920, chain=False)
CONFIG1 = Workload("chain_4k_10bit", 3840, 2160, 10, 3840, chain=True)
CONFIG2 = Workload("superres_2880to3840_10bit", 2880, 2160, 10, 3840, chain=True)
CONFIG2_DENOM12 = Workload("superres_2560to3840_10bit", 2560, 2160, 10, 3840, chain=True)
BATCH_MIX = [
    (Workload("chain_360p_8bit", 640, 360, 8, 640, True), 16),
    (Workload("chain_720p_8bit", 1280, 720, 8, 1280, True), 16),
    (Workload("chain_1080p_10bit", 1920, 1080, 10, 1920, True), 16),
    (Workload("chain_4k_10bit", 3840, 2160, 10, 3840, True), 16),
]


def seed_for(config: int, frame_index: int) -> int:
    return 0xA1F0 + 1000 * config + frame_index


def content_plane(rng: np.random.Generator, rows: int, cols: int, bit_depth: int) -> np.ndarray:
    ys = np.arange(rows, dtype=np.float32)[:, None]
    xs = np.arange(cols, dtype=np.float32)[None, :]
    acc = np.full((rows, cols), 128.0, np.float32)
    amps = rng.dirichlet([2.0, 2.0, 2.0]) * 112.0
    for k in range(3):
        period = rng.uniform(32.0, 512.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        u, v = np.cos(theta) / period, np.sin(theta) / period
        acc += np.float32(amps[k]) * np.sin(np.float32(2.0 * np.pi) * (xs * np.float32(u) + ys * np.float32(v)) + np.float32(phase))
    acc += rng.normal(0.0, 4.0, size=(rows, cols)).astype(np.float32)
    if bit_depth == 8:
        return np.clip(np.rint(acc), 0, 255).astype(np.uint16)
    scaled = acc * np.float32(((1 << bit_depth) - 1) / 255.0)
    return np.clip(np.rint(scaled), 0, (1 << bit_depth) - 1).astype(np.uint16)


def _partition(rng, r0, c0, size, mi_rows, mi_cols, out):
    """Recursive 64x64 split; appends (mi_row, mi_col, mi_h, mi_w)."""
    n = size // 4
    inside = r0 + n <= mi_rows and c0 + n <= mi_cols
    if r0 >= mi_rows or c0 >= mi_cols:
        return
    if not inside and size > 8:
        for dr in (0, n // 2):
            for dc in (0, n // 2):
                _partition(rng, r0 + dr, c0 + dc, size // 2, mi_rows, mi_cols, out)
        return
    choice = rng.integers(0, 4) if size > 8 else 0
    if size == 64 and choice == 0 and rng.random() < 0.5:
        choice = 3  # fewer 64x64 blocks: more edges
    if choice == 0:
        out.append((r0, c0, n, n))
    elif choice == 1:  # horizontal halves
        out.append((r0, c0, n // 2, n))
        out.append((r0 + n // 2, c0, n // 2, n))
    elif choice == 2:  # vertical halves
        out.append((r0, c0, n, n // 2))
        out.append((r0, c0 + n // 2, n, n // 2))
    else:
        for dr in (0, n // 2):
            for dc in (0, n // 2):
                _partition(rng, r0 + dr, c0 + dc, size // 2, mi_rows, mi_cols, out)


def tx_maps(rng, mi_rows: int, mi_cols: int, ssx: int = 1, ssy: int = 1):
    """Luma and chroma TX_SIZE maps for a random intra partition."""
    blocks = []
    for r in range(0, mi_rows, 16):
        for c in range(0, mi_cols, 16):
            _partition(rng, r, c, 64, mi_rows, mi_cols, blocks)
    tx_l = np.zeros((mi_rows, mi_cols), np.uint8)
    cr, cc = (mi_rows + ssy) >> ssy, (mi_cols + ssx) >> ssx
    tx_c = np.zeros((cr, cc), np.uint8)
    depths = rng.integers(0, 3, size=len(blocks))
    for (r, c, h, w), d in zip(blocks, depths):
        bw, bh = 4 * w, 4 * h
        tw, th = max(min(bw, 64) >> d, 4), max(min(bh, 64) >> d, 4)
        tx_l[r: r + h, c: c + w] = TX_BY_DIMS[(tw, th)]
        cw, ch = max(bw >> ssx, 4), max(bh >> ssy, 4)
        uw, uh = min(cw, 32), min(ch, 32)
        tx_c[r >> ssy: (r + h + ssy) >> ssy, c >> ssx: (c + w + ssx) >> ssx] = TX_BY_DIMS[(uw, uh)]
    return tx_l, tx_c


def lr_units(rng, width: int, height: int, unit_size: int, chroma: bool) -> np.ndarray:
    cols = max((width + unit_size // 2) // unit_size, 1)
    rows = max((height + unit_size // 2) // unit_size, 1)
    n = cols * rows
    units = np.zeros(n, abi.lr_unit_dtype())
    types = rng.integers(0, 3, size=n)
    for i in range(n):
        t = int(types[i])
        if t == 1:
            v = [int(rng.integers(-5, 11)), int(rng.integers(-23, 9)), int(rng.integers(-17, 47))]
            h = [int(rng.integers(-5, 11)), int(rng.integers(-23, 9)), int(rng.integers(-17, 47))]
            if chroma:
                v[0] = h[0] = 0
            units[i]["type"] = abi.LR_WIENER
            units[i]["vertical"], units[i]["horizontal"] = v, h
        elif t == 2:
            s = int(rng.integers(0, 16))
            r0, r1 = SGR_RADII[s]
            x0 = int(rng.integers(-96, 32)) if r0 else 0
            x1 = int(rng.integers(-32, 96)) if r1 else int(np.clip(128 - x0, -32, 95))
            units[i]["type"] = abi.LR_SGRPROJ
            units[i]["set"] = s
            units[i]["xqd"] = (x0, x1)
    return units


def cdef_settings(rng) -> CdefSettings:
    secs = np.array([0, 1, 2, 4])
    return CdefSettings(
        enabled=True,
        damping=int(rng.integers(3, 7)),
        y_primary=[int(v) for v in rng.integers(0, 16, 8)],
        y_secondary=[int(v) for v in secs[rng.integers(0, 4, 8)]],
        uv_primary=[int(v) for v in rng.integers(0, 16, 8)],
        uv_secondary=[int(v) for v in secs[rng.integers(0, 4, 8)]],
    )


def make_frame(w: Workload, seed: int, *, sharpness: Optional[int] = 0, with_lvl_map: bool = False,
               lr_unit: int = 64, subsampling=(1, 1), monochrome: bool = False) -> FrameInputs:
    """A seeded frame.  subsampling = (x, y): (1, 1) 4:2:0, (1, 0) 4:2:2,
    (0, 0) 4:4:4; monochrome keeps luma only (the chroma planes are still
    drawn, so the luma content matches the 4:2:0 frame of the same seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ssx, ssy = subsampling
    mi_cols = 2 * ((w.width + 7) >> 3)
    mi_rows = 2 * ((w.height + 7) >> 3)
    planes: List[np.ndarray] = []
    for k in range(3):
        sx, sy = (ssx, ssy) if k else (0, 0)
        planes.append(content_plane(rng, (mi_rows * 4) >> sy, (mi_cols * 4) >> sx, w.bit_depth))
    tx_l, tx_c = tx_maps(rng, mi_rows, mi_cols, ssx, ssy)
    # 20% of 8x8 blocks skipped (all four 4x4 cells)
    skip8 = (rng.random(((mi_rows + 1) // 2, (mi_cols + 1) // 2)) < 0.2).astype(np.uint8)
    skip = np.repeat(np.repeat(skip8, 2, 0), 2, 1)[:mi_rows, :mi_cols].copy()
    idx = rng.integers(0, 8, size=((mi_rows + 15) // 16, (mi_cols + 15) // 16)).astype(np.int32)
    cdef = cdef_settings(rng)
    levels = [int(v) for v in rng.integers(0, 64, 4)]
    if levels[0] == 0 and levels[1] == 0:
        levels[2] = levels[3] = 0
    if sharpness is None:
        sharpness = int(rng.integers(0, 8))
    lvl_map = None
    if with_lvl_map:
        base = np.array(levels, np.int32)
        delta = rng.integers(-8, 9, size=((mi_rows + 15) // 16, (mi_cols + 15) // 16, 1))
        per_sb = np.clip(base[None, None, :] + delta, 0, 63)
        lvl_map = np.repeat(np.repeat(per_sb, 16, 0), 16, 1)[:mi_rows, :mi_cols].astype(np.uint8).copy()
    f = FrameInputs(
        bit_depth=w.bit_depth, coded_width=w.width, coded_height=w.height,
        upscaled_width=w.upscaled_width, planes=planes, tx_luma=tx_l, tx_chroma=tx_c,
        skip=skip, cdef_idx=idx, lvl_map=lvl_map, sharpness=sharpness, cdef=cdef,
        subsampling_x=ssx, subsampling_y=ssy, monochrome=monochrome,
    )
    if w.chain:
        f.deblock_levels = levels
        f.lr_type = (abi.FRAME_LR_SWITCHABLE,) * 3
        f.lr_unit_size = (lr_unit, lr_unit, lr_unit)
        f.lr_units = []
        for k in range(3):
            rows, cols = f.output_shape(k)
            units = lr_units(rng, cols, rows, lr_unit, k > 0)
            if k < f.num_planes:
                f.lr_units.append(units)
    else:
        f.deblock_levels = (0, 0, 0, 0)
        f.lr_type = (abi.FRAME_LR_NONE,) * 3
        f.lr_units = []
    return f


def make_small(seed: int, width: int = 200, height: int = 136, bit_depth: int = 10,
               upscaled_width: Optional[int] = None, chain: bool = True, **kw) -> FrameInputs:
    """A small frame of arbitrary geometry for parity tests."""
    w = Workload("small", width, height, bit_depth, upscaled_width or width, chain)
    return make_frame(w, seed, **kw)
