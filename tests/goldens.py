"""Golden-vector cases for the AV1 post-filters, rebuilt exactly as vaco's own
tests build them, with the expected outputs read from tests/golden/.

  CDEF          crates/tool/vaco-checkasm/tests/av1_cdef.rs:28-83 (7,680 cases)
  superres      crates/codec/vaco-codec-av1/tests/superres.rs:22-84 (18 records)
  restoration   crates/codec/vaco-codec-av1/tests/restoration.rs:142-227 (300 cases)
                and :49-93 (48 constant SGR cases + Wiener identity)
"""
from __future__ import annotations

import functools
import gzip
import pathlib

import numpy as np

from vaco_b200 import abi

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _read(name: str) -> bytes:
    return gzip.decompress((GOLDEN / name).read_bytes())


def _xorshift32(state: int) -> int:
    state ^= (state << 13) & 0xFFFFFFFF
    state ^= state >> 17
    state ^= (state << 5) & 0xFFFFFFFF
    return state & 0xFFFFFFFF


# ---------------------------------------------------------------- CDEF
@functools.lru_cache(maxsize=1)
def cdef_cases():
    """Inputs (7680,144), params (structured), expected dir, var, out (7680,64)."""
    raw = _read("av1-cdef-dav1d.bin.gz")
    n = 3 * 5 * 8 * 16 * 4
    assert len(raw) == n * 136
    inputs = np.zeros((n, 144), np.uint16)
    params = np.zeros(n, abi.cdef_filter_params_dtype())
    cid = 0
    for bd in (8, 10, 12):
        low = (1 << (bd - 8)) - 1
        for damping in range(2, 7):
            for direction in range(8):
                for primary in range(16):
                    for secondary in (0, 1, 2, 4):
                        state = (0x9E3779B9 ^ cid) & 0xFFFFFFFF
                        for k in range(144):
                            state = _xorshift32(state)
                            hi = (96 + state % 33) if cid & 1 else (state & 255)
                            inputs[cid, k] = ((hi << (bd - 8)) | ((state >> 8) & 0xFFFF & low)) & 0xFFFF
                        p = params[cid]
                        p["width"] = 8 if cid % 3 == 0 else 4
                        p["height"] = 4 if cid % 3 == 2 else 8
                        p["edges"] = (cid // 3) % 16
                        p["bit_depth"] = bd
                        p["direction"] = direction
                        p["primary"] = primary << (bd - 8)
                        p["secondary"] = secondary << (bd - 8)
                        p["damping"] = damping + bd - 8
                        cid += 1
    rec = np.frombuffer(raw, np.uint8).reshape(n, 136)
    exp_dir = rec[:, 0:4].copy().view("<u4").reshape(n)
    exp_var = rec[:, 4:8].copy().view("<u4").reshape(n)
    exp_out = rec[:, 8:].copy().view("<u2").reshape(n, 64)
    return inputs, params, exp_dir, exp_var, exp_out


def cdef_luma_blocks(inputs: np.ndarray) -> np.ndarray:
    """The 8x8 centre of each 12x12 neighborhood (av1_cdef.rs:90-95)."""
    return inputs.reshape(-1, 12, 12)[:, 2:10, 2:10].reshape(-1, 64).copy()


# ---------------------------------------------------------------- superres
@functools.lru_cache(maxsize=1)
def superres_cases():
    """List of dicts: bd, visible, padded, out, height, input (h, padded), expected (h, out)."""
    raw = np.frombuffer(_read("superres-dav1d.u16le.gz"), "<u2")
    cases, off, case_id = [], 0, 0
    while off < raw.size:
        bd, vis, padded, out, h = (int(v) for v in raw[off: off + 5])
        off += 5
        mx = (1 << bd) - 1
        state = (0x6D2B79F5 ^ case_id) & 0xFFFFFFFF
        inp = np.zeros((h, padded), np.uint16)
        for y in range(h):
            for x in range(padded):
                state = _xorshift32(state)
                inp[y, x] = ((state + x * 37 + y * 91) & 0xFFFF) & mx
        exp = raw[off: off + out * h].reshape(h, out).copy()
        off += out * h
        cases.append(dict(bd=bd, visible=vis, padded=padded, out=out, height=h, input=inp,
                          expected=exp))
        case_id += 1
    assert case_id == 18
    return cases


# ---------------------------------------------------------------- restoration
LR_GEOMETRIES = [(7, 9, False, 64), (13, 65, False, 64), (97, 130, False, 64),
                 (48, 81, True, 32), (135, 129, False, 128)]


def lr_sample(x, y, depth, after):
    """tests/restoration.rs:142-145."""
    return ((x * 71 + y * 47 + x * y * 13 + (39 if after else 0)) ^ ((x + y) * 29)) & ((1 << depth) - 1)


def lr_oracle_unit(mode: int, index: int, chroma: bool):
    """tests/restoration.rs:147-169 as a vaco_av1_lr_unit tuple."""
    if mode < 16:
        return (abi.LR_SGRPROJ, (mode + index) % 16, (0, 0, 0), (0, 0, 0),
                (-96 + (mode * 11 + index * 7) % 128, -32 + (mode * 17 + index * 13) % 128))
    coeffs = [[-5, -23, -17], [10, 8, 46], [3, -7, 15], [0, 0, 0]]
    horizontal = list(coeffs[(mode - 16 + index) % 4])
    vertical = list(coeffs[(mode - 16 + index + 1) % 4])
    if chroma:
        horizontal[0] = 0
        vertical[0] = 0
    return (abi.LR_WIENER, 0, tuple(vertical), tuple(horizontal), (0, 0))


def lr_units_array(tuples) -> np.ndarray:
    a = np.zeros(len(tuples), abi.lr_unit_dtype())
    for i, (t, s, v, h, q) in enumerate(tuples):
        a[i]["type"], a[i]["set"] = t, s
        a[i]["vertical"], a[i]["horizontal"], a[i]["xqd"] = v, h, q
    return a


def lr_unit_counts(width, height, unit_size):
    c = lambda e: max((e + unit_size // 2) // unit_size, 1)  # noqa: E731
    return c(width), c(height)


@functools.lru_cache(maxsize=1)
def lr_cases():
    """300 cases: dict(bd, width, height, sub_y, unit_size, mode, before, after, units, expected)."""
    raw = np.frombuffer(_read("restoration-dav1d-8.u16le.gz") + _read("restoration-dav1d-high.u16le.gz"),
                        "<u2")
    cases, off = [], 0
    for bd in (8, 10, 12):
        for (w, h, sub_y, unit) in LR_GEOMETRIES:
            ys, xs = np.mgrid[0:h, 0:w]
            before = np.zeros((h + 8, w + 8), np.uint16)
            after = np.zeros((h + 8, w + 8), np.uint16)
            before[:h, :w] = lr_sample(xs, ys, bd, False)
            after[:h, :w] = lr_sample(xs, ys, bd, True)
            cols, rows = lr_unit_counts(w, h, unit)
            for mode in range(20):
                units = lr_units_array([lr_oracle_unit(mode, i, sub_y) for i in range(cols * rows)])
                exp = raw[off: off + w * h].reshape(h, w).copy()
                off += w * h
                cases.append(dict(bd=bd, width=w, height=h, sub_y=sub_y, unit_size=unit, mode=mode,
                                  before=before, after=after, units=units, expected=exp))
    assert off == raw.size and len(cases) == 300
    return cases


@functools.lru_cache(maxsize=1)
def lr_constant_cases():
    """48 SGR cases on a constant 7x9 plane at the depth's maximum value."""
    raw = np.frombuffer(_read("restoration-constant-8.u16le.gz") + _read("restoration-constant-high.u16le.gz"),
                        "<u2")
    cases, off = [], 0
    for bd in (8, 10, 12):
        plane = np.full((9, 7), (1 << bd) - 1, np.uint16)
        for s in range(16):
            units = lr_units_array([(abi.LR_SGRPROJ, s, (0, 0, 0), (0, 0, 0), (-32, 31))])
            cases.append(dict(bd=bd, plane=plane, units=units, set=s,
                              expected=raw[off: off + 63].reshape(9, 7).copy()))
            off += 63
    assert off == raw.size
    return cases
