"""Cross-check of the deblocking oracle's sample filter against vaco's own VP9
loop filter, on random lines, where the two specifications coincide.

vaco has no AV1 deblocking filter, so the oracle's AV1 7.14 restatement has
no golden vector.  vaco's VP9 loop filter
(crates/codec/vaco-codec-vp9/src/loopfilter.rs) shares part of the
arithmetic with it:

  * the strength derivation: limit / blimit / thresh from the level and the
    sharpness (adaptive_strength, loopfilter.rs:377-388; AV1 7.14.4);
  * the narrow filter (filter4_clamp :497-499, narrow_filter :501-547; AV1
    7.14.6.3), driven by the same hev test (:418-420);
  * for a luma edge of filter size 8, the whole sample filter: the filter
    mask over p3..q3 (:422-432), the flat mask over p3..q3 (:434-445) and the
    choice between the narrow filter and the log2Size = 3 wide filter
    (:447-477, wide_filter :560-600), which is AV1's 8-tap luma filter.

The VP9 functions are restated below line for line in numpy (vectorised over
lines) and compared with the oracle's filter (oracle/vaco_oracle.cpp
Deblocker::filter_line) bit-exactly.  Where the specifications differ -- the
AV1 4-tap mask reads only p1..q1, chroma uses a 6-tap filter, luma size 16 a
13-tap one -- there is nothing in vaco to compare with: the 4-tap case is
compared on the lines VP9's mask admits, and the 6-tap and 14-tap filters
stay unpinned.
"""
import numpy as np
import pytest

import oracle

N_LINES = 120_000  # per bit depth and filter size


# ---------------------------------------------------------------- VP9 restatement (loopfilter.rs)
def vp9_strength(lvl, sharpness):
    """adaptive_strength (:377-388): (limit, blimit, thresh) from lvl."""
    shift = 2 if sharpness > 4 else int(sharpness > 0)
    if sharpness > 0:
        limit = np.clip(lvl >> shift, 1, 9 - sharpness)
    else:
        limit = np.maximum(lvl >> shift, 1)
    blimit = 2 * (lvl + 2) + limit
    thresh = lvl >> 4
    return limit, blimit, thresh


def vp9_filter4_clamp(v, bd):
    """filter4_clamp (:497-499)."""
    return np.clip(v, -(1 << (bd - 1)), (1 << (bd - 1)) - 1)


def vp9_narrow_filter(s, out, sel, hev, bd):
    """narrow_filter (:501-547) on the lines `sel`; s[:, 8 + i] = sample(i)."""
    q0, q1, p0, p1 = s[:, 8], s[:, 9], s[:, 7], s[:, 6]
    bias = 0x80 << (bd - 8)
    ps1, ps0, qs0, qs1 = p1 - bias, p0 - bias, q0 - bias, q1 - bias
    filt = np.where(hev, vp9_filter4_clamp(ps1 - qs1, bd), 0)
    filt = vp9_filter4_clamp(filt + 3 * (qs0 - ps0), bd)
    filter1 = vp9_filter4_clamp(filt + 4, bd) >> 3
    filter2 = vp9_filter4_clamp(filt + 3, bd) >> 3
    oq0 = vp9_filter4_clamp(qs0 - filter1, bd) + bias
    op0 = vp9_filter4_clamp(ps0 + filter2, bd) + bias
    mx = (1 << bd) - 1
    out[sel, 8] = np.clip(oq0, 0, mx)[sel]
    out[sel, 7] = np.clip(op0, 0, mx)[sel]
    r = (filter1 + 1) >> 1  # round1
    oq1 = vp9_filter4_clamp(qs1 - r, bd) + bias
    op1 = vp9_filter4_clamp(ps1 + r, bd) + bias
    nh = sel & ~hev
    out[nh, 9] = np.clip(oq1, 0, mx)[nh]
    out[nh, 6] = np.clip(op1, 0, mx)[nh]


def vp9_wide_filter(s, out, sel, log2_size, bd):
    """wide_filter (:560-600): t = sample(i) + sum_j sample(clamp(i + j))."""
    n = (1 << (log2_size - 1)) - 1
    mx = (1 << bd) - 1
    res = {}
    for i in range(-n, n):
        t = s[:, 8 + i].copy()
        for j in range(-n, n + 1):
            t += s[:, 8 + int(np.clip(i + j, -(n + 1), n))]
        res[i] = (t + (1 << (log2_size - 1))) >> log2_size
    for i in range(-n, n):
        out[sel, 8 + i] = np.clip(res[i], 0, mx)[sel]


def vp9_filter_sample(s, lvl, sharpness, filter_size_is_8, bd):
    """filter_sample (:392-477) for TX_4X4 (False) or TX_8X8 (True) on a
    luma line; returns (output lines, lines the filter mask admitted)."""
    q0, q1, q2, q3 = s[:, 8], s[:, 9], s[:, 10], s[:, 11]
    p0, p1, p2, p3 = s[:, 7], s[:, 6], s[:, 5], s[:, 4]
    limit, blimit, thresh = vp9_strength(lvl, sharpness)
    shift_bd = bd - 8
    thresh_bd = thresh << shift_bd
    hev = (np.abs(p1 - p0) > thresh_bd) | (np.abs(q1 - q0) > thresh_bd)
    limit_bd, blimit_bd = limit << shift_bd, blimit << shift_bd
    mask = np.abs(p3 - p2) > limit_bd
    mask |= np.abs(p2 - p1) > limit_bd
    mask |= np.abs(p1 - p0) > limit_bd
    mask |= np.abs(q1 - q0) > limit_bd
    mask |= np.abs(q2 - q1) > limit_bd
    mask |= np.abs(q3 - q2) > limit_bd
    mask |= np.abs(p0 - q0) * 2 + np.abs(p1 - q1) // 2 > blimit_bd
    admit = ~mask
    thr = 1 << shift_bd
    m = np.abs(p1 - p0) > thr
    m |= np.abs(q1 - q0) > thr
    m |= np.abs(p2 - p0) > thr
    m |= np.abs(q2 - q0) > thr
    m |= np.abs(p3 - p0) > thr
    m |= np.abs(q3 - q0) > thr
    flat = np.full(len(s), bool(filter_size_is_8)) & ~m
    out = s.copy()
    vp9_narrow_filter(s, out, admit & ~flat, hev, bd)
    vp9_wide_filter(s, out, admit & flat, 3, bd)
    return out, admit


# ---------------------------------------------------------------- random lines
def random_lines(rng, n, bd):
    """A mix that reaches every branch: smooth lines with a step at the edge
    (flat and wide filters), moderately noisy lines (narrow filter, hev on and
    off) and uniformly random lines (mask rejects)."""
    mx = (1 << bd) - 1
    one = 1 << (bd - 8)
    kind = rng.integers(0, 3, n)
    base_p = rng.integers(0, mx + 1, n)
    step = rng.integers(-24 * one, 24 * one + 1, n)
    base_q = np.clip(base_p + step, 0, mx)
    lines = np.empty((n, 16), np.int64)
    lines[:, :8] = base_p[:, None]
    lines[:, 8:] = base_q[:, None]
    noise = np.where(kind[:, None] == 0, rng.integers(-one, one + 1, (n, 16)),
                     rng.integers(-6 * one, 6 * one + 1, (n, 16)))
    lines = np.clip(lines + noise, 0, mx)
    uniform = rng.integers(0, mx + 1, (n, 16))
    return np.where(kind[:, None] == 2, uniform, lines)


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_luma_size8_sample_filter_equals_vp9(bd):
    rng = np.random.default_rng(0x7E9 + bd)
    for sharpness in (0, 3, 7):
        lines = random_lines(rng, N_LINES // 3, bd)
        lvl = rng.integers(1, 64, len(lines))
        want, admit = vp9_filter_sample(lines, lvl, sharpness, True, bd)
        got = oracle.deblock_lines(lines, 0, 8, lvl, sharpness, bd).astype(np.int64)
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert bad.size == 0, (f"bd={bd} sharpness={sharpness}: {bad.size} lines differ, first {lines[bad[0]]} "
                               f"lvl={lvl[bad[0]]}: oracle {got[bad[0]]} vp9 {want[bad[0]]}")
        changed = (want != lines).any(axis=1)
        # every branch was reached: rejected, narrow and wide lines
        assert (~admit).sum() > 1000 and changed.sum() > 1000
        assert (want[:, 5] != lines[:, 5]).sum() > 100  # p2 written: the wide filter ran


@pytest.mark.parametrize("bd", [8, 10, 12])
@pytest.mark.parametrize("plane", [0, 1])
def test_size4_narrow_filter_equals_vp9_where_vp9_filters(bd, plane):
    rng = np.random.default_rng(0x4E9 + bd + 16 * plane)
    sharpness = int(rng.integers(0, 8))
    lines = random_lines(rng, N_LINES // 2, bd)
    lvl = rng.integers(1, 64, len(lines))
    want, admit = vp9_filter_sample(lines, lvl, sharpness, False, bd)
    got = oracle.deblock_lines(lines, plane, 4, lvl, sharpness, bd).astype(np.int64)
    # VP9's mask also reads p3, p2, q2, q3; where it admits a line, the AV1
    # 4-tap mask (p1..q1 only) admits it too and the narrow filters agree.
    assert admit.sum() > len(lines) // 5
    bad = np.nonzero((got[admit] != want[admit]).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} admitted lines differ"
    # The 4-tap filter writes only p1, p0, q0, q1 on every line.
    outside = np.r_[0:6, 10:16]
    assert (got[:, outside] == lines[:, outside]).all()
