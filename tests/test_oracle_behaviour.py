"""Behavioural tests ported from vaco's own unit tests, run on the CPU oracle
(and, for geometry, on the host-side PlaneConfig mirror).

  crates/codec/vaco-codec-av1/tests/restoration.rs:23-46, 96-140, 229-264
  crates/codec/vaco-codec-av1/src/cdef_frame_tests.rs:72-105
"""
import numpy as np
import pytest

import goldens
import oracle
from vaco_b200 import abi, synth
from vaco_b200.frame import CdefSettings, FrameInputs
from vaco_b200.restoration import PlaneConfig


def test_unit_geometry_merges_short_tails_and_shifts_vertical_boundaries():
    config = PlaneConfig(width=95, height=161, bit_depth=8, unit_size=64, subsampling_y=False)
    assert config.unit_counts() == (1, 3)
    assert config.unit_index(94, 55) == 0
    assert config.unit_index(94, 56) == 1
    assert config.unit_index(94, 119) == 1
    assert config.unit_index(94, 120) == 2
    chroma = PlaneConfig(width=48, height=81, bit_depth=8, unit_size=32, subsampling_y=True)
    assert chroma.unit_counts() == (2, 3)
    assert chroma.unit_index(32, 27) == 1
    assert chroma.unit_index(32, 28) == 3


def test_invalid_configuration_and_coefficients_are_rejected():
    plane = np.full((4, 4), 100, np.uint16)
    none = np.zeros(1, abi.lr_unit_dtype())
    for (w, h, bd, unit) in [(4, 4, 8, 0), (4, 4, 16, 64), (5, 4, 8, 64), (4, 0, 8, 64)]:
        _, m = oracle.restore_plane(plane, plane, w, h, bd, unit, False, none)
        assert m == abi.MSG["LR_GEOMETRY"]
    for unit in [(2, 16, (0, 0, 0), (0, 0, 0), (0, 0)), (2, 0, (0, 0, 0), (0, 0, 0), (32, 0)),
                 (1, 0, (11, 0, 0), (0, 0, 0), (0, 0))]:
        _, m = oracle.restore_plane(plane, plane, 4, 4, 8, 64, False, goldens.lr_units_array([unit]))
        assert m == abi.MSG["LR_COEFFICIENT"]
    _, m = oracle.restore_plane(plane, plane, 4, 4, 8, 64, False, np.zeros(0, abi.lr_unit_dtype()))
    assert m == abi.MSG["LR_UNIT_COUNT"]


def test_none_preserves_visible_cdef_pixels_and_out_of_depth_input_is_rejected():
    before = np.full((12, 12), 16, np.uint16)
    after = np.full((12, 12), 235, np.uint16)
    none = np.zeros(1, abi.lr_unit_dtype())
    out, m = oracle.restore_plane(before, after, 7, 9, 8, 64, False, none)
    assert m == 0 and out.shape == (9, 7) and (out == 235).all()
    after[8, 6] = 256
    _, m = oracle.restore_plane(before, after, 7, 9, 8, 64, False, none)
    assert m == abi.MSG["LR_SAMPLE"]


def cdef_context():
    """src/cdef_frame_tests.rs:12-69: a 16x16 monochrome 8-bit picture, every
    cell skipped, damping 6, luma strengths (15, 4) for all eight entries."""
    ys, xs = np.mgrid[0:16, 0:16]
    plane = (70 + ys * 5 + (xs % 2) * 3).astype(np.uint16)
    return FrameInputs(
        bit_depth=8, coded_width=16, coded_height=16, upscaled_width=16, planes=[plane],
        tx_luma=np.zeros((4, 4), np.uint8), tx_chroma=np.zeros((2, 2), np.uint8),
        skip=np.ones((4, 4), np.uint8), cdef_idx=np.zeros((1, 1), np.int32), monochrome=True,
        cdef=CdefSettings(enabled=True, damping=6, y_primary=[15] * 8, y_secondary=[4] * 8,
                          uv_primary=[0] * 8, uv_secondary=[0] * 8))


def cdef_frame_cases(run):
    """Shared by the oracle test here and the GPU test in test_gpu_behaviour.py."""
    for active in (0, 1, 4, 5):
        f = cdef_context()
        before = f.planes[0].copy()
        out = run(f)
        np.testing.assert_array_equal(out[0], before)
        f.skip.reshape(-1)[active] = 0
        out = run(f)[0]
        region = np.zeros((16, 16), bool)
        region[:8, :8] = True
        np.testing.assert_array_equal(out[~region], before[~region])
        assert (out[region] != before[region]).sum() > 0
    f = cdef_context()
    f.skip[:] = 0
    f.cdef_idx[0, 0] = -1
    np.testing.assert_array_equal(run(f)[0], f.planes[0])


def test_cdef_frame_skip_and_missing_index_semantics():
    def run(f):
        out, m = oracle.cdef_picture(f)
        assert m == 0
        return out
    cdef_frame_cases(run)


def test_deblock_level_zero_is_identity_and_flat_input_is_unchanged():
    f = synth.make_small(21, 136, 72, 10)
    f.deblock_levels = (0, 0, 17, 30)
    out, m = oracle.deblock_picture(f)
    assert m == 0
    for o, p in zip(out, f.planes):
        np.testing.assert_array_equal(o, p)
    f = synth.make_small(21, 136, 72, 10)
    f.deblock_levels = (40, 40, 40, 40)
    f.planes = [np.full_like(p, 512) for p in f.planes]
    out, m = oracle.deblock_picture(f)
    assert m == 0
    for o, p in zip(out, f.planes):
        np.testing.assert_array_equal(o, p)


def test_deblock_only_touches_samples_near_transform_edges():
    f = synth.make_small(22, 200, 136, 8)
    f.deblock_levels = (63, 63, 63, 63)
    out, m = oracle.deblock_picture(f)
    assert m == 0
    diff = out[0].astype(int) != f.planes[0].astype(int)
    assert diff.any()
    # every changed luma sample lies within 6 samples of a 4-aligned edge line
    ys, xs = np.nonzero(diff)
    assert np.all((np.minimum(xs % 4, 4 - xs % 4) <= 6) | (np.minimum(ys % 4, 4 - ys % 4) <= 6))
    # and the 14-tap reach bound holds against the transform map
    txw = np.array([4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64])
    assert txw[f.tx_luma].min() >= 4


def test_deblock_rejects_bad_parameters_and_samples():
    f = synth.make_small(23, 64, 64, 8)
    f.sharpness = 8
    _, m = oracle.deblock_picture(f)
    assert m == abi.MSG["DB_PARAMS"]
    f = synth.make_small(23, 64, 64, 8)
    f.tx_luma[3, 3] = 19
    _, m = oracle.deblock_picture(f)
    assert m == abi.MSG["DB_PARAMS"]
    f = synth.make_small(23, 64, 64, 8)
    f.planes[0][7, 9] = 256
    _, m = oracle.deblock_picture(f)
    assert m == abi.MSG["DB_SAMPLE"]


def test_synthetic_frames_are_deterministic():
    a = synth.make_small(5, 96, 64, 10)
    b = synth.make_small(5, 96, 64, 10)
    for x, y in zip(a.planes, b.planes):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.tx_luma, b.tx_luma)
    assert a.planes[0].max() <= 1023 and a.planes[0].dtype == np.uint16


def test_synthetic_side_information_is_in_range():
    f = synth.make_frame(synth.Workload("t", 640, 360, 8, 640, True), 1)
    assert f.tx_luma.max() <= 18 and f.tx_chroma.max() <= 18
    assert 0.1 < f.skip.mean() < 0.3
    for u in f.lr_units:
        assert set(np.unique(u["type"])) <= {0, 1, 2}
    assert all(0 <= v <= 63 for v in f.deblock_levels)
