"""The CUDA library against vaco's dav1d golden vectors, through the C ABI.

Same cases as tests/test_oracle_golden.py (vaco's own golden tests), but the
outputs come from the sm_100a kernels."""
import numpy as np
import pytest

import goldens

pytestmark = pytest.mark.gpu


def test_cdef_find_direction_and_filter_block_match_dav1d(ctx):
    inputs, params, exp_dir, exp_var, exp_out = goldens.cdef_cases()
    blocks = goldens.cdef_luma_blocks(inputs)
    for bd in (8, 10, 12):
        sel = params["bit_depth"] == bd
        dirs, var = ctx.find_direction(blocks[sel], bd)
        np.testing.assert_array_equal(dirs, exp_dir[sel])
        np.testing.assert_array_equal(var, exp_var[sel])
    out = ctx.filter_block(inputs, params)
    np.testing.assert_array_equal(out, exp_out)


def test_superres_matches_every_dav1d_record(ctx):
    for case in goldens.superres_cases():
        out = ctx.upscale_plane(case["input"], case["visible"], case["out"], case["height"], case["bd"])
        np.testing.assert_array_equal(out, case["expected"])


def test_restoration_matches_all_2089260_dav1d_samples(ctx):
    pixels = 0
    for c in goldens.lr_cases():
        out = ctx.restore_plane(c["before"], c["after"], c["width"], c["height"], c["bd"], c["unit_size"],
                                c["sub_y"], c["units"])
        np.testing.assert_array_equal(out, c["expected"],
                                      err_msg=f"{c['bd']} {c['width']}x{c['height']} mode={c['mode']}")
        pixels += out.size
    assert pixels == 2_089_260


def test_restoration_constant_planes_match_dav1d(ctx):
    for c in goldens.lr_constant_cases():
        out = ctx.restore_plane(c["plane"], c["plane"], 7, 9, c["bd"], 64, False, c["units"])
        np.testing.assert_array_equal(out, c["expected"])
    for bd in (8, 10, 12):
        plane = np.full((9, 7), (1 << bd) - 1, np.uint16)
        units = goldens.lr_units_array([(1, 0, (-5, -23, -17), (10, 8, 46), (0, 0))])
        np.testing.assert_array_equal(ctx.restore_plane(plane, plane, 7, 9, bd, 64, False, units), plane)
