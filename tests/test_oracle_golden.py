"""The CPU oracle against vaco's checked-in dav1d golden vectors.

Mirrors vaco's own golden tests: every CDEF case of
crates/tool/vaco-checkasm/tests/av1_cdef.rs:106-124, every superres record of
crates/codec/vaco-codec-av1/tests/superres.rs:37-84 and every restoration
sample of crates/codec/vaco-codec-av1/tests/restoration.rs:48-93,171-227.
"""
import numpy as np

import goldens
import oracle


def test_cdef_every_direction_strength_and_damping_matches_dav1d():
    inputs, params, exp_dir, exp_var, exp_out = goldens.cdef_cases()
    blocks = goldens.cdef_luma_blocks(inputs)
    for bd in (8, 10, 12):
        sel = params["bit_depth"] == bd
        (dirs, var), m = oracle.find_direction(blocks[sel], bd)
        assert m == 0
        np.testing.assert_array_equal(dirs, exp_dir[sel])
        np.testing.assert_array_equal(var, exp_var[sel])
    out, m = oracle.filter_block(inputs, params)
    assert m == 0
    np.testing.assert_array_equal(out, exp_out)


def test_cdef_oracle_exercises_all_directions_and_edge_masks():
    inputs, params, exp_dir, _, _ = goldens.cdef_cases()
    assert len(inputs) == 7680
    assert set(np.unique(exp_dir)) == set(range(8))
    assert set(np.unique(params["edges"])) == set(range(16))


def test_superres_matches_every_pinned_dav1d_case():
    for case in goldens.superres_cases():
        out, m = oracle.upscale_plane(case["input"], case["visible"], case["out"], case["height"],
                                      case["bd"])
        assert m == 0
        np.testing.assert_array_equal(out, case["expected"])


def test_restoration_dav1d_matches_all_pixels_across_depths_units_and_stripes():
    pixels = 0
    for c in goldens.lr_cases():
        out, m = oracle.restore_plane(c["before"], c["after"], c["width"], c["height"], c["bd"],
                                      c["unit_size"], c["sub_y"], c["units"])
        assert m == 0
        np.testing.assert_array_equal(out, c["expected"], err_msg=f"{c['bd']} {c['width']}x{c['height']} mode={c['mode']}")
        pixels += out.size
    assert pixels == 2_089_260


def test_restoration_constant_plane_rounding_matches_dav1d():
    for c in goldens.lr_constant_cases():
        out, m = oracle.restore_plane(c["plane"], c["plane"], 7, 9, c["bd"], 64, False, c["units"])
        assert m == 0
        np.testing.assert_array_equal(out, c["expected"])
    # Wiener identity at the maximum value (tests/restoration.rs:65-74)
    for bd in (8, 10, 12):
        plane = np.full((9, 7), (1 << bd) - 1, np.uint16)
        units = goldens.lr_units_array([(1, 0, (-5, -23, -17), (10, 8, 46), (0, 0))])
        out, m = oracle.restore_plane(plane, plane, 7, 9, bd, 64, False, units)
        assert m == 0
        np.testing.assert_array_equal(out, plane)
