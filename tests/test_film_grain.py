"""Film grain synthesis (AV1 7.18.3): vaco parses film_grain_params()
(src/frame_header.rs:1125-1210) and has no synthesis, so no vaco code or
golden vector pins this part.  CPU tests check the C++ oracle against an
independent pure-Python restatement (tests/film_grain_ref.py) on small
frames, and the entry points' rules (no grain, parameter and sample
errors).  GPU tests check both CUDA entry points against the oracle,
bit-exact, from small odd frames to 4K."""
import ctypes as C

import numpy as np
import pytest

import oracle
from film_grain_ref import film_grain as py_film_grain
from vaco_b200 import abi

FORMATS = {"420": (1, 1, False), "444": (0, 0, False), "422": (1, 0, False), "mono": (1, 1, True)}


def gauss_table(seed=7):
    """A synthetic stand-in for the spec's Gaussian_Sequence (the caller
    supplies the normative table): 2048 values in its 12-bit range."""
    return np.random.default_rng(seed).integers(-2048, 2048, 2048).astype(np.int16)


def random_params(seed, mono=False, **over):
    rng = np.random.default_rng(seed)
    over = dict(over)  # the cases' dicts are shared between tests
    p = abi.FilmGrainParams()
    p.apply_grain = 1
    p.grain_seed = int(rng.integers(0, 1 << 16))

    def pts(arr_v, arr_s, n):
        vals = np.sort(rng.choice(256, size=n, replace=False))
        for i in range(n):
            arr_v[i] = int(vals[i])
            arr_s[i] = int(rng.integers(0, 256))
        return n

    n_y = int(rng.integers(0, 15))
    p.num_y_points = pts(p.point_y_value, p.point_y_scaling, over.pop("num_y_points", n_y))
    p.chroma_scaling_from_luma = 0 if mono else int(rng.integers(0, 2))
    if not mono and not p.chroma_scaling_from_luma:
        p.num_cb_points = pts(p.point_cb_value, p.point_cb_scaling, int(rng.integers(0, 11)))
        p.num_cr_points = pts(p.point_cr_value, p.point_cr_scaling, int(rng.integers(0, 11)))
    p.grain_scaling_minus_8 = int(rng.integers(0, 4))
    p.ar_coeff_lag = int(rng.integers(0, 4))
    for arr, n in ((p.ar_coeffs_y_plus_128, 24), (p.ar_coeffs_cb_plus_128, 25), (p.ar_coeffs_cr_plus_128, 25)):
        for i in range(n):
            arr[i] = int(np.clip(128 + rng.normal(0, 20), 0, 255))
    p.ar_coeff_shift_minus_6 = int(rng.integers(0, 4))
    p.grain_scale_shift = int(rng.integers(0, 4))
    p.cb_mult, p.cb_luma_mult, p.cb_offset = (int(v) for v in rng.integers(0, [256, 256, 512]))
    p.cr_mult, p.cr_luma_mult, p.cr_offset = (int(v) for v in rng.integers(0, [256, 256, 512]))
    p.overlap_flag = int(rng.integers(0, 2))
    p.clip_to_restricted_range = int(rng.integers(0, 2))
    p.mc_identity = int(rng.integers(0, 2))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def frame(seed, w, h, bd, fmt):
    sx, sy, mono = FORMATS[fmt]
    info = abi.FrameInfo()
    info.bit_depth, info.subsampling_x, info.subsampling_y, info.monochrome = bd, sx, sy, int(mono)
    info.upscaled_width, info.coded_width, info.coded_height = w, w, h
    info.mi_cols, info.mi_rows = 2 * ((w + 7) >> 3), 2 * ((h + 7) >> 3)
    rng = np.random.default_rng(seed)
    shapes = [(h, w)] + ([] if mono else [((h + sy) >> sy, (w + sx) >> sx)] * 2)
    planes = [rng.integers(0, 1 << bd, s).astype(np.uint16) for s in shapes]
    return info, planes


# (seed, w, h, bit depth, format, overrides)
SMALL = [
    (1, 70, 45, 8, "420", {}), (2, 70, 45, 10, "420", {"overlap_flag": 1, "ar_coeff_lag": 3}),
    (3, 67, 37, 12, "444", {"overlap_flag": 1}), (4, 70, 45, 10, "422", {"overlap_flag": 1, "ar_coeff_lag": 2}),
    (5, 53, 41, 10, "mono", {"overlap_flag": 1}), (6, 70, 45, 8, "420", {"chroma_scaling_from_luma": 1}),
    (7, 66, 34, 10, "420", {"clip_to_restricted_range": 1, "overlap_flag": 1}),
    (8, 35, 33, 12, "420", {"num_y_points": 0, "ar_coeff_lag": 1}),
]


@pytest.mark.parametrize("case", SMALL, ids=[f"{c[4]}-{c[3]}bit-{c[0]}" for c in SMALL])
def test_oracle_matches_python_restatement(case):
    seed, w, h, bd, fmt, over = case
    info, planes = frame(seed, w, h, bd, fmt)
    p = random_params(100 + seed, mono=FORMATS[fmt][2], **over)
    g = gauss_table(seed)
    got, m = oracle.film_grain(planes, info, p, g)
    assert m == 0
    sx, sy, mono = FORMATS[fmt]
    want = py_film_grain(planes, bd, sx, sy, mono, p, [int(v) for v in g])
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"plane {k}: {int((a != b).sum())} samples differ"


@pytest.mark.parametrize("seed", range(300, 316))
def test_oracle_matches_python_restatement_random(seed):
    """Sixteen more random cases: format, depth, size and every parameter
    drawn from the seed."""
    rng = np.random.default_rng(seed)
    fmt = ["420", "444", "422", "mono"][seed % 4]
    bd = [8, 10, 12][int(rng.integers(0, 3))]
    w, h = int(rng.integers(17, 90)), int(rng.integers(17, 70))
    info, planes = frame(seed, w, h, bd, fmt)
    p = random_params(seed, mono=FORMATS[fmt][2])
    g = gauss_table(seed)
    got, m = oracle.film_grain(planes, info, p, g)
    assert m == 0
    sx, sy, mono = FORMATS[fmt]
    want = py_film_grain(planes, bd, sx, sy, mono, p, [int(v) for v in g])
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"plane {k}: {int((a != b).sum())} samples differ"


def test_oracle_no_grain_is_a_copy_and_grain_changes_samples():
    info, planes = frame(11, 70, 45, 10, "420")
    p = random_params(11, num_y_points=2)
    p.point_y_value[0], p.point_y_value[1], p.point_y_scaling[0], p.point_y_scaling[1] = 0, 255, 200, 200
    out, m = oracle.film_grain(planes, info, p, gauss_table())
    assert m == 0 and not np.array_equal(out[0], planes[0])
    p.apply_grain = 0
    out, m = oracle.film_grain(planes, info, p, gauss_table())
    assert m == 0 and all(np.array_equal(a, b) for a, b in zip(out, planes))


def test_oracle_rejects_bad_parameters_and_samples():
    info, planes = frame(12, 40, 40, 10, "420")
    p = random_params(12, num_y_points=2)
    p.point_y_value[0], p.point_y_value[1] = 50, 50  # not increasing
    assert oracle.film_grain(planes, info, p, gauss_table())[1] == abi.MSG["FG_PARAMS"]
    p = random_params(12, ar_coeff_lag=4)
    assert oracle.film_grain(planes, info, p, gauss_table())[1] == abi.MSG["FG_PARAMS"]
    p = random_params(12)
    planes[1][3, 4] = 1 << 10
    assert oracle.film_grain(planes, info, p, gauss_table())[1] == abi.MSG["FG_SAMPLE"]


# ---------------------------------------------------------------- GPU
GPU_CASES = SMALL + [
    (21, 1920, 1080, 10, "420", {"overlap_flag": 1, "ar_coeff_lag": 3}),
    (22, 3840, 2160, 10, "420", {"overlap_flag": 1, "ar_coeff_lag": 3, "num_y_points": 8}),
    (23, 1279, 719, 8, "444", {"overlap_flag": 1}),
    (24, 641, 359, 12, "422", {"overlap_flag": 0, "clip_to_restricted_range": 1}),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES, ids=[f"{c[4]}-{c[1]}x{c[2]}-{c[3]}bit" for c in GPU_CASES])
def test_film_grain_host_matches_oracle(ctx, case):
    seed, w, h, bd, fmt, over = case
    info, planes = frame(seed, w, h, bd, fmt)
    p = random_params(200 + seed, mono=FORMATS[fmt][2], **over)
    g = gauss_table(seed)
    want, m = oracle.film_grain(planes, info, p, g)
    assert m == 0
    got = ctx.film_grain(planes, info, p, g)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"plane {k}: {int((a != b).sum())} samples differ"


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(300, 316))
def test_film_grain_host_matches_oracle_random(ctx, seed):
    rng = np.random.default_rng(seed)
    fmt = ["420", "444", "422", "mono"][seed % 4]
    bd = [8, 10, 12][int(rng.integers(0, 3))]
    w, h = int(rng.integers(17, 90)), int(rng.integers(17, 70))
    info, planes = frame(seed, w, h, bd, fmt)
    p = random_params(seed, mono=FORMATS[fmt][2])
    g = gauss_table(seed)
    want, m = oracle.film_grain(planes, info, p, g)
    assert m == 0
    got = ctx.film_grain(planes, info, p, g)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"plane {k}: {int((a != b).sum())} samples differ"


@pytest.mark.gpu
def test_film_grain_dev_matches_oracle_twice(ctx):
    import torch

    from vaco_b200._lib import lib
    from vaco_b200.frame import picture_struct

    for seed in (31, 32):  # two calls in a row through the same workspace
        info, planes = frame(seed, 1920, 1080, 10, "420")
        p = random_params(seed, overlap_flag=1)
        g = gauss_table(seed)
        want, m = oracle.film_grain(planes, info, p, g)
        assert m == 0
        din = [torch.from_numpy(q.view(np.int16)).cuda() for q in planes]
        dout = [torch.empty_like(t) for t in din]
        pin = picture_struct([t.data_ptr() for t in din], [q.shape for q in planes])
        pout = picture_struct([t.data_ptr() for t in dout], [q.shape for q in planes])
        msg = C.c_int32()
        st = lib().vaco_av1_film_grain_dev(ctx.handle, None, C.byref(pin), C.byref(pout), C.byref(info), C.byref(p),
                                           g.ctypes.data, C.byref(msg))
        assert st == abi.OK, abi.MESSAGES.get(msg.value)
        for t, x in zip(dout, want):
            assert np.array_equal(t.cpu().numpy().view(np.uint16), x)


@pytest.mark.gpu
def test_film_grain_errors_match_oracle(ctx):
    from vaco_b200.gpu import VacoError

    info, planes = frame(41, 200, 120, 10, "420")
    p = random_params(41)
    planes[0][70, 150] = 1 << 10
    assert oracle.film_grain(planes, info, p, gauss_table())[1] == abi.MSG["FG_SAMPLE"]
    with pytest.raises(VacoError) as e:
        ctx.film_grain(planes, info, p, gauss_table())
    assert e.value.status == abi.INVALID_DATA and e.value.msg == abi.MSG["FG_SAMPLE"]
    planes[0][70, 150] = 0
    p = random_params(41, grain_scale_shift=4)
    with pytest.raises(VacoError) as e:
        ctx.film_grain(planes, info, p, gauss_table())
    assert e.value.msg == abi.MSG["FG_PARAMS"]
    # the context is still usable
    p = random_params(42)
    want, _ = oracle.film_grain(planes, info, p, gauss_table())
    got = ctx.film_grain(planes, info, p, gauss_table())
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


@pytest.mark.gpu
def test_film_grain_dev_deferred():
    """Under deferred status the device entry point only enqueues; outputs of
    back-to-back calls are the oracle's, and a sample error surfaces at the
    flush."""
    import torch

    from vaco_b200._lib import lib
    from vaco_b200.frame import picture_struct
    from vaco_b200.gpu import Context, VacoError

    c = Context(0)
    c.set_deferred_status(True)
    try:
        runs = []
        for seed in (51, 52, 53):
            info, planes = frame(seed, 640, 360, 10, "420")
            if seed == 52:
                planes[2][10, 20] = 1 << 10  # above the bit depth
            p = random_params(seed, overlap_flag=1)
            g = gauss_table(seed)
            din = [torch.from_numpy(q.view(np.int16)).cuda() for q in planes]
            dout = [torch.empty_like(t) for t in din]
            pin = picture_struct([t.data_ptr() for t in din], [q.shape for q in planes])
            pout = picture_struct([t.data_ptr() for t in dout], [q.shape for q in planes])
            msg = C.c_int32()
            st = lib().vaco_av1_film_grain_dev(c.handle, None, C.byref(pin), C.byref(pout), C.byref(info),
                                               C.byref(p), g.ctypes.data, C.byref(msg))
            assert st == abi.OK
            runs.append((info, planes, p, g, dout, din))
        with pytest.raises(VacoError) as e:
            c.flush()
        assert e.value.msg == abi.MSG["FG_SAMPLE"]
        for info, planes, p, g, dout, _ in (runs[0], runs[2]):
            want, m = oracle.film_grain(planes, info, p, g)
            assert m == 0
            for t, x in zip(dout, want):
                assert np.array_equal(t.cpu().numpy().view(np.uint16), x)
        c.flush()
    finally:
        c.set_deferred_status(False)
        c.close()


@pytest.mark.gpu
def test_film_grain_many_frames_in_flight():
    """Twelve frames back to back under deferred status: more frames than
    the context has workspace sets, so each set is reused while other frames'
    templates and grain are still queued.  Every frame must match the oracle."""
    import torch

    from vaco_b200._lib import lib
    from vaco_b200.frame import picture_struct
    from vaco_b200.gpu import Context

    c = Context(0)
    c.set_deferred_status(True)
    try:
        runs = []
        for seed in range(60, 72):
            fmt = ("420", "444", "422")[seed % 3]
            info, planes = frame(seed, 96 + seed, 64 + seed % 7, (8, 10, 12)[seed % 3], fmt)
            p = random_params(seed, overlap_flag=seed % 2, ar_coeff_lag=seed % 4)
            g = gauss_table(seed)
            din = [torch.from_numpy(q.view(np.int16)).cuda() for q in planes]
            dout = [torch.empty_like(t) for t in din]
            pin = picture_struct([t.data_ptr() for t in din], [q.shape for q in planes])
            pout = picture_struct([t.data_ptr() for t in dout], [q.shape for q in planes])
            msg = C.c_int32()
            st = lib().vaco_av1_film_grain_dev(c.handle, None, C.byref(pin), C.byref(pout), C.byref(info),
                                               C.byref(p), g.ctypes.data, C.byref(msg))
            assert st == abi.OK, abi.MESSAGES.get(msg.value)
            runs.append((info, planes, p, g, dout, din))
        c.flush()
        for info, planes, p, g, dout, _ in runs:
            want, m = oracle.film_grain(planes, info, p, g)
            assert m == 0
            for t, x in zip(dout, want):
                assert np.array_equal(t.cpu().numpy().view(np.uint16), x)
    finally:
        c.set_deferred_status(False)
        c.close()
