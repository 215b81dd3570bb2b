"""Frame-level parity: every CUDA entry point against the CPU oracle on the
same seeded inputs, bit-exact, from small odd geometries up to the full
benchmark sizes (4K 10-bit chain, 2880->3840 and 2560->3840 superres chains,
1080p 8-bit CDEF)."""
import numpy as np
import pytest

import oracle
from vaco_b200 import abi, synth
from vaco_b200.gpu import DeviceFrame, VacoError

pytestmark = pytest.mark.gpu

SMALL = [  # (width, height, bit_depth, upscaled_width)
    (64, 64, 8, None), (200, 136, 10, None), (96, 80, 12, None), (328, 200, 10, 400),
    (120, 72, 8, 136), (520, 264, 10, None),
    # coded sizes that are not multiples of 8 (the planes are mi-aligned,
    # the chain's outputs are cropped to the coded / upscaled size)
    (60, 44, 10, None), (204, 130, 8, None), (118, 70, 12, None), (100, 58, 10, 124),
]


def assert_planes_equal(got, want, what):
    assert len(got) == len(want)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g.shape == w.shape, (what, k)
        if not np.array_equal(g, w):
            ys, xs = np.nonzero(g != w)
            raise AssertionError(f"{what} plane {k}: {len(ys)} samples differ, first at y={ys[0]} x={xs[0]} "
                                 f"got {g[ys[0], xs[0]]} want {w[ys[0], xs[0]]}")


@pytest.mark.parametrize("geom", SMALL)
@pytest.mark.parametrize("seed", [1, 2])
def test_cdef_picture_small(ctx, geom, seed, oracle_threads):
    w, h, bd, _ = geom
    f = synth.make_small(seed, w, h, bd)
    want, m = oracle.cdef_picture(f, threads=oracle_threads)
    assert m == 0
    assert_planes_equal(ctx.cdef_picture(f), want, "cdef")


def test_cdef_picture_config0_full_size(ctx, oracle_threads):
    f = synth.make_frame(synth.CONFIG0, synth.seed_for(0, 0))
    want, m = oracle.cdef_picture(f, threads=oracle_threads)
    assert m == 0
    assert_planes_equal(ctx.cdef_picture(f), want, "cdef 1080p")


@pytest.mark.parametrize("geom", SMALL)
@pytest.mark.parametrize("sharp", [0, None])
def test_deblock_small(ctx, geom, sharp, oracle_threads):
    w, h, bd, _ = geom
    for seed, lvl_map in ((3, False), (4, True)):
        f = synth.make_small(seed, w, h, bd, sharpness=sharp, with_lvl_map=lvl_map)
        want, m = oracle.deblock_picture(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.deblock_picture(f), want, f"deblock seed={seed}")


TX_W = [4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64]
TX_H = [4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16]


def luma_edge_reach(tx_luma):
    """Luma samples a 7.14 deblocking pass may write: for every 4x4 cell on a
    transform edge (its x (y) a multiple of its transform's width (height)),
    the samples the edge's filter reaches, from the filter size min(16, both
    sides' transform extents): size 4 writes p1..q1, size 8 p2..q2, size 16
    p5..q5 (7.14.6)."""
    tw = np.array(TX_W)[tx_luma]
    th = np.array(TX_H)[tx_luma]
    rows, cols = tx_luma.shape
    reach = np.zeros((rows * 4, cols * 4), bool)
    span = {4: (2, 1), 8: (3, 2), 16: (6, 5)}
    for r in range(rows):
        for c in range(cols):
            x, y = 4 * c, 4 * r
            if c > 0 and x % tw[r, c] == 0:
                before, after = span[min(16, tw[r, c], tw[r, c - 1])]
                reach[y:y + 4, max(0, x - before):x + after + 1] = True
            if r > 0 and y % th[r, c] == 0:
                before, after = span[min(16, th[r, c], th[r - 1, c])]
                reach[max(0, y - before):y + after + 1, x:x + 4] = True
    return reach


def test_deblock_changes_samples_only_near_edges(ctx):
    f = synth.make_small(5, 256, 128, 10)
    out = ctx.deblock_picture(f)
    diff = out[0] != f.planes[0]
    assert diff.any()
    reach = luma_edge_reach(f.tx_luma)
    # Nothing farther from a transform edge than its filter reaches changes,
    # and a good part of the plane (transform interiors) is out of reach.
    ys, xs = np.nonzero(diff & ~reach)
    assert ys.size == 0, f"{ys.size} samples changed away from every edge, first at y={ys[0]} x={xs[0]}"
    assert (~reach).mean() > 0.2


def test_superres_plane_full_size(ctx, oracle_threads):
    f = synth.make_frame(synth.CONFIG2, synth.seed_for(2, 0))
    for k, (vis, out_w) in enumerate([(2880, 3840), (1440, 1920), (1440, 1920)]):
        p = f.planes[k]
        want, m = oracle.upscale_plane(p, vis, out_w, p.shape[0], 10, threads=oracle_threads)
        assert m == 0
        got = ctx.upscale_plane(p, vis, out_w, p.shape[0], 10)
        assert_planes_equal([got], [want], f"superres plane {k}")


@pytest.mark.parametrize("unit", [32, 64, 128, 256])
@pytest.mark.parametrize("sub_y", [False, True])
def test_restore_plane_synthetic(ctx, unit, sub_y, oracle_threads):
    rng = np.random.default_rng(unit * 2 + sub_y)
    for bd in (8, 10, 12):
        h, w = 150 + unit // 8, 230 + unit // 4
        before = rng.integers(0, 1 << bd, size=(h + 3, w + 5), dtype=np.uint16)
        after = np.clip(before.astype(np.int32) + rng.integers(-9, 10, size=before.shape), 0, (1 << bd) - 1).astype(np.uint16)
        units = synth.lr_units(rng, w, h, unit, sub_y)
        want, m = oracle.restore_plane(before, after, w, h, bd, unit, sub_y, units, threads=oracle_threads)
        assert m == 0
        got = ctx.restore_plane(before, after, w, h, bd, unit, sub_y, units)
        assert_planes_equal([got], [want], f"lr unit={unit} sub_y={sub_y} bd={bd}")


@pytest.mark.parametrize("geom", SMALL)
def test_postfilter_chain_small(ctx, geom, oracle_threads):
    w, h, bd, up = geom
    for seed in (7, 8):
        f = synth.make_small(seed, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=seed == 8)
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.postfilter_frame(f), want, f"chain seed={seed}")


LAYOUTS = [((1, 0), False), ((0, 0), False), ((1, 1), True)]
LAYOUT_IDS = ["422", "444", "mono"]


@pytest.mark.parametrize("layout", LAYOUTS, ids=LAYOUT_IDS)
@pytest.mark.parametrize("geom", [(200, 136, 10, None), (60, 44, 8, None), (100, 58, 12, 124), (520, 264, 10, None)])
def test_postfilter_chain_layouts(ctx, layout, geom, oracle_threads):
    """4:2:2, 4:4:4 and monochrome frames through the whole chain, through
    the host and the device entry points."""
    w, h, bd, up = geom
    sub, mono = layout
    for seed, lvl_map in ((21, False), (22, True)):
        f = synth.make_small(seed, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=lvl_map,
                             subsampling=sub, monochrome=mono)
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.postfilter_frame(f), want, f"chain {layout} seed={seed}")
        d = DeviceFrame(f)
        ctx.postfilter_frame_dev(d)
        assert_planes_equal(d.outputs_numpy(), want, f"chain dev {layout} seed={seed}")


@pytest.mark.parametrize("layout", LAYOUTS, ids=LAYOUT_IDS)
def test_cdef_and_deblock_layouts(ctx, layout, oracle_threads):
    """The standalone CDEF and deblocking entry points on the same layouts."""
    sub, mono = layout
    for seed, (w, h, bd) in enumerate([(200, 136, 10), (60, 44, 8), (96, 80, 12)]):
        f = synth.make_small(30 + seed, w, h, bd, sharpness=None, with_lvl_map=seed == 1, subsampling=sub,
                             monochrome=mono)
        want, m = oracle.cdef_picture(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.cdef_picture(f), want, f"cdef {layout}")
        want, m = oracle.deblock_picture(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.deblock_picture(f), want, f"deblock {layout}")


def test_postfilter_chain_444_1080p(ctx, oracle_threads):
    """A full-size 4:4:4 frame: every plane takes the 64x64 tile layout."""
    f = synth.make_frame(synth.Workload("chain_1080p_444", 1920, 1080, 10, 1920, True), synth.seed_for(9, 4),
                         subsampling=(0, 0))
    want, m = oracle.postfilter_frame(f, threads=oracle_threads)
    assert m == 0
    assert_planes_equal(ctx.postfilter_frame(f), want, "chain 1080p 4:4:4")


@pytest.mark.parametrize("workload", [synth.CONFIG1, synth.CONFIG2, synth.CONFIG2_DENOM12, synth.CONFIG0],
                         ids=lambda w: w.name)
def test_postfilter_chain_full_size(ctx, workload, oracle_threads):
    f = synth.make_frame(workload, synth.seed_for(9, 0))
    want, m = oracle.postfilter_frame(f, threads=oracle_threads)
    assert m == 0
    assert_planes_equal(ctx.postfilter_frame(f), want, workload.name)


def test_device_entry_matches_host_entry(ctx):
    f = synth.make_small(11, 328, 200, 10, upscaled_width=400)
    host = ctx.postfilter_frame(f)
    d = DeviceFrame(f)
    ctx.postfilter_frame_dev(d)
    assert_planes_equal(d.outputs_numpy(), host, "dev vs host")


# ---------------------------------------------------------------- error behaviour
def _expect_same_error(fn_gpu, oracle_msg):
    assert oracle_msg != 0
    with pytest.raises(VacoError) as e:
        fn_gpu()
    assert e.value.status == abi.INVALID_DATA
    assert e.value.msg == oracle_msg, (abi.MESSAGES[e.value.msg], abi.MESSAGES[oracle_msg])


def test_errors_match_oracle(ctx):
    # CDEF: a luma sample above the bit depth inside a filtered block
    f = synth.make_small(12, 128, 64, 8, chain=False)
    f.skip[:] = 0
    f.planes[0][10, 10] = 300
    _, m = oracle.cdef_picture(f)
    _expect_same_error(lambda: ctx.cdef_picture(f), m)
    # CDEF: strength index beyond the table
    f = synth.make_small(12, 128, 64, 8, chain=False)
    f.skip[:] = 0
    f.cdef_idx[0, 1] = 9
    _, m = oracle.cdef_picture(f)
    _expect_same_error(lambda: ctx.cdef_picture(f), m)
    # superres: sample out of range, bad geometry, bad depth
    p = np.full((4, 16), 5, np.uint16)
    p[2, 3] = 1024
    _, m = oracle.upscale_plane(p, 16, 20, 4, 10)
    _expect_same_error(lambda: ctx.upscale_plane(p, 16, 20, 4, 10), m)
    _, m = oracle.upscale_plane(p, 16, 16, 4, 10)
    _expect_same_error(lambda: ctx.upscale_plane(p, 16, 16, 4, 10), m)
    _, m = oracle.upscale_plane(p, 16, 20, 4, 9)
    _expect_same_error(lambda: ctx.upscale_plane(p, 16, 20, 4, 9), m)
    # restoration: tests/restoration.rs:96-140, 229-264
    plane = np.full((4, 4), 100, np.uint16)
    none = np.zeros(1, abi.lr_unit_dtype())
    for (w, h, bd, unit) in [(4, 4, 8, 0), (4, 4, 16, 64), (5, 4, 8, 64), (4, 0, 8, 64)]:
        _, m = oracle.restore_plane(plane, plane, w, h, bd, unit, False, none)
        _expect_same_error(lambda: ctx.restore_plane(plane, plane, w, h, bd, unit, False, none), m)
    import goldens
    for unit in [(2, 16, (0, 0, 0), (0, 0, 0), (0, 0)), (2, 0, (0, 0, 0), (0, 0, 0), (32, 0)),
                 (1, 0, (11, 0, 0), (0, 0, 0), (0, 0))]:
        u = goldens.lr_units_array([unit])
        _, m = oracle.restore_plane(plane, plane, 4, 4, 8, 64, False, u)
        _expect_same_error(lambda: ctx.restore_plane(plane, plane, 4, 4, 8, 64, False, u), m)
    empty = np.zeros(0, abi.lr_unit_dtype())
    _, m = oracle.restore_plane(plane, plane, 4, 4, 8, 64, False, empty)
    _expect_same_error(lambda: ctx.restore_plane(plane, plane, 4, 4, 8, 64, False, empty), m)
    before = np.full((12, 12), 16, np.uint16)
    after = np.full((12, 12), 235, np.uint16)
    after[8, 6] = 256
    _, m = oracle.restore_plane(before, after, 7, 9, 8, 64, False, none)
    _expect_same_error(lambda: ctx.restore_plane(before, after, 7, 9, 8, 64, False, none), m)
    # chain: a reconstruction sample above the bit depth fails in deblocking first
    f = synth.make_small(13, 200, 136, 10)
    f.planes[1][5, 5] = 2000
    _, m = oracle.postfilter_frame(f)
    _expect_same_error(lambda: ctx.postfilter_frame(f), m)


def test_restoration_none_preserves_visible_cdef_pixels(ctx):
    before = np.full((12, 12), 16, np.uint16)
    after = np.full((12, 12), 235, np.uint16)
    none = np.zeros(1, abi.lr_unit_dtype())
    out = ctx.restore_plane(before, after, 7, 9, 8, 64, False, none)
    assert out.shape == (9, 7) and (out == 235).all()


def _sr_picture(rng, coded_w, up_w, coded_h, ssx, ssy, mono, bd):
    """Mi-padded planes of a picture (8-aligned luma, as the decoder pads) and
    its superres::PictureConfig."""
    cfg = abi.SuperresPictureConfig(coded_w, up_w, coded_h, ssx, ssy, int(mono), bd)
    pw, ph = (coded_w + 7) // 8 * 8, (coded_h + 7) // 8 * 8
    planes = [rng.integers(0, 1 << bd, (ph, pw), dtype=np.uint16)]
    if not mono:
        planes += [rng.integers(0, 1 << bd, (ph >> ssy, pw >> ssx), dtype=np.uint16) for _ in range(2)]
    return planes, cfg


@pytest.mark.parametrize("layout", [(1, 1, False), (1, 0, False), (0, 0, False), (1, 1, True)],
                         ids=["420", "422", "444", "mono"])
@pytest.mark.parametrize("geom", [(2880, 3840, 2160, 10), (1439, 1918, 217, 8), (95, 120, 15, 12)],
                         ids=lambda g: f"{g[0]}to{g[1]}x{g[2]}_{g[3]}bit")
def test_upscale_picture_matches_oracle(ctx, layout, geom, oracle_threads):
    ssx, ssy, mono = layout
    coded_w, up_w, coded_h, bd = geom
    rng = np.random.default_rng(coded_w + 7 * ssx + 3 * ssy + int(mono))
    planes, cfg = _sr_picture(rng, coded_w, up_w, coded_h, ssx, ssy, mono, bd)
    want, m = oracle.upscale_picture(planes, cfg, threads=oracle_threads)
    assert m == 0
    got = ctx.upscale_picture(planes, cfg)
    assert_planes_equal(got, want, f"upscale_picture {layout} {geom}")
    # chroma geometry is the ceil division of the luma's (superres.rs:247-250)
    if not mono:
        assert got[1].shape == (-(-coded_h // (1 << ssy)), -(-up_w // (1 << ssx)))


def test_upscale_picture_errors_follow_plane_order(ctx):
    rng = np.random.default_rng(5)
    planes, cfg = _sr_picture(rng, 64, 80, 16, 1, 1, False, 10)
    # a missing U plane fails after luma succeeds
    _, m = oracle.upscale_picture([planes[0], None, planes[2]], cfg)
    assert m == abi.MSG["SR_MISSING_U"]
    _expect_same_error(lambda: ctx.upscale_picture([planes[0], None, planes[2]], cfg), m)
    _, m = oracle.upscale_picture([planes[0], planes[1], None], cfg)
    assert m == abi.MSG["SR_MISSING_V"]
    _expect_same_error(lambda: ctx.upscale_picture([planes[0], planes[1], None], cfg), m)
    # a luma sample above the bit depth comes before the missing plane
    bad = planes[0].copy()
    bad[3, 40] = 1024
    _, m = oracle.upscale_picture([bad, None, planes[2]], cfg)
    assert m == abi.MSG["SR_SAMPLE"]
    _expect_same_error(lambda: ctx.upscale_picture([bad, None, planes[2]], cfg), m)
    # a chroma sample error after a clean luma; a bad depth; a bad geometry
    badv = planes[2].copy()
    badv[2, 2] = 2000
    _, m = oracle.upscale_picture([planes[0], planes[1], badv], cfg)
    _expect_same_error(lambda: ctx.upscale_picture([planes[0], planes[1], badv], cfg), m)
    cfg9 = abi.SuperresPictureConfig(64, 80, 16, 1, 1, 0, 9)
    _, m = oracle.upscale_picture(planes, cfg9)
    _expect_same_error(lambda: ctx.upscale_picture(planes, cfg9), m)
    cfg_eq = abi.SuperresPictureConfig(64, 64, 16, 1, 1, 0, 10)
    _, m = oracle.upscale_picture(planes, cfg_eq)
    _expect_same_error(lambda: ctx.upscale_picture(planes, cfg_eq), m)


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_chain_extreme_samples(ctx, bd, oracle_threads):
    """Planes of 4x4 cells drawn from {0, max, max/2, 1, max-1} with small
    noise, at the highest loop-filter levels and every sharpness: the packed
    deblocking arithmetic (biased narrow filter, 16-bit halves) meets its
    extreme differences and saturating clamps."""
    rng = np.random.default_rng(900 + bd)
    maxv = (1 << bd) - 1
    for seed, sharp in enumerate(range(8)):
        f = synth.make_small(40 + seed, 200, 136, bd, sharpness=sharp, with_lvl_map=seed % 2 == 1)
        f.deblock_levels = (63, 63, 63, 63) if seed % 3 else (40, 63, 12, 50)
        for k, p in enumerate(f.planes):
            cells = rng.choice(np.array([0, maxv, maxv // 2, 1, maxv - 1]), size=((p.shape[0] + 3) // 4,
                                                                                  (p.shape[1] + 3) // 4))
            v = np.repeat(np.repeat(cells, 4, 0), 4, 1)[: p.shape[0], : p.shape[1]].astype(np.int64)
            v += rng.integers(-2, 3, size=v.shape)
            f.planes[k] = np.clip(v, 0, maxv).astype(np.uint16)
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        assert_planes_equal(ctx.postfilter_frame(f), want, f"extreme bd={bd} sharpness={sharp}")


@pytest.mark.parametrize("lr_off", [(0,), (1, 2), (0, 1, 2)], ids=["y", "uv", "all"])
@pytest.mark.parametrize("geom", [(200, 136, 10, None), (118, 70, 12, None), (60, 44, 8, None), (100, 58, 10, 124)])
def test_chain_planes_without_restoration(ctx, lr_off, geom, oracle_threads):
    """Planes whose restoration is off take the CDEF picture as their output
    (without superres the fused kernel writes it there directly), next to
    restored planes; odd visible widths end rows on a single sample."""
    w, h, bd, up = geom
    f = synth.make_small(60 + len(lr_off), w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=True)
    f.lr_type = tuple(abi.FRAME_LR_NONE if k in lr_off else t for k, t in enumerate(f.lr_type))
    want, m = oracle.postfilter_frame(f, threads=oracle_threads)
    assert m == 0
    assert_planes_equal(ctx.postfilter_frame(f), want, f"chain lr_off={lr_off}")
    d = DeviceFrame(f)
    ctx.postfilter_frame_dev(d)
    assert_planes_equal(d.outputs_numpy(), want, f"chain dev lr_off={lr_off}")
