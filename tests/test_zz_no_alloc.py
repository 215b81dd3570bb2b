"""vaco_av1_postfilter_frame_noalloc: the whole chain for callers that cannot
call cudaMalloc.

Such a caller might be a decoder plugin whose host application owns all
device memory and forbids plugins from allocating, or a real-time path that
cannot afford an allocation's device-wide synchronization.  The entry point
keeps its intermediates in a fixed 16 MiB device array inside the library,
so it must give exactly the planes the oracle gives and the context-based
vaco_av1_postfilter_frame_dev gives, on consecutive calls that share the
array, and it must refuse exactly the frames whose intermediates do not fit
and the layouts the context entry point refuses.  This file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from vaco_b200 import abi, synth
from vaco_b200._lib import lib
from vaco_b200.gpu import Context, DeviceFrame, VacoError

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20


def scratch_bytes(f) -> int:
    """Bytes the entry point carves for frame `f`: the deblocked and the CDEF
    picture at the Mi-padded size per plane, plus with superres the upscaled
    CDEF picture and (when restoration runs) the upscaled pre-CDEF picture;
    each plane's pitch rounded up to 64 samples and its size to 256 bytes."""
    def plane(w, h):
        pitch = -(-max(w, 1) // 64) * 64
        return -(-(pitch * max(h, 1) * 2) // 256) * 256

    total = 0
    superres = f.upscaled_width != f.coded_width
    for k in range(f.num_planes):
        rows, cols = f.padded_shape(k)
        total += 2 * plane(cols, rows)
        if superres:
            sx, sy = f.plane_sub(k)
            w, h = (f.upscaled_width + sx) >> sx, (f.coded_height + sy) >> sy
            total += plane(w, h) * (2 if f.lr_active() else 1)
    return total


def _noalloc(dev: DeviceFrame):
    import torch

    m = C.c_int32(-1)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib().vaco_av1_postfilter_frame_noalloc(stream, C.byref(dev.job), C.byref(m))
    torch.cuda.synchronize()
    return st, m.value


def _fresh_device_frame(f):
    d = DeviceFrame(f)
    for o in d.outputs:
        o.fill_(-1)  # stale contents that a correct call overwrites
    return d


def _check_against_oracle_and_context(ctx, f, oracle_threads, what):
    want, m = oracle.postfilter_frame(f, threads=oracle_threads)
    assert m == 0
    ref = DeviceFrame(f)
    ctx.postfilter_frame_dev(ref)
    d = _fresh_device_frame(f)
    st, m = _noalloc(d)
    assert (st, m) == (abi.OK, 0), abi.MESSAGES.get(m)
    for k, (g, r, w) in enumerate(zip(d.outputs_numpy(), ref.outputs_numpy(), want)):
        assert np.array_equal(g, w), f"{what}: plane {k} differs from the oracle"
        assert np.array_equal(g, r), f"{what}: plane {k} differs from the context entry point"


# (width, height, bit depth, upscaled width): small superres, 720p, the
# documented 1920x1088 4:2:0 case, and 1280x720 with superres and restoration
GEOMS = [(328, 200, 10, 400), (1280, 720, 8, None), (1920, 1088, 10, None), (1024, 720, 10, 1280)]


@pytest.mark.parametrize("geom", GEOMS, ids=lambda g: "x".join(str(v) for v in g if v))
def test_noalloc_matches_oracle_and_context_on_two_calls_in_a_row(geom, oracle_threads):
    import torch

    torch.cuda.init()
    w, h, bd, up = geom
    ctx = Context(0)
    try:
        for seed in (31, 32):  # two calls in a row share the scratch array
            f = synth.make_small(seed, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=seed == 32)
            assert scratch_bytes(f) <= SCRATCH_BYTES
            _check_against_oracle_and_context(ctx, f, oracle_threads, f"{geom} seed {seed}")
    finally:
        ctx.close()


def test_noalloc_scratch_limit_edge(oracle_threads):
    """The tallest 1920-wide 4:2:0 frame that fits runs bit-exactly; one Mi
    row pair taller is refused with LIMIT_EXCEEDED before any work."""
    fit = synth.make_small(34, 1920, 1456, 10, sharpness=None)
    over = synth.make_small(35, 1920, 1464, 10, sharpness=None)
    assert scratch_bytes(fit) <= SCRATCH_BYTES < scratch_bytes(over)
    ctx = Context(0)
    try:
        _check_against_oracle_and_context(ctx, fit, oracle_threads, "1920x1456")
    finally:
        ctx.close()
    st, m = _noalloc(DeviceFrame(over))
    assert st == abi.LIMIT_EXCEEDED and m == abi.MSG["SCRATCH_LIMIT"]


def test_noalloc_superres_limit_edge():
    """With superres and restoration the upscaled pictures count too."""
    ok = synth.make_small(36, 1024, 720, 10, upscaled_width=1280)
    big = synth.make_small(37, 1440, 1080, 10, upscaled_width=1920)
    assert scratch_bytes(ok) <= SCRATCH_BYTES < scratch_bytes(big)
    st, m = _noalloc(DeviceFrame(big))
    assert st == abi.LIMIT_EXCEEDED and m == abi.MSG["SCRATCH_LIMIT"]
    st, m = _noalloc(DeviceFrame(ok))
    assert (st, m) == (abi.OK, 0)


def test_noalloc_rejects_frames_beyond_its_scratch():
    f = synth.make_frame(synth.CONFIG1, synth.seed_for(1, 0))  # 4K needs ~75 MB of intermediates
    d = DeviceFrame(f)
    st, m = _noalloc(d)
    assert st == abi.LIMIT_EXCEEDED and m == abi.MSG["SCRATCH_LIMIT"]


def _as_440(f):
    """The same frame relabelled 4:4:0 (full-width, half-height chroma), with
    planes and maps of the shapes that layout would have."""
    f.subsampling_x, f.subsampling_y = 0, 1
    rows, cols = f.padded_shape(1)
    f.planes = [f.planes[0]] + [np.full((rows, cols), 200, np.uint16) for _ in range(2)]
    f.tx_chroma = np.zeros(((f.mi_rows + 1) >> 1, f.mi_cols), np.uint8)
    f.lr_units = []
    f.lr_type = (abi.FRAME_LR_NONE,) * 3
    return f


def test_noalloc_refuses_440_like_the_context_entry_point():
    f = _as_440(synth.make_small(38, 200, 136, 10))
    st, m = _noalloc(DeviceFrame(f))
    assert st == abi.INVALID_DATA and m == abi.MSG["FRAME_GEOMETRY"]
    ctx = Context(0)
    try:
        with pytest.raises(VacoError) as e:
            ctx.postfilter_frame_dev(DeviceFrame(f))
        assert e.value.status == abi.INVALID_DATA and e.value.msg == abi.MSG["FRAME_GEOMETRY"]
    finally:
        ctx.close()


def test_noalloc_reports_data_errors_like_the_context_entry_point():
    f = synth.make_small(33, 200, 136, 10)
    f.planes[0][9, 9] = 4000  # above 10-bit
    st, m = _noalloc(DeviceFrame(f))
    assert st == abi.INVALID_DATA and m == abi.MSG["DB_SAMPLE"]
