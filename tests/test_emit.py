"""Frame emission: vaco's pic_to_frame / blit (src/decode.rs:3795-3891).

CPU tests pin the oracle's restatement to blit's rules: one byte per sample
at 8 bits with values above 255 becoming 0, little-endian u16 above 8 bits,
frame extents with chroma rounded up and cut to the source plane, row
padding untouched, and no pixel format for 8-bit 4:4:0.  GPU tests check the
three CUDA entry points against the oracle, bit-exact."""
import numpy as np
import pytest

import oracle
from vaco_b200 import abi, synth
from vaco_b200.frame import frame_buffer, frame_layout, picture_struct, ptr

FILL = 0xA5  # padding marker: emission must not touch it


def info_of(width, height, bd, ssx=1, ssy=1, mono=False):
    i = abi.FrameInfo()
    i.bit_depth, i.subsampling_x, i.subsampling_y, i.monochrome = bd, ssx, ssy, int(mono)
    i.upscaled_width, i.coded_width, i.coded_height = width, width, height
    i.mi_cols, i.mi_rows = 2 * ((width + 7) >> 3), 2 * ((height + 7) >> 3)
    return i


def planes_for(info, seed, shrink=0, hi=None):
    """Source planes of the frame's chroma-rounded-up extents (minus `shrink`
    columns and rows, to exercise the cut to the source plane)."""
    rng = np.random.default_rng(seed)
    hi = hi if hi is not None else (1 << info.bit_depth)
    out = []
    for k in range(1 if info.monochrome else 3):
        sx = info.subsampling_x if k else 0
        sy = info.subsampling_y if k else 0
        w = ((info.upscaled_width + (1 << sx) - 1) >> sx) - shrink
        h = ((info.coded_height + (1 << sy) - 1) >> sy) - shrink
        out.append(rng.integers(0, hi, (h, w)).astype(np.uint16))
    return out


def reference_pack(planes, info):
    """blit by hand, for the oracle's own check."""
    frame = frame_layout(info, FILL)
    for k, (p, b) in enumerate(zip(planes, frame)):
        h = min(p.shape[0], b.shape[0])
        sx = info.subsampling_x if k else 0
        w = min(p.shape[1], (info.upscaled_width + (1 << sx) - 1) >> sx)
        v = p[:h, :w]
        if info.bit_depth > 8:
            b[:h, : 2 * w] = v.astype("<u2").view(np.uint8).reshape(h, 2 * w)
        else:
            b[:h, :w] = np.where(v > 255, 0, v).astype(np.uint8)
    return frame


LAYOUTS = [  # (width, height, bit depth, ssx, ssy, mono)
    (200, 136, 8, 1, 1, False), (199, 135, 8, 1, 1, False), (130, 66, 10, 1, 1, False),
    (97, 41, 12, 1, 0, False), (64, 32, 10, 0, 0, False), (75, 33, 8, 0, 0, True),
    (121, 77, 10, 0, 1, False), (80, 40, 12, 0, 0, True),
]


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("shrink", [0, 3])
def test_oracle_emission_follows_blit(layout, shrink):
    w, h, bd, ssx, ssy, mono = layout
    info = info_of(w, h, bd, ssx, ssy, mono)
    planes = planes_for(info, seed=w + h + shrink, hi=1024 if bd == 8 else None)  # 8-bit: values above 255 too
    got, m = oracle.emit_frame(planes, info, frame_layout(info, FILL))
    assert m == 0
    want = reference_pack(planes, info)
    for g, x in zip(got, want):
        assert np.array_equal(g, x)


def test_oracle_rejects_8bit_440():
    info = info_of(64, 64, 8, 0, 1)
    _, m = oracle.emit_frame(planes_for(info, 1), info, frame_layout(info))
    assert m == abi.MSG["PIXEL_FORMAT"]


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("shrink", [0, 3])
def test_emit_host_matches_oracle(ctx, layout, shrink):
    w, h, bd, ssx, ssy, mono = layout
    info = info_of(w, h, bd, ssx, ssy, mono)
    planes = planes_for(info, seed=7 * w + h + shrink, hi=1024 if bd == 8 else None)
    want, m = oracle.emit_frame(planes, info, frame_layout(info, FILL))
    assert m == 0
    got = ctx.emit_frame(planes, info, fill=FILL)
    for g, x in zip(got, want):
        assert np.array_equal(g, x)


@pytest.mark.gpu
@pytest.mark.parametrize("pad", [0, 5])  # 5: rows not vector-aligned, the per-sample path
def test_emit_dev_matches_oracle(ctx, pad):
    import ctypes as C

    import torch

    from vaco_b200._lib import lib

    for (w, h, bd, ssx, ssy, mono) in [(3840, 2160, 10, 1, 1, False), (1920, 1080, 8, 1, 1, False),
                                       (199, 135, 8, 1, 1, False)]:
        info = info_of(w, h, bd, ssx, ssy, mono)
        planes = planes_for(info, seed=w, hi=1024 if bd == 8 else None)
        want, m = oracle.emit_frame(planes, info, frame_layout(info, FILL))
        assert m == 0
        dev_in = [torch.from_numpy(p.view(np.int16)).cuda() for p in planes]
        host_frame = frame_layout(info, FILL)
        dev_out = [torch.from_numpy(np.pad(b, ((0, 0), (0, pad)), constant_values=FILL)).cuda() for b in host_frame]
        pic = picture_struct([t.data_ptr() for t in dev_in], [p.shape for p in planes])
        fb = abi.FrameBuffer()
        for k, t in enumerate(dev_out):
            fb.planes[k] = t.data_ptr()
            fb.linesize[k] = t.shape[1]
        msg = C.c_int32()
        st = lib().vaco_av1_emit_frame_dev(ctx.handle, None, C.byref(pic), C.byref(info), C.byref(fb), C.byref(msg))
        assert st == abi.OK, abi.MESSAGES.get(msg.value)
        torch.cuda.synchronize()  # the device entry point only enqueues
        for t, x in zip(dev_out, want):
            assert np.array_equal(t.cpu().numpy()[:, : x.shape[1]], x)


@pytest.mark.gpu
def test_emit_rejects_8bit_440(ctx):
    from vaco_b200.gpu import VacoError

    info = info_of(64, 64, 8, 0, 1)
    with pytest.raises(VacoError) as e:
        ctx.emit_frame(planes_for(info, 1), info)
    assert e.value.status == abi.INVALID_DATA and e.value.msg == abi.MSG["PIXEL_FORMAT"]


@pytest.mark.gpu
@pytest.mark.parametrize("geom", [(200, 136, 8, None), (328, 200, 10, 400), (96, 80, 12, None)])
def test_postfilter_then_emit_matches_oracle(ctx, geom, oracle_threads):
    w, h, bd, up = geom
    f = synth.make_small(60 + w, w, h, bd, upscaled_width=up)
    filtered, m = oracle.postfilter_frame(f, threads=oracle_threads)
    assert m == 0
    want, m = oracle.emit_frame(filtered, f.info(), frame_layout(f.info(), FILL))
    assert m == 0
    got = ctx.postfilter_frame_emit(f, fill=FILL)
    for g, x in zip(got, want):
        assert np.array_equal(g, x)
