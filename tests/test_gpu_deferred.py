"""Deferred status: vaco_av1_postfilter_frame_dev enqueues the chain without a
host round trip per frame, and vaco_av1_ctx_flush reports the earliest
device-side error of the frames since the previous flush.  The outputs must
be the oracle's, bit-exact, and an error must carry the message the
synchronous call gives for the same frame."""
import numpy as np
import pytest

import oracle
from vaco_b200 import synth
from vaco_b200.gpu import Context, DeviceFrame, VacoError

pytestmark = pytest.mark.gpu

GEOMS = [(200, 136, 10, None), (328, 200, 10, 400), (64, 64, 8, None), (520, 264, 10, None)]


def _same(got, want, what):
    for k, (g, w) in enumerate(zip(got, want)):
        assert g.shape == w.shape, (what, k)
        assert np.array_equal(g, w), f"{what} plane {k}: {int((g != w).sum())} samples differ"


@pytest.fixture
def deferred_ctx():
    c = Context(0)  # its own context: the session one stays synchronous
    c.set_deferred_status(True)
    yield c
    c.set_deferred_status(False)
    c.close()


def test_deferred_frames_match_oracle(deferred_ctx, oracle_threads):
    frames = [synth.make_small(40 + i, w, h, bd, upscaled_width=up) for i, (w, h, bd, up) in enumerate(GEOMS)]
    devs = [DeviceFrame(f) for f in frames]
    for _ in range(2):  # the same frames twice in a row, one flush at the end
        for d in devs:
            deferred_ctx.postfilter_frame_dev(d)
    deferred_ctx.flush()
    for i, (f, d) in enumerate(zip(frames, devs)):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        _same(d.outputs_numpy(), want, f"frame {i}")


def test_deferred_error_is_reported_at_flush(ctx, deferred_ctx, oracle_threads):
    good = [synth.make_small(50 + i, 200, 136, 10) for i in range(2)]
    bad = synth.make_small(52, 200, 136, 10)
    bad.planes[0][40, 33] = 1 << bad.bit_depth  # one luma sample above the bit depth
    # The synchronous call names the error at once.
    with pytest.raises(VacoError) as sync_err:
        ctx.postfilter_frame_dev(DeviceFrame(bad))
    _, m = oracle.postfilter_frame(bad, threads=oracle_threads)
    assert sync_err.value.msg == m
    # Deferred: every call returns; the flush names the same error.
    devs = [DeviceFrame(good[0]), DeviceFrame(bad), DeviceFrame(good[1])]
    for d in devs:
        deferred_ctx.postfilter_frame_dev(d)
    with pytest.raises(VacoError) as flush_err:
        deferred_ctx.flush()
    assert flush_err.value.status == sync_err.value.status
    assert flush_err.value.msg == sync_err.value.msg
    # The good frames around it are filtered correctly, and the word is clear again.
    for f, d in ((good[0], devs[0]), (good[1], devs[2])):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        _same(d.outputs_numpy(), want, "good frame")
    deferred_ctx.flush()
