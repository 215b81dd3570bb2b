"""Pipelined host entry points: vaco_av1_postfilter_frame_host_submit / _wait
keep up to three frames in flight (copies of one overlapping the filtering
of another).  Each frame's outputs must be the oracle's, bit-exact, and a
frame's error must come back from its own wait with the message the
synchronous call gives."""
import ctypes as C

import numpy as np
import pytest

import oracle
from vaco_b200 import abi, synth
from vaco_b200._lib import lib
from vaco_b200.frame import pinned_copy

pytestmark = pytest.mark.gpu

GEOMS = [(200, 136, 10, None), (328, 200, 10, 400), (64, 64, 8, None), (520, 264, 10, None), (96, 80, 12, None)]


def _submit(ctx, job):
    t, m = C.c_uint64(), C.c_int32()
    st = lib().vaco_av1_postfilter_frame_host_submit(ctx.handle, C.byref(job), C.byref(t), C.byref(m))
    return st, m.value, t.value


def _wait(ctx, ticket):
    m = C.c_int32()
    st = lib().vaco_av1_postfilter_frame_host_wait(ctx.handle, ticket, C.byref(m))
    return st, m.value


def test_pipelined_frames_match_oracle(ctx, oracle_threads):
    frames = [synth.make_small(70 + i, w, h, bd, upscaled_width=up) for i, (w, h, bd, up) in enumerate(GEOMS)]
    staged = [pinned_copy(f) for f in frames]
    tickets = []
    for i, (_, _, job) in enumerate(staged):
        if len(tickets) == 3:  # three in flight at most
            st, m = _wait(ctx, tickets.pop(0)[1])
            assert st == abi.OK, abi.MESSAGES.get(m)
        st, m, t = _submit(ctx, job)
        assert st == abi.OK, abi.MESSAGES.get(m)
        tickets.append((i, t))
    for _, t in tickets:
        st, m = _wait(ctx, t)
        assert st == abi.OK, abi.MESSAGES.get(m)
    for f, (_, outs, _) in zip(frames, staged):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        for g, x in zip(outs, want):
            assert np.array_equal(g, x)


def test_pipeline_reports_errors_per_frame_and_queue_limit(ctx, oracle_threads):
    from vaco_b200.gpu import VacoError

    good = [synth.make_small(80 + i, 200, 136, 10) for i in range(2)]
    bad = synth.make_small(82, 200, 136, 10)
    bad.planes[0][40, 33] = 1 << bad.bit_depth
    with pytest.raises(VacoError) as sync_err:
        ctx.postfilter_frame(bad)
    staged = [pinned_copy(f) for f in (good[0], bad, good[1])]
    tickets = []
    for _, _, job in staged:
        st, m, t = _submit(ctx, job)
        assert st == abi.OK
        tickets.append(t)
    # A fourth frame before any wait is refused.
    st, m, _ = _submit(ctx, staged[0][2])
    assert st == abi.LIMIT_EXCEEDED and m == abi.MSG["QUEUE_FULL"]
    results = [_wait(ctx, t) for t in tickets]
    assert results[0] == (abi.OK, 0) and results[2] == (abi.OK, 0)
    assert results[1] == (sync_err.value.status, sync_err.value.msg)
    for f, (_, outs, _) in ((good[0], staged[0]), (good[1], staged[2])):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        for g, x in zip(outs, want):
            assert np.array_equal(g, x)
    # A ticket is waited once.
    assert _wait(ctx, tickets[0])[0] == abi.INVALID_DATA
