"""The served form: continuous batching across streams.  Each frame's result
is the same alone and in a mix with many other streams' frames in flight
(bit-exact), admission refuses streams beyond the memory budget, and errors
stay with their own frame."""
import numpy as np
import pytest

import oracle
from vaco_b200 import abi, synth
from vaco_b200.serve import Server, frame_params

pytestmark = pytest.mark.gpu


def small_streams(seed0, count=6):
    geoms = [(200, 136, 10), (328, 200, 8), (520, 264, 12), (640, 360, 8), (1280, 720, 8), (96, 80, 10)]
    return [synth.make_small(seed0 + i, *geoms[i % len(geoms)], sharpness=None) for i in range(count)]


def test_frame_alone_equals_frame_in_mix():
    srv = Server(0, max_batch_frames=8, inflight_batches=2, memory_budget_bytes=2 << 30)
    try:
        frames = small_streams(600, 6)
        ids = []
        for f in frames:
            st, msg, sid = srv.open_stream(f, buffers=2)
            assert st == abi.OK
            srv.upload(sid, 0, f)
            srv.upload(sid, 1, f)
            ids.append(sid)
        # alone: one frame, nothing else in flight
        t = srv.submit(ids[0], 0, frame_params(frames[0]))
        st, msg, lat = srv.wait(t, 10_000)
        assert st == abi.OK and lat > 0
        alone = srv.download(ids[0], 0, frames[0])
        # in a mix: every stream submits both slots back to back, many rounds
        tickets = []
        for rnd in range(6):
            for sid, f in zip(ids, frames):
                tickets.append((sid, rnd % 2, srv.submit(sid, rnd % 2, frame_params(f))))
            for sid, slot, t in tickets[-len(ids):]:
                assert srv.wait(t, 30_000)[0] == abi.OK
        mix = srv.download(ids[0], 1, frames[0])
        want, m = oracle.postfilter_frame(frames[0])
        assert m == 0
        for a, b, w in zip(alone, mix, want):
            np.testing.assert_array_equal(a, w)
            np.testing.assert_array_equal(b, w)
        for sid, f in zip(ids[1:], frames[1:]):
            want, _ = oracle.postfilter_frame(f)
            for g, w in zip(srv.download(sid, 0, f), want):
                np.testing.assert_array_equal(g, w)
        assert srv.stats().max_batch >= 2  # frames were packed together
    finally:
        srv.close()


def test_admission_refuses_streams_beyond_budget():
    srv = Server(0, max_batch_frames=4, inflight_batches=1, memory_budget_bytes=64 << 20)
    try:
        f = synth.make_frame(synth.CONFIG1, 1)  # a 4K stream needs far more than 48 MiB of buffers
        st, msg, sid = srv.open_stream(f, buffers=4)
        assert st == abi.LIMIT_EXCEEDED and msg == abi.MSG["QUEUE_FULL"]
        small = synth.make_small(1, 64, 64, 8)
        st, msg, sid = srv.open_stream(small, buffers=2)
        assert st == abi.OK
    finally:
        srv.close()


def test_errors_stay_with_their_frame():
    srv = Server(0, max_batch_frames=8, inflight_batches=1, memory_budget_bytes=1 << 30)
    try:
        good, bad = synth.make_small(700, 200, 136, 10), synth.make_small(701, 200, 136, 10)
        bad.planes[0][4, 4] = 5000
        ids = []
        for f in (good, bad):
            st, _, sid = srv.open_stream(f, buffers=1)
            srv.upload(sid, 0, f)
            ids.append(sid)
        tg = srv.submit(ids[0], 0, frame_params(good))
        tb = srv.submit(ids[1], 0, frame_params(bad))
        assert srv.wait(tb, 10_000)[:2] == (abi.INVALID_DATA, abi.MSG["DB_SAMPLE"])
        assert srv.wait(tg, 10_000)[0] == abi.OK
    finally:
        srv.close()
