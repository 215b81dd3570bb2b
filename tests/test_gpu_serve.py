"""The served form: continuous batching across streams.  Each frame's result
is the same alone and in a mix with many other streams' frames in flight
(bit-exact), admission refuses streams beyond the memory budget, and errors
stay with their own frame."""
import ctypes as C

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


def test_config4_streams_alone_equal_mix_with_1080p_and_4k():
    """The config-4 resolutions (640x360 and 1280x720 8-bit, 1920x1080 and
    3840x2160 10-bit) in one mix: each stream's frame is the oracle's alone
    and in the mix, whether its input was resident or uploaded with it."""
    from vaco_b200.frame import host_job

    srv = Server(0, max_batch_frames=16, inflight_batches=3, memory_budget_bytes=8 << 30)
    try:
        frames = [synth.make_frame(wl, synth.seed_for(4, 8800 + i)) for i, (wl, _) in enumerate(synth.BATCH_MIX)]
        frames += [synth.make_frame(synth.BATCH_MIX[3][0], synth.seed_for(4, 8810)),
                   synth.make_frame(synth.BATCH_MIX[2][0], synth.seed_for(4, 8811))]
        ids = []
        for f in frames:
            st, msg, sid = srv.open_stream(f, buffers=2)
            assert st == abi.OK, abi.MESSAGES.get(msg)
            srv.upload(sid, 0, f)
            ids.append(sid)
        wants = []
        for f in frames:
            w, m = oracle.postfilter_frame(f, threads=32)
            assert m == 0
            wants.append(w)
        # alone: the 4K stream's frame with nothing else in flight
        t = srv.submit(ids[3], 0, frame_params(frames[3]))
        assert srv.wait(t, 30_000)[0] == abi.OK
        for g, w in zip(srv.download(ids[3], 0, frames[3]), wants[3]):
            np.testing.assert_array_equal(g, w)
        # mix: slot 0 resident, slot 1 uploaded inside submit_host, all streams at once, three rounds
        host_jobs = [host_job(f, [np.zeros((1, 1), np.uint16)] * f.num_planes) for f in frames]
        for rnd in range(3):
            tickets = []
            for sid, f, hj in zip(ids, frames, host_jobs):
                tickets.append(srv.submit(sid, 0, frame_params(f)))
                tickets.append(srv.submit_host(sid, 1, hj))
            for t in tickets:
                st, msg, lat = srv.wait(t, 60_000)
                assert st == abi.OK, abi.MESSAGES.get(msg)
        for sid, f, w in zip(ids, frames, wants):
            for slot in (0, 1):
                for g, ww in zip(srv.download(sid, slot, f), w):
                    np.testing.assert_array_equal(g, ww)
        # every stream's resident slot at once: frames that queue while the
        # launch slots are busy are packed into one launch set
        n = len(ids)
        tickets = (C.c_uint64 * n)()
        params = (abi.FrameJob * n)(*[frame_params(f) for f in frames])
        assert srv.l.vaco_av1_server_submit_many(srv.h, n, (C.c_int32 * n)(*ids), (C.c_int32 * n)(*[0] * n),
                                                  params, tickets) == abi.OK
        assert srv.l.vaco_av1_server_wait_many(srv.h, n, tickets, 60_000, None, None, None) == abi.OK
        for sid, f, w in zip(ids, frames, wants):
            for g, ww in zip(srv.download(sid, 0, f), w):
                np.testing.assert_array_equal(g, ww)
        assert srv.stats().max_batch >= 2
    finally:
        srv.close()


def _busy_server_streams(srv, n_streams=4, buffers=4):
    f = synth.make_frame(synth.CONFIG1, synth.seed_for(4, 8900))
    ids = []
    for _ in range(n_streams):
        st, _, sid = srv.open_stream(f, buffers=buffers)
        assert st == abi.OK
        for b in range(buffers):
            srv.upload(sid, b, f)
        ids.append(sid)
    return f, ids


def test_wait_with_zero_timeout_reports_timeout_then_collects():
    srv = Server(0, max_batch_frames=8, inflight_batches=2, memory_budget_bytes=8 << 30)
    try:
        f, ids = _busy_server_streams(srv)
        tickets = [srv.submit(sid, b, frame_params(f)) for sid in ids for b in range(4)]
        st, msg, _ = srv.wait(tickets[-1], 0)  # 16 4K frames queued: the last cannot be done yet
        assert st == abi.TIMEOUT and msg == abi.MSG["TIMEOUT"]
        for t in tickets:  # every ticket, the timed-out one included, is collected later
            assert srv.wait(t, 60_000)[0] == abi.OK
    finally:
        srv.close()


def test_close_stream_waits_for_frames_in_flight():
    srv = Server(0, max_batch_frames=8, inflight_batches=2, memory_budget_bytes=8 << 30)
    try:
        f, ids = _busy_server_streams(srv)
        resident = srv.stats().resident_bytes
        tickets = [srv.submit(sid, b, frame_params(f)) for sid in ids for b in range(4)]
        assert srv.close_stream(ids[-1]) == abi.OK  # returns once its frames are done
        for t in tickets:
            assert srv.wait(t, 60_000)[0] == abi.OK
        assert srv.stats().resident_bytes * 4 == resident * 3  # one of four equal streams is gone
    finally:
        srv.close()


def test_close_stream_and_backpressure_time_out_with_a_tiny_bound():
    """With a 1 ms bound on the host waits, closing a stream whose frames sit
    behind a queue of 4K frames, and re-submitting a slot still in flight,
    both return TIMEOUT; the frames still complete and the close then works."""
    # one frame per launch set, one set in flight: 24 4K frames run one after
    # another (several ms), and the last stream's are at the back
    srv = Server(0, max_batch_frames=1, inflight_batches=1, memory_budget_bytes=8 << 30, host_wait_ms=1)
    try:
        f, ids = _busy_server_streams(srv, n_streams=6)
        tickets = [srv.submit(sid, b, frame_params(f)) for sid in ids for b in range(4)]
        assert srv.close_stream(ids[-1]) == abi.TIMEOUT
        st, _ = srv.try_submit(ids[-1], 3, frame_params(f))
        assert st == abi.TIMEOUT
        for t in tickets:
            assert srv.wait(t, 60_000)[0] == abi.OK
        assert srv.close_stream(ids[-1]) == abi.OK
        want, m = oracle.postfilter_frame(f, threads=32)
        assert m == 0
        for g, w in zip(srv.download(ids[0], 3, f), want):
            np.testing.assert_array_equal(g, w)
    finally:
        srv.close()
