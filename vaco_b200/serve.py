"""Served form: Python handle on the library's request server, and the
serving benchmark (32 streams, Poisson arrivals at 1x / 2x / 4x real time).

The server itself is native (vaco_b200/csrc/server.cu): a worker thread packs
pending frames into batched launch sets as launch slots free up.  This module
only opens streams, uploads frames into their device-resident slots, submits
with Poisson timing and collects per-frame latencies.
"""
from __future__ import annotations

import ctypes as C
import json
import random
import statistics
import threading
import time
from collections import deque
from typing import List, Optional

import numpy as np

from . import abi, synth
from ._lib import lib
from .frame import FrameInputs, host_job, picture_struct, pinned_copy, ptr


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_batch_frames", C.c_int32),
        ("inflight_batches", C.c_int32),
        ("host_wait_ms", C.c_int32),
        ("memory_budget_bytes", C.c_int64),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("batches", C.c_uint64),
        ("max_batch", C.c_uint64),
        ("resident_bytes", C.c_int64),
        ("scratch_bytes", C.c_int64),
    ]


def _declare():
    """The library handle; the server entry points are declared in _lib."""
    return lib()


class Server:
    """Handle on vaco_av1_server."""

    def __init__(self, device=0, max_batch_frames=64, inflight_batches=3, memory_budget_bytes=40 << 30,
                 host_wait_ms=0):
        self.l = _declare()
        cfg = ServerConfig(device, max_batch_frames, inflight_batches, host_wait_ms, memory_budget_bytes)
        h = C.c_void_p()
        st = self.l.vaco_av1_server_create(C.byref(cfg), C.byref(h))
        if st != abi.OK:
            raise RuntimeError(f"vaco_av1_server_create failed with status {st}")
        self.h = h

    def close(self):
        if self.h:
            self.l.vaco_av1_server_destroy(self.h)
            self.h = None

    def open_stream(self, f: FrameInputs, buffers: int = 4):
        """Admit a stream with f's geometry and restoration unit sizes; returns (status, msg, id)."""
        info = f.info()
        sizes = (C.c_int32 * 3)(*[(f.lr_unit_size[k] if f.lr_units else 0) for k in range(3)])
        sid, msg = C.c_int32(-1), C.c_int32(0)
        st = self.l.vaco_av1_server_open_stream(self.h, C.byref(info), sizes, buffers, C.byref(sid), C.byref(msg))
        return st, msg.value, sid.value

    def upload(self, sid: int, slot: int, f: FrameInputs):
        job = host_job(f, [np.zeros((1, 1), np.uint16)] * f.num_planes)
        st = self.l.vaco_av1_server_upload(self.h, sid, slot, C.byref(job))
        if st != abi.OK:
            raise RuntimeError(f"upload failed: {st}")
        return job

    def download(self, sid: int, slot: int, f: FrameInputs) -> List[np.ndarray]:
        outs = [np.zeros(f.output_shape(k), np.uint16) for k in range(f.num_planes)]
        pic = picture_struct([ptr(o) for o in outs], [o.shape for o in outs])
        st = self.l.vaco_av1_server_download(self.h, sid, slot, C.byref(pic))
        if st != abi.OK:
            raise RuntimeError(f"download failed: {st}")
        return outs

    def submit(self, sid: int, slot: int, params: abi.FrameJob) -> int:
        t = C.c_uint64()
        st = self.l.vaco_av1_server_submit(self.h, sid, slot, C.byref(params), C.byref(t))
        if st != abi.OK:
            raise RuntimeError(f"submit refused: {st}")
        return t.value

    def try_submit(self, sid: int, slot: int, params: abi.FrameJob):
        """submit() returning (status, ticket) instead of raising."""
        t = C.c_uint64()
        st = self.l.vaco_av1_server_submit(self.h, sid, slot, C.byref(params), C.byref(t))
        return st, t.value

    def submit_host(self, sid: int, slot: int, host: abi.FrameJob) -> int:
        """Queue slot `slot` with its inputs copied from the host frame job
        `host` (host pointers; they must stay valid until wait returns)."""
        t = C.c_uint64()
        st = self.l.vaco_av1_server_submit_host(self.h, sid, slot, C.byref(host), C.byref(t))
        if st != abi.OK:
            raise RuntimeError(f"submit_host refused: {st}")
        return t.value

    def close_stream(self, sid: int) -> int:
        return self.l.vaco_av1_server_close_stream(self.h, sid)

    def wait(self, ticket: int, timeout_ms: int = -1):
        msg, lat = C.c_int32(0), C.c_double(0)
        st = self.l.vaco_av1_server_wait(self.h, ticket, timeout_ms, C.byref(msg), C.byref(lat))
        return st, msg.value, lat.value

    def stats(self) -> ServerStats:
        s = ServerStats()
        self.l.vaco_av1_server_get_stats(self.h, C.byref(s))
        return s


def frame_params(f: FrameInputs) -> abi.FrameJob:
    """Frame-level parameters of f (deblock, cdef, restoration types) for submit()."""
    j = abi.FrameJob()
    j.deblock = f.deblock_c()
    j.cdef = f.cdef.to_c()
    for k in range(3):
        j.lr_type[k] = f.lr_type[k] if k < f.num_planes else 0
    j.lvl_map = 1 if f.lvl_map is not None else None
    return j


# ---------------------------------------------------------------- serving benchmark
def _percentile(xs, q):
    if not xs:
        return None
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(q / 100.0 * (len(xs) - 1))))]


def run_load(server: Server, streams, rate_mult: float, seconds: float, fps: float = 30.0, seed: int = 0,
             upload: bool = False):
    """Poisson arrivals per stream at fps*rate_mult for `seconds`.

    A frame's latency is measured from its scheduled arrival: the submitter's
    lag behind the schedule, any backpressure wait inside submit (slot still
    in flight) and the server's submit-to-completion time.  With `upload`,
    every frame arrives in host memory (pinned) and goes in through
    vaco_av1_server_submit_host, so its latency also covers the copy of its
    inputs to the device; otherwise the frames are already resident."""
    rng = random.Random(seed)
    arrivals = []
    for s_idx, st in enumerate(streams):
        t = rng.expovariate(fps * rate_mult)
        while t < seconds:
            arrivals.append((t, s_idx))
            t += rng.expovariate(fps * rate_mult)
    arrivals.sort()
    inflight = deque()
    latencies, pixels, errors = [], 0, 0
    done = threading.Event()
    lock = threading.Lock()

    def collector():
        nonlocal pixels, errors
        while not (done.is_set() and not inflight):
            with lock:
                item = inflight.popleft() if inflight else None
            if item is None:
                time.sleep(0.0002)
                continue
            ticket, px, queued_ms = item
            st, msg, lat = server.wait(ticket, -1)
            if st != abi.OK:
                errors += 1
            latencies.append(queued_ms + lat)
            pixels += px

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    next_slot = [0] * len(streams)
    for t, s_idx in arrivals:
        now = time.perf_counter() - t0
        if t > now:
            time.sleep(t - now)
        st = streams[s_idx]
        slot = next_slot[s_idx]
        next_slot[s_idx] = (slot + 1) % st["buffers"]
        if upload:
            ticket = server.submit_host(st["id"], slot, st["host_jobs"][slot])
        else:
            ticket = server.submit(st["id"], slot, st["params"][slot])
        queued_ms = max(0.0, (time.perf_counter() - t0) - t) * 1e3
        with lock:
            inflight.append((ticket, st["pixels"], queued_ms))
    done.set()
    th.join()
    wall = time.perf_counter() - t0
    return {
        "rate_x_realtime": rate_mult, "uploads": upload, "offered_fps": round(len(streams) * fps * rate_mult, 1),
        "frames": len(latencies), "errors": errors, "seconds": round(wall, 2),
        "mpixel_s": round(pixels / wall / 1e6, 1),
        "p50_ms": round(_percentile(latencies, 50), 3) if latencies else None,
        "p99_ms": round(_percentile(latencies, 99), 3) if latencies else None,
        "max_ms": round(max(latencies), 3) if latencies else None,
    }


def saturation(server: Server, streams, rounds: int = 20, upload: bool = False):
    """Every slot of every stream submitted at once, round after round, with
    the bulk entry points: the served path's peak Mpixel/s.  With `upload`
    every frame goes in from pinned host memory through submit_host."""
    if upload:
        px = sum(st["pixels"] * st["buffers"] for st in streams)
        t0 = time.perf_counter()
        for _ in range(rounds):
            tickets = [server.submit_host(st["id"], b, st["host_jobs"][b]) for st in streams
                       for b in range(st["buffers"])]
            for t in tickets:
                assert server.wait(t, -1)[0] == abi.OK
        wall = time.perf_counter() - t0
        return {"frames": rounds * len(tickets), "mpixel_s": round(rounds * px / wall / 1e6, 1),
                "seconds": round(wall, 3), "uploads": True}
    ids, slots, params, px = [], [], [], 0
    for st in streams:
        for b in range(st["buffers"]):
            ids.append(st["id"])
            slots.append(b)
            params.append(st["params"][b])
            px += st["pixels"]
    n = len(ids)
    c_ids = (C.c_int32 * n)(*ids)
    c_slots = (C.c_int32 * n)(*slots)
    c_params = (abi.FrameJob * n)(*params)
    tickets = (C.c_uint64 * n)()
    l = server.l
    t0 = time.perf_counter()
    for _ in range(rounds):
        st = l.vaco_av1_server_submit_many(server.h, n, c_ids, c_slots, c_params, tickets)
        assert st == abi.OK, st
        st = l.vaco_av1_server_wait_many(server.h, n, tickets, -1, None, None, None)
        assert st == abi.OK, st
    wall = time.perf_counter() - t0
    return {"frames": rounds * n, "mpixel_s": round(rounds * px / wall / 1e6, 1), "seconds": round(wall, 3),
            "uploads": False}


def plain_dropin_mixed(device=0, frames_per_res=4, rounds=8):
    """The plain one-frame-per-call drop-in on the same mixed-resolution
    frames, two ways:
      with copies  vaco_av1_postfilter_frame_host: H2D + D2H every call, one
                   frame at a time, from pinned preallocated host buffers (the
                   drop-in's best case, so the served/plain ratio is not
                   inflated by pageable copies);
      resident     vaco_av1_postfilter_frame_dev on device-resident frames,
                   one call per frame, each synchronizing for its status.
    Mpixel/s of each."""
    from .gpu import Context, DeviceFrame

    ctx = Context(device)
    jobs, frames, px_per_round = [], [], 0
    for wl, _ in synth.BATCH_MIX:
        for i in range(frames_per_res):
            f = synth.make_frame(wl, synth.seed_for(4, 7000 + len(jobs)))
            pf, outs, job = pinned_copy(f)
            jobs.append((pf, outs, job))
            frames.append(f)
            px_per_round += f.output_pixels
    l, m = lib(), C.c_int32()
    for _, _, job in jobs:  # warm: every frame size once (scratch reaches its final size)
        assert l.vaco_av1_postfilter_frame_host(ctx.handle, C.byref(job), C.byref(m)) == abi.OK
    t0 = time.perf_counter()
    for _ in range(rounds):
        for _, _, job in jobs:
            st = l.vaco_av1_postfilter_frame_host(ctx.handle, C.byref(job), C.byref(m))
            if st != abi.OK:
                raise RuntimeError(f"host postfilter failed: {st}")
    wall = time.perf_counter() - t0
    devs = [DeviceFrame(f, device) for f in frames]
    for d in devs:
        ctx.postfilter_frame_dev(d)
    t1 = time.perf_counter()
    for _ in range(rounds):
        for d in devs:
            ctx.postfilter_frame_dev(d)
    wall_dev = time.perf_counter() - t1
    ctx.close()
    return {"frames": rounds * len(jobs), "mpixel_s": round(rounds * px_per_round / wall / 1e6, 1),
            "entry": "vaco_av1_postfilter_frame_host (pinned host buffers)",
            "resident_mpixel_s": round(rounds * px_per_round / wall_dev / 1e6, 1),
            "resident_entry": "vaco_av1_postfilter_frame_dev, one synchronous call per device-resident frame"}


def build_streams(server: Server, per_res: int = 8, buffers: int = 4, base_seed: int = 9000, pinned: bool = False):
    streams = []
    for wl, _ in synth.BATCH_MIX:
        for i in range(per_res):
            frames = [synth.make_frame(wl, synth.seed_for(4, base_seed + 100 * len(streams) + b)) for b in range(buffers)]
            st, msg, sid = server.open_stream(frames[0], buffers)
            if st != abi.OK:
                raise RuntimeError(f"stream admission refused: {abi.MESSAGES.get(msg)}")
            for b, f in enumerate(frames):
                server.upload(sid, b, f)
            entry = {"id": sid, "buffers": buffers, "pixels": frames[0].output_pixels,
                     "params": [frame_params(f) for f in frames], "frames": frames, "workload": wl.name}
            if pinned:  # host copies for submit_host: arrays stay referenced by the entry
                staged = [pinned_copy(f) for f in frames]
                entry["pinned"] = staged
                entry["host_jobs"] = [job for _, _, job in staged]
            streams.append(entry)
    return streams


SERVE_CONFIG = {"workload": "serve_32_streams", "streams": "8 x each of 640x360 8-bit, 1280x720 8-bit, "
                "1920x1080 10-bit, 3840x2160 10-bit", "fps_per_stream": 30, "memory_budget_gb": 40,
                "max_batch_frames": 64, "inflight_batches": 3, "buffers_per_stream": 4}


def served(device: int, seconds: float, rates=(1.0, 2.0, 4.0), saturation_rounds: int = 20):
    """Config 4 on one GPU: Poisson load at each rate for `seconds`, twice --
    frames resident in their slots, and every frame uploaded from pinned host
    memory inside its latency -- plus saturation both ways and the plain
    one-frame-per-call drop-in on the same mixed frames."""
    server = Server(device, max_batch_frames=64, inflight_batches=3)
    try:
        streams = build_streams(server, pinned=True)
        saturation(server, streams, rounds=3)  # warm: first launches of every batch shape
        saturation(server, streams, rounds=2, upload=True)
        resident = [run_load(server, streams, m, seconds, seed=int(m * 10)) for m in rates]
        uploaded = [run_load(server, streams, m, seconds, seed=int(m * 10) + 1, upload=True) for m in rates]
        sat = saturation(server, streams, rounds=saturation_rounds)
        sat_up = saturation(server, streams, rounds=max(2, saturation_rounds // 4), upload=True)
        stats = server.stats()
    finally:
        server.close()
    plain = plain_dropin_mixed(device)
    return {
        "config": dict(SERVE_CONFIG, seconds_per_rate=seconds),
        "resident": resident, "with_uploads": uploaded,
        "saturation": {"resident": sat, "with_uploads": sat_up},
        "plain_dropin_mixed": plain,
        "served_over_plain": {
            "with_copies": round(sat_up["mpixel_s"] / plain["mpixel_s"], 2) if plain["mpixel_s"] else None,
            "resident": round(sat["mpixel_s"] / plain["resident_mpixel_s"], 2) if plain["resident_mpixel_s"] else None,
            "note": "saturation with uploads / plain host drop-in (both copy every frame); "
                    "resident saturation / plain device-resident drop-in"},
        "server": {"batches": int(stats.batches), "max_batch": int(stats.max_batch),
                   "resident_gb": round(stats.resident_bytes / 2**30, 3)},
    }


def bench_main(args, world, rank, local):
    """bench.py --mode serve: config 4 (32 streams, Poisson arrivals)."""
    import torch

    torch.cuda.set_device(local)
    seconds = float(getattr(args, "serve_seconds", 0) or 60.0)
    res = served(local, seconds)
    if rank == 0:
        print(json.dumps(dict({"metric": "AV1 post-filter served p50/p99 ms/frame and Mpixel/s", "mode": "serve"},
                              **res)), flush=True)
