"""Benchmark: AV1 post-filter chain (deblock -> CDEF -> superres -> loop
restoration) on synthetic 4K 10-bit 4:2:0 frames, bit-exact to vaco's filters.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vaco_b200|reference]
                    [--workload chain_4k_10bit|superres_2880to3840_10bit|...]

One step = one frame through the whole chain.  Under torchrun each rank is an
independent replica on its own GPU (frames are independent; no collective on
the data path); the timed region is bracketed by a barrier and
torch.cuda.synchronize(), and the time reported is the max over ranks.

`value`      device throughput (Mpixel/s of output luma, whole job): inputs
             already resident in HBM, each step is vaco_av1_postfilter_frame_dev
             under deferred status (frames back to back, one flush at the end).
`e2e`        the same metric from host memory (pinned buffers): every step
             copies the frame's planes and side information host->device and
             the output planes device->host, through
             vaco_av1_postfilter_frame_host_submit / _wait with three frames
             in flight (the one-call-per-frame entry is reported beside it).
`roofline`   the dominant kernel's algorithmic bytes / its CUDA-event duration
             (per-stage events on the launching stream, on one frame in
             STAGE_SAMPLE across the timed region).
`cpu_baseline` the oracle (C++ restatement of vaco's scalar filters), one
             thread, on a bounded sample of the same workload.
`--impl reference` times that CPU restatement with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import pathlib
import statistics
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from vaco_b200 import synth  # noqa: E402

L2_BYTES = 126 * 2**20
ROTATE_FRAMES = 8  # distinct frames cycled through: > L2 of input planes at 4K

WORKLOADS = {w.name: (cfg, w) for cfg, w in [(1, synth.CONFIG1), (2, synth.CONFIG2), (2, synth.CONFIG2_DENOM12),
                                               (0, synth.CONFIG0)]}
METRIC = "AV1 post-filter Mpixel/s at 4K 10-bit (bit-exact); served p50/p99 ms/frame"
STAGES = ["deblock_cdef", "unused", "superres", "restoration"]  # vaco_av1_ctx_stage_ms slots
# Per-stage CUDA events go on one frame in STAGE_SAMPLE, spread over the whole
# timed region, so the events' own stream time barely touches the throughput.
STAGE_SAMPLE = 8
E2E_MIN_STEPS = 100          # e2e frames timed at least (each with its H2D and D2H copies)
SERVED_SECONDS_DEFAULT = 5.0  # seconds per arrival rate and mode in the default line's served block


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons of the benchmarked GPU during
    the timed region, read in-process through NVML.

    A thread samples every 2 ms from start() on; mark_start() / mark_end()
    also take one sample each, right at the edges of the timed region, so a
    region of a few milliseconds still yields a record made of the samples
    inside it plus the two bracketing ones.  The GPU is found by the UUID CUDA
    reports for the device (CUDA_VISIBLE_DEVICES may renumber it), so the
    sampled GPU is the one the kernels run on.  Falls back to None without
    NVML."""

    REASONS = {"hw_slowdown": "HwSlowdown", "hw_thermal_slowdown": "HwThermalSlowdown",
               "sw_thermal_slowdown": "SwThermalSlowdown", "sw_power_cap": "SwPowerCap",
               "hw_power_brake_slowdown": "HwPowerBrakeSlowdown"}

    def __init__(self, cuda_device: int):
        self.cuda_device = cuda_device
        self.samples = []  # (time, sm_mhz, reasons bitmask, watts)
        self.handle = None
        self.stop_flag = threading.Event()
        self.t_start = self.t_end = None

    def _open(self):
        import pynvml as nv
        import torch

        nv.nvmlInit()
        props = torch.cuda.get_device_properties(self.cuda_device)
        try:
            return nv.nvmlDeviceGetHandleByUUID(f"GPU-{props.uuid}")
        except Exception:
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)

    def sample(self):
        if self.handle is None:
            return
        nv = self.nv
        try:
            sm = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
            watts = nv.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
        except Exception:
            return
        self.samples.append((time.perf_counter(), sm, reasons, watts))

    def start(self):
        try:
            import pynvml

            self.nv = pynvml
            self.handle = self._open()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.handle = None
            return

        def loop():
            while not self.stop_flag.wait(0.002):
                self.sample()

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def mark_start(self):
        self.sample()
        self.t_start = time.perf_counter()

    def mark_end(self):
        self.t_end = time.perf_counter()
        self.sample()

    def stop(self):
        if self.handle is None:
            return None
        self.stop_flag.set()
        self.thread.join(timeout=2)
        return self.summary()

    def summary(self):
        """The record of the timed region: samples inside it plus the last
        one before and the first one after."""
        t0 = self.t_start if self.t_start is not None else -float("inf")
        t1 = self.t_end if self.t_end is not None else float("inf")
        inside = [x for x in self.samples if t0 <= x[0] <= t1]
        before = [x for x in self.samples if x[0] < t0][-1:]
        after = [x for x in self.samples if x[0] > t1][:1]
        window = before + inside + after
        if not window:
            return None
        reasons = set()
        for _, _, mask, _ in window:
            for name, suffix in self.REASONS.items():
                bit = getattr(self.nv, "nvmlClocksEventReason" + suffix, 0)
                if mask & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(x[1] for x in window), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "power_w_median": round(statistics.median(x[3] for x in window), 1),
                "samples": len(window), "samples_inside_region": len(inside),
                "source": "NVML, every 2 ms plus one sample at each edge of the timed region"}


# ---------------------------------------------------------------- algorithmic bytes
def frame_bytes(f):
    """Required bytes per frame: inputs read once + outputs written once + side info."""
    sample = 1 if f.bit_depth == 8 else 2
    fin = sum(p.size for p in f.planes[: f.num_planes]) * sample
    fout = sum(int(np.prod(f.output_shape(k))) for k in range(f.num_planes)) * sample
    side = sum(a.nbytes for a in f.side_arrays().values() if a is not None)
    side += sum(u.nbytes for u in f.lr_units)
    return fin, fout, side


def issue_roofline(workload: str, per_stage: dict, clock_info: dict, chain_ms: float, sms: int):
    """The chain's kernels are integer work that HBM does not bound, so beside
    the HBM roofline this reports the instruction-issue one: warp
    instructions per launch (ncu smsp__inst_executed.sum on the same
    workload, committed in profiles/instructions_per_launch.txt) over the
    stage's measured launch time, against one warp instruction per SM
    sub-partition per clock (4 per SM) at the SM clock sampled during the
    timed region.  None when the workload has no committed counts."""
    counts = {}
    tp = ROOT / "profiles" / "instructions_per_launch.txt"
    if tp.exists():
        for ln in tp.read_text().splitlines():
            parts = ln.split()
            if len(parts) == 3 and not ln.startswith("#") and parts[0] == workload:
                counts[parts[1]] = int(parts[2])
    mhz = (clock_info or {}).get("sm_mhz")
    if not counts or not mhz:
        return None
    peak = sms * 4 * mhz * 1e6  # warp instructions per second
    kernels = {}
    for stage, n in counts.items():
        t = per_stage.get(stage, 0.0)
        if t > 0:
            kernels[stage] = {"warp_instructions_per_launch": n, "launch_ms": round(t, 5),
                              "frac": round(n / (t / 1e3) / peak, 4)}
    total = sum(counts.values())
    return {"bound": "issue", "unit": "warp instructions/s", "peak": peak, "sms": sms, "sm_mhz": mhz,
            "kernels": kernels, "chain_frac": round(total / (chain_ms / 1e3) / peak, 4),
            "source": "ncu smsp__inst_executed.sum per launch (profiles/instructions_per_launch.txt)"}


def stage_bytes(f):
    """Algorithmic bytes per launch of each chain kernel (u16 planes).

    deblock_cdef (fused): read the reconstruction once, write the CDEF picture
    once, plus the transform/level/skip/index side information and the four
    pre-CDEF rows per stripe boundary that restoration needs.
    restoration: read the CDEF picture and those boundary rows, write the output.
    """
    pin = sum(p.size for p in f.planes[: f.num_planes]) * 2
    pout = sum(int(np.prod(f.output_shape(k))) for k in range(f.num_planes)) * 2
    side = f.tx_luma.nbytes + f.tx_chroma.nbytes + f.skip.nbytes + f.cdef_idx.nbytes
    if f.lvl_map is not None:
        side += f.lvl_map.nbytes
    boundary = 0
    for k in range(f.num_planes):
        rows, cols = f.padded_shape(k)
        sy = 1 if k else 0
        boundary += 4 * ((rows + (8 >> sy) + 2) // (64 >> sy) + 1) * cols * 2
    return {
        "deblock_cdef": 2 * pin + side + boundary,
        "unused": 0,
        "superres": 0,
        "restoration": pin + pout + boundary + sum(u.nbytes for u in f.lr_units),
    }


# ---------------------------------------------------------------- frames
def workload_frames(cfg_idx: int, workload, rank: int, count: int = ROTATE_FRAMES):
    """The frames rank `rank` of the GPU arm rotates through; the CPU legs
    filter the same frames (rank 0's)."""
    from vaco_b200 import replicas

    return [synth.make_frame(workload, s) for s in replicas.frame_seeds(rank, count, cfg_idx)]


def band_of(f, rows: int):
    """The top `rows` luma rows (a multiple of 64) of frame f as a frame of
    its own: same width, content, side information and restoration units
    (the first unit rows).  A bounded CPU sample of f's workload."""
    import dataclasses

    assert rows % 64 == 0 and 0 < rows <= f.coded_height
    g = dataclasses.replace(f, coded_height=rows)
    mi_rows = g.mi_rows
    g.planes = [np.ascontiguousarray(p[: g.padded_shape(k)[0]]) for k, p in enumerate(f.planes)]
    g.tx_luma = np.ascontiguousarray(f.tx_luma[:mi_rows])
    g.tx_chroma = np.ascontiguousarray(f.tx_chroma[: (mi_rows + f.subsampling_y) >> f.subsampling_y])
    g.skip = np.ascontiguousarray(f.skip[:mi_rows])
    g.cdef_idx = np.ascontiguousarray(f.cdef_idx[: (mi_rows + 15) // 16])
    g.lvl_map = None if f.lvl_map is None else np.ascontiguousarray(f.lvl_map[:mi_rows])
    units = []
    for k, u in enumerate(f.lr_units):
        h, w = g.output_shape(k)
        size = f.lr_unit_size[k]
        cols = max((w + size // 2) // size, 1)
        urows = max((h + size // 2) // size, 1)
        units.append(np.ascontiguousarray(u[: urows * cols]))
    g.lr_units = units
    return g


# ---------------------------------------------------------------- CPU legs
def time_oracle(f, threads, repeats):
    import oracle

    t0 = time.perf_counter()
    for _ in range(repeats):
        _, m = oracle.postfilter_frame(f, threads=threads)
        assert m == 0
    return (time.perf_counter() - t0) / repeats


def cpu_baseline(frames, workload, seconds: float = 12.0):
    """The oracle on 1 core over the GPU arm's own frames, whole frames one
    after another until about `seconds` of CPU work (at least one)."""
    import oracle

    oracle.lib()  # load (page in) outside the timing
    t0 = time.perf_counter()
    n, px = 0, 0
    while n < len(frames) and (n == 0 or time.perf_counter() - t0 < seconds):
        _, m = oracle.postfilter_frame(frames[n], threads=1)
        assert m == 0
        px += frames[n].output_pixels
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(px / dt / 1e6, 3), "unit": "Mpixel/s", "cores": 1, "kind": "port",
            "sample": f"{n} whole {workload.upscaled_width}x{workload.height} frames of the timed rotation "
                      f"({workload.name}, full chain), 1 thread"}


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement with every host thread, on the
    frames the GPU arm filters (rank 0's rotation).  A step is one whole
    frame when K + W of them fit in about two minutes, else the top band of
    the same frame, as many rows as fit."""
    if rank != 0:
        return
    cfg_idx, workload = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    frames = workload_frames(cfg_idx, workload, 0)
    import oracle

    oracle.lib()
    t_frame = time_oracle(frames[0], threads, 1)  # also the first warm-up step
    per_step = 120.0 / max(1, args.steps + args.warmup)
    if t_frame <= per_step:
        samples, rows = frames, workload.height
    else:
        rows = max(64, int(workload.height * per_step / t_frame) // 64 * 64)
        samples = [band_of(f, rows) for f in frames]
    for i in range(1, args.warmup):
        oracle.postfilter_frame(samples[i % len(samples)], threads=threads)
    t0 = time.perf_counter()
    px = 0
    for i in range(args.steps):
        f = samples[i % len(samples)]
        _, m = oracle.postfilter_frame(f, threads=threads)
        assert m == 0
        px += f.output_pixels
    dt = time.perf_counter() - t0
    value = px / dt / 1e6
    what = "whole frames" if rows == workload.height else f"top {rows}-row bands"
    sample = (f"{what} of the GPU arm's {len(frames)} rotated {workload.name} frames (same seeds), "
              f"{threads} threads, one per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mpixel/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic (the GPU arm's seeded frames)",
        "config": {"workload": workload.name, "width": workload.width, "height": workload.height,
                   "upscaled_width": workload.upscaled_width, "bit_depth": workload.bit_depth,
                   "sample_rows": rows, "frames_rotated": len(frames)},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mpixel/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mpixel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU leg
def hbm_peak():
    pp = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(pp.read_text()) if pp.exists() else {}
    return float(peaks.get("hbm_gbs", 6650.0)), ("measured" if "hbm_gbs" in peaks else "fallback")


def run_gpu(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from vaco_b200 import abi, replicas
    from vaco_b200._lib import lib
    from vaco_b200.frame import pinned_copy
    from vaco_b200.gpu import Context, DeviceFrame

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    cfg_idx, workload = WORKLOADS[args.workload]
    frames = workload_frames(cfg_idx, workload, rank)
    ctx = Context(local)
    dev = [DeviceFrame(f, local) for f in frames]
    stream = torch.cuda.current_stream(local)
    sptr = C.c_void_p(stream.cuda_stream)
    m = C.c_int32()

    def step(i):
        st = lib().vaco_av1_postfilter_frame_dev(ctx.handle, sptr, C.byref(dev[i % ROTATE_FRAMES].job), C.byref(m))
        if st != abi.OK:
            raise RuntimeError(f"postfilter failed: status {st} msg {abi.MESSAGES.get(m.value)}")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, device="cuda")

    # -------- device-resident throughput.  Frames go back to back with
    # deferred status: no host round trip between frames, one flush (which
    # raises any device-side error of the timed frames) after the region.
    clocks = ClockSampler(local)
    clocks.start()  # sampling runs from before warm-up; the timed region's samples are kept
    for i in range(args.warmup):
        step(i)
    lib().vaco_av1_ctx_set_deferred_status(ctx.handle, 1)
    lib().vaco_av1_ctx_set_stage_timing(ctx.handle, STAGE_SAMPLE)
    launches0 = ctx.launches
    barrier()
    clocks.mark_start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        step(i)
    ev1.record(stream)
    if lib().vaco_av1_ctx_flush(ctx.handle, sptr, C.byref(m)) != abi.OK:
        raise RuntimeError(f"postfilter failed: {abi.MESSAGES.get(m.value)}")
    barrier()
    clocks.mark_end()
    clock_info = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches = ctx.launches - launches0
    stage_ms = (C.c_double * 4)()
    nframes = C.c_uint64()
    lib().vaco_av1_ctx_stage_ms(ctx.handle, stage_ms, C.byref(nframes))
    lib().vaco_av1_ctx_set_stage_timing(ctx.handle, 0)
    lib().vaco_av1_ctx_set_deferred_status(ctx.handle, 0)
    px = frames[0].output_pixels
    value = replicas.aggregate_mpixels(world, args.steps, px, ms)

    # -------- end to end from host memory (pinned buffers): every step copies
    # its frame's planes and side information to the device and its output
    # planes back.  vaco_av1_postfilter_frame_host_submit / _wait keep three
    # frames in flight, so one frame's copies overlap another's filtering;
    # the one-call-per-frame vaco_av1_postfilter_frame_host is timed too.
    staged = [pinned_copy(f) for f in frames[:3]]
    jobs = [job for _, _, job in staged]
    fin, fout, side = frame_bytes(frames[0])
    h2d = sum(p.nbytes for p in staged[0][0].planes) + side
    d2h = sum(o.nbytes for o in staged[0][1])
    e2e_steps = max(E2E_MIN_STEPS, args.steps // 4)

    def pipelined(n):
        inflight = []
        t = C.c_uint64()
        for i in range(n):
            if len(inflight) == 3:
                if lib().vaco_av1_postfilter_frame_host_wait(ctx.handle, inflight.pop(0), C.byref(m)) != abi.OK:
                    raise RuntimeError(f"host postfilter failed: {abi.MESSAGES.get(m.value)}")
            if lib().vaco_av1_postfilter_frame_host_submit(ctx.handle, C.byref(jobs[i % 3]), C.byref(t),
                                                           C.byref(m)) != abi.OK:
                raise RuntimeError(f"host postfilter submit failed: {abi.MESSAGES.get(m.value)}")
            inflight.append(t.value)
        for tk in inflight:
            if lib().vaco_av1_postfilter_frame_host_wait(ctx.handle, tk, C.byref(m)) != abi.OK:
                raise RuntimeError(f"host postfilter failed: {abi.MESSAGES.get(m.value)}")

    pipelined(args.warmup)
    barrier()
    t0 = time.perf_counter()
    pipelined(e2e_steps)
    barrier()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3)
    e2e_value = replicas.aggregate_mpixels(world, e2e_steps, px, e2e_ms)
    sync_steps = max(E2E_MIN_STEPS // 4, e2e_steps // 4)
    for i in range(args.warmup):
        lib().vaco_av1_postfilter_frame_host(ctx.handle, C.byref(jobs[i % 3]), C.byref(m))
    barrier()
    t0 = time.perf_counter()
    for i in range(sync_steps):
        if lib().vaco_av1_postfilter_frame_host(ctx.handle, C.byref(jobs[i % 3]), C.byref(m)) != abi.OK:
            raise RuntimeError(f"host postfilter failed: {abi.MESSAGES.get(m.value)}")
    barrier()
    sync_ms = max_over_ranks((time.perf_counter() - t0) * 1e3)
    e2e_sync_value = replicas.aggregate_mpixels(world, sync_steps, px, sync_ms)
    del staged, jobs

    line = None
    if rank == 0:
        peak, peak_src = hbm_peak()
        per_stage = {STAGES[k]: stage_ms[k] / max(1, nframes.value) for k in range(4)}
        sb = stage_bytes(frames[0])
        dominant = max(per_stage, key=per_stage.get)
        dom_ms = per_stage[dominant]
        achieved = sb[dominant] / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
        traffic = None
        tp = ROOT / "profiles" / "dram_traffic_per_launch.txt"
        if tp.exists():
            for ln in tp.read_text().splitlines():
                parts = ln.split()
                if len(parts) == 3 and not ln.startswith("#") and parts[0] == args.workload and parts[1] == dominant:
                    traffic = int(parts[2])
        chain_ms = ms / args.steps
        required = fin + fout + side
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        issue = issue_roofline(args.workload, per_stage, clock_info, chain_ms, sms)
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "Mpixel/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(chain_ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
            "data": "synthetic (seeded content/side-info model; 8 distinct frames rotated)",
            "config": {"workload": workload.name, "width": workload.width, "height": workload.height,
                       "upscaled_width": workload.upscaled_width, "bit_depth": workload.bit_depth,
                       "subsampling": "4:2:0", "frames_rotated": ROTATE_FRAMES,
                       "l2": f"inputs rotate over {ROTATE_FRAMES} frames ({ROTATE_FRAMES * fin / 2**20:.0f} MiB of "
                             f"input planes) > L2",
                       "parallelism": f"replicas x{world}",
                       "entry": "vaco_av1_postfilter_frame_dev, deferred status, one flush per timed region"},
            "e2e": {"value": round(e2e_value, 1), "unit": "Mpixel/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "entry": "vaco_av1_postfilter_frame_host_submit/_wait (pinned host buffers, 3 frames in flight)",
                    "one_call_per_frame": {"value": round(e2e_sync_value, 1), "steps": sync_steps,
                                           "entry": "vaco_av1_postfilter_frame_host"}},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_launch": int(sb[dominant]),
                         "launch_ms": round(dom_ms, 5), "launches_timed": int(nframes.value)},
            "chain_roofline": {"required_bytes_per_frame": int(required),
                               "achieved_gbs": round(required / (chain_ms / 1e3) / 1e9, 1),
                               "frac_of_hbm": round(required / (chain_ms / 1e3) / 1e9 / peak, 4)},
            "stage_ms": {k: round(v, 5) for k, v in per_stage.items()},
            "issue_roofline": issue,
            "gpu_launches": int(launches),
            "clocks": clock_info,
        }
    ctx.close()
    del dev
    if world == 1 and args.extras:
        # The batched and served forms of the metric, on the same GPU (one
        # replica only: their configs are single-GPU workloads).
        line["batched"] = batched_block(args, local)
        line["served"] = serve_mod().served(local, args.serve_seconds or SERVED_SECONDS_DEFAULT)
    if rank == 0:
        if args.cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(frames, workload)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def serve_mod():
    from vaco_b200 import serve

    return serve


def run_emit(args, world, rank, local):
    """--mode emit: pic_to_frame on the device (vaco_av1_emit_frame_dev).

    A stream kernel: bytes = the u16 planes read once + the packed frame
    written once.  Eight pictures rotate (more than L2 holds) and the step
    count is fixed so the run stays short."""
    import torch

    from vaco_b200 import abi
    from vaco_b200._lib import lib
    from vaco_b200.frame import frame_layout, picture_struct
    from vaco_b200.gpu import Context

    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.current_stream(local)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    lines = []
    for name, (w, h, bd) in {"emit_4k_10bit": (3840, 2160, 10), "emit_1080p_8bit": (1920, 1080, 8)}.items():
        info = abi.FrameInfo()
        info.bit_depth, info.subsampling_x, info.subsampling_y = bd, 1, 1
        info.upscaled_width, info.coded_width, info.coded_height = w, w, h
        info.mi_cols, info.mi_rows = 2 * ((w + 7) >> 3), 2 * ((h + 7) >> 3)
        shapes = [(h, w), (h // 2, w // 2), (h // 2, w // 2)]
        gen = torch.Generator(device="cuda").manual_seed(w)
        pics, outs, args_c = [], [], []
        for _ in range(8):
            planes = [torch.randint(0, 1 << bd, s, dtype=torch.int16, device="cuda", generator=gen) for s in shapes]
            frame = [torch.zeros(b.shape, dtype=torch.uint8, device="cuda") for b in frame_layout(info)]
            fb = abi.FrameBuffer()
            for k, t in enumerate(frame):
                fb.planes[k] = t.data_ptr()
                fb.linesize[k] = t.shape[1]
            pics.append(planes)
            outs.append(frame)
            args_c.append((picture_struct([t.data_ptr() for t in planes], shapes), fb))
        m = C.c_int32()
        sptr = C.c_void_p(stream.cuda_stream)

        def step(i):
            pic, fb = args_c[i % 8]
            if lib().vaco_av1_emit_frame_dev(ctx.handle, sptr, C.byref(pic), C.byref(info), C.byref(fb),
                                             C.byref(m)) != abi.OK:
                raise RuntimeError(f"emit failed: {abi.MESSAGES.get(m.value)}")

        for i in range(max(args.warmup, 3)):
            step(i)
        steps = 400
        # The device entry point only enqueues, so the launches run back to back.
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            step(i)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        bytes_in = sum(a * b for a, b in shapes) * 2
        bytes_out = sum(a * b for a, b in shapes) * (2 if bd > 8 else 1)
        gbs = (bytes_in + bytes_out) / (ms / 1e3) / 1e9
        lines.append({"workload": name, "ms_per_frame": round(ms, 5), "bytes_per_frame": bytes_in + bytes_out,
                      "achieved_gbs": round(gbs, 1), "frac_of_hbm": round(gbs / hbm_peak, 4),
                      "mpixel_s": round(w * h / (ms / 1e3) / 1e6, 1)})
    # End to end from host buffers (pinned): the chain alone returning u16
    # planes, against the chain followed by emission returning the packed
    # frame (half the bytes back at 8 bits).
    from vaco_b200.frame import frame_buffer, pinned_copy

    e2e = []
    for wl in (synth.BATCH_MIX[1][0], synth.CONFIG1):
        f = synth.make_frame(wl, synth.seed_for(3, 9100))
        pf, outs, job = pinned_copy(f)
        frame = [torch.from_numpy(b).pin_memory().numpy() for b in frame_layout(f.info())]
        fb = frame_buffer(frame)
        m = C.c_int32()
        res = {"workload": wl.name}
        ctx2 = Context(local)
        calls = {
            "chain_u16_out": (lambda: lib().vaco_av1_postfilter_frame_host(ctx2.handle, C.byref(job), C.byref(m)),
                              sum(o.nbytes for o in outs)),
            "chain_then_emit": (lambda: lib().vaco_av1_postfilter_frame_emit_host(ctx2.handle, C.byref(job),
                                                                                  C.byref(fb), C.byref(m)),
                                sum(b.nbytes for b in frame)),
        }
        for label, (call, d2h) in calls.items():
            for _ in range(3):
                assert call() == abi.OK
            n = 50
            t0 = time.perf_counter()
            for _ in range(n):
                assert call() == abi.OK
            dt = (time.perf_counter() - t0) / n
            res[label] = {"mpixel_s": round(f.output_pixels / dt / 1e6, 1), "d2h_bytes": int(d2h)}
        ctx2.close()
        e2e.append(res)
    ctx.close()
    if rank == 0:
        print(json.dumps({"metric": "AV1 frame emission (pic_to_frame) GB/s on the device", "mode": "emit",
                          "unit": "GB/s", "peak": hbm_peak, "lines": lines, "e2e_host": e2e}), flush=True)


def grain_params_4k():
    """Film grain parameters of the grain workload: 8 luma and 4 + 4 chroma
    scaling points, auto-regression lag 3, overlap on (the most work per
    sample the syntax allows)."""
    from vaco_b200 import abi

    rng = np.random.default_rng(0x6A1)
    p = abi.FilmGrainParams()
    p.apply_grain, p.grain_seed, p.overlap_flag = 1, 0x1234, 1
    for n, v, sc in ((8, p.point_y_value, p.point_y_scaling), (4, p.point_cb_value, p.point_cb_scaling),
                     (4, p.point_cr_value, p.point_cr_scaling)):
        for i, x in enumerate(np.sort(rng.choice(256, n, replace=False))):
            v[i], sc[i] = int(x), int(rng.integers(16, 128))
    p.num_y_points, p.num_cb_points, p.num_cr_points = 8, 4, 4
    p.grain_scaling_minus_8, p.ar_coeff_lag, p.ar_coeff_shift_minus_6 = 3, 3, 1
    for arr, n in ((p.ar_coeffs_y_plus_128, 24), (p.ar_coeffs_cb_plus_128, 25), (p.ar_coeffs_cr_plus_128, 25)):
        for i in range(n):
            arr[i] = int(np.clip(128 + rng.normal(0, 12), 0, 255))
    p.cb_mult, p.cb_luma_mult, p.cb_offset = 128, 192, 256
    p.cr_mult, p.cr_luma_mult, p.cr_offset = 128, 192, 256
    return p


def run_grain(args, world, rank, local):
    """--mode grain: film grain synthesis (AV1 7.18.3) of 4K 10-bit 4:2:0
    frames on the device (vaco_av1_film_grain_dev under deferred status, so
    frames run back to back).  Eight input frames rotate (more than L2
    holds).  The Gaussian table is a seeded synthetic stand-in for the spec's
    normative one, which the caller supplies."""
    import torch

    from vaco_b200 import abi
    from vaco_b200._lib import lib
    from vaco_b200.frame import picture_struct
    from vaco_b200.gpu import Context

    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.current_stream(local)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    w, h, bd = 3840, 2160, 10
    info = abi.FrameInfo()
    info.bit_depth, info.subsampling_x, info.subsampling_y = bd, 1, 1
    info.upscaled_width, info.coded_width, info.coded_height = w, w, h
    info.mi_cols, info.mi_rows = 2 * ((w + 7) >> 3), 2 * ((h + 7) >> 3)
    shapes = [(h, w), (h // 2, w // 2), (h // 2, w // 2)]
    gen = torch.Generator(device="cuda").manual_seed(w)
    gauss = np.random.default_rng(7).integers(-2048, 2048, 2048).astype(np.int16)
    params = grain_params_4k()
    frames = []
    for _ in range(8):
        src = [torch.randint(0, 1 << bd, s, dtype=torch.int16, device="cuda", generator=gen) for s in shapes]
        dst = [torch.empty_like(t) for t in src]
        frames.append((src, dst, picture_struct([t.data_ptr() for t in src], shapes),
                       picture_struct([t.data_ptr() for t in dst], shapes)))
    m = C.c_int32()
    sptr = C.c_void_p(stream.cuda_stream)
    ctx.set_deferred_status(True)

    def step(i):
        _, _, pin, pout = frames[i % 8]
        if lib().vaco_av1_film_grain_dev(ctx.handle, sptr, C.byref(pin), C.byref(pout), C.byref(info),
                                         C.byref(params), gauss.ctypes.data, C.byref(m)) != abi.OK:
            raise RuntimeError(f"film grain failed: {abi.MESSAGES.get(m.value)}")

    for i in range(max(args.warmup, 3)):
        step(i)
    ctx.flush(stream.cuda_stream)
    steps = 400
    launches0 = ctx.launches
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        step(i)
    e1.record(stream)
    e1.synchronize()
    ctx.flush(stream.cuda_stream)
    ms = e0.elapsed_time(e1) / steps
    launches = ctx.launches - launches0
    ctx.set_deferred_status(False)
    ctx.close()
    samples = sum(a * b for a, b in shapes)
    bytes_ = 2 * samples * 2  # u16 planes read once and written once
    gbs = bytes_ / (ms / 1e3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": "AV1 film grain synthesis Mpixel/s on the device", "mode": "grain", "unit": "Mpixel/s",
            "value": round(w * h / (ms / 1e3) / 1e6, 1), "ms_per_frame": round(ms, 5), "steps": steps,
            "config": {"workload": "grain_4k_10bit", "width": w, "height": h, "bit_depth": bd, "subsampling": "4:2:0",
                       "ar_coeff_lag": 3, "overlap": 1, "points": [8, 4, 4], "frames_rotated": 8,
                       "gaussian_table": "seeded synthetic stand-in (caller-supplied in the product)"},
            "hbm_roofline": {"bytes_per_frame": bytes_, "achieved_gbs": round(gbs, 1), "peak": hbm_peak,
                             "frac": round(gbs / hbm_peak, 4)},
            "gpu_launches": launches}), flush=True)


def batched_block(args, local, steps=None):
    """Config 3: 64 frames of mixed sizes (16 each of 640x360 8-bit, 1280x720
    8-bit, 1920x1080 10-bit, 3840x2160 10-bit), independently seeded, through
    vaco_av1_postfilter_batch_dev (persistent per-stage kernels over a device
    tile queue, CUDA-graph replay, tuned launch shape), beside the same 64
    frames through the per-frame entry point back to back (deferred status),
    and a batch of 16 4K 10-bit frames."""
    import torch

    from vaco_b200 import autotune
    from vaco_b200.gpu import Context, DeviceFrame

    steps = steps or max(5, min(args.steps, 50))
    ctx = Context(local)
    tuning = autotune.load_tuning()
    ctx.set_tuning(**tuning)
    stream = torch.cuda.current_stream(local)
    hbm, _ = hbm_peak()

    def rates(frames, ms):
        px = sum(f.output_pixels for f in frames)
        req = sum(sum(frame_bytes(f)) for f in frames)
        return {"value": round(px / (ms / 1e3) / 1e6, 1), "ms_per_batch": round(ms, 4),
                "frames_per_batch": len(frames),
                "hbm_roofline": {"required_bytes_per_batch": int(req),
                                 "achieved_gbs": round(req / (ms / 1e3) / 1e9, 1), "peak": hbm,
                                 "frac": round(req / (ms / 1e3) / 1e9 / hbm, 4)}}

    def time_batch(devs):
        jobs = ctx.batch_jobs(devs)
        for _ in range(max(3, args.warmup)):
            st, _ = ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs)
            assert all(x == 0 for x in st)
        torch.cuda.synchronize()
        launches0 = ctx.launches
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / steps, (ctx.launches - launches0) / steps

    def time_per_frame(devs):
        ctx.set_deferred_status(True)
        for d in devs:
            ctx.postfilter_frame_dev(d, stream.cuda_stream)
        ctx.flush(stream.cuda_stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            for d in devs:
                ctx.postfilter_frame_dev(d, stream.cuda_stream)
        ev1.record(stream)
        ctx.flush(stream.cuda_stream)
        ctx.set_deferred_status(False)
        return ev0.elapsed_time(ev1) / steps

    mix = []
    for wl, count in synth.BATCH_MIX:
        for i in range(count):
            mix.append(synth.make_frame(wl, synth.seed_for(3, len(mix))))
    devs = [DeviceFrame(f, local) for f in mix]
    ms, launches = time_batch(devs)
    mixed = rates(mix, ms)
    mixed["gpu_launches_per_batch"] = launches
    per_frame = rates(mix, time_per_frame(devs))
    del devs
    k4 = [synth.make_frame(synth.CONFIG1, synth.seed_for(3, 500 + i)) for i in range(16)]
    devs = [DeviceFrame(f, local) for f in k4]
    ms4, _ = time_batch(devs)
    only4k = rates(k4, ms4)
    del devs
    ctx.close()
    return dict(mixed, steps=steps, tuning=tuning,
                config={"workload": "batch_mix_64", "mix": [[w.name, c] for w, c in synth.BATCH_MIX]},
                per_frame_same_mix={"value": per_frame["value"], "ms_per_64_frames": per_frame["ms_per_batch"],
                                    "entry": "vaco_av1_postfilter_frame_dev per frame, deferred status"},
                batch_4k_10bit_16=only4k)


def run_batch(args, world, rank, local):
    """--mode batch: the batched block alone, as its own JSON line."""
    import torch

    torch.cuda.set_device(local)
    res = batched_block(args, local, steps=args.steps)
    if rank == 0:
        print(json.dumps(dict({"metric": "AV1 post-filter Mpixel/s, batched mixed-resolution frames",
                               "mode": "batch", "unit": "Mpixel/s", "warmup": args.warmup}, **res)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="vaco_b200", choices=["vaco_b200", "reference"])
    ap.add_argument("--workload", default="chain_4k_10bit", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--mode", default="headline", choices=["headline", "batch", "serve", "emit", "grain"])
    ap.add_argument("--serve-seconds", type=float, default=None,
                    help="seconds per arrival rate and mode: --mode serve (default 60) and the default line's "
                         "served block (default 5)")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="headline line without its batched and served blocks")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.mode == "batch":
        run_batch(args, world, rank, local)
        return
    if args.mode == "emit":
        run_emit(args, world, rank, local)
        return
    if args.mode == "grain":
        run_grain(args, world, rank, local)
        return
    if args.mode == "serve":
        from vaco_b200 import serve

        serve.bench_main(args, world, rank, local)
        return
    run_gpu(args, world, rank, local)


if __name__ == "__main__":
    main()
