"""Launch-shape autotuner for the batched form and the per-frame chain.

Sweeps, with CUDA-event timing on the target GPU:
  batch  (64 mixed frames, config 3): threads per 64x64 tile of the fused
         deblock+CDEF kernel (256 or 128) with the resident CTAs per SM its
         body is compiled for (its register budget), the same for the
         restoration kernel, CUDA-graph replay, the frames' tile order, and
         the stage fusion (deblocking and CDEF in one kernel, or as separate
         kernels);
  frame  (4K 10-bit frames back to back): threads per tile of the fused
         kernel on the per-frame path.
and writes the fastest settings to tuned/<gpu>.json, which load_tuning()
reads.  Run on the target GPU:

    python -m vaco_b200.autotune
"""
from __future__ import annotations

import itertools
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
TUNED = ROOT / "tuned"
DEFAULT = {"dbcdef_ctas_per_sm": 3, "lr_ctas_per_sm": 4, "use_graphs": 1, "largest_first": 1, "dbcdef_threads": 256,
           "stage_fusion": 1}


def gpu_key() -> str:
    try:
        import torch

        if torch.cuda.is_available():
            name = torch.cuda.get_device_name(0)
            return "".join(c if c.isalnum() else "_" for c in name).strip("_").lower()
    except Exception:
        pass
    return "nvidia_b200"


def load_tuning() -> dict:
    """The tuned table for this GPU, else the committed B200 table, else defaults."""
    for name in (gpu_key(), "nvidia_b200"):
        p = TUNED / f"{name}.json"
        if p.exists():
            t = json.loads(p.read_text()).get("batch", {})
            return {k: int(t.get(k, v)) for k, v in DEFAULT.items()}
    return dict(DEFAULT)


# (threads per tile, resident CTAs per SM its body is compiled for) of the
# fused kernel: the three bodies there are (256 threads at 80 or 64 registers,
# 128 threads at 5 per SM)
DBCDEF_SHAPES = ((256, 3), (256, 4), (128, 5))


def _time(fn, reps, stream):
    import torch

    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main(argv=None):
    import itertools

    import torch

    from vaco_b200 import synth
    from vaco_b200.gpu import Context, DeviceFrame

    frames = []
    for wl, count in synth.BATCH_MIX:
        for _ in range(count):
            frames.append(synth.make_frame(wl, synth.seed_for(3, 5000 + len(frames))))
    ctx = Context(0)
    devs = [DeviceFrame(f) for f in frames]
    jobs = ctx.batch_jobs(devs)
    stream = torch.cuda.current_stream()
    results = []
    for (threads, db), lr, graphs, largest in itertools.product(DBCDEF_SHAPES, (3, 4), (0, 1), (0, 1)):
        cfg = {"dbcdef_threads": threads, "dbcdef_ctas_per_sm": db, "lr_ctas_per_sm": lr, "use_graphs": graphs,
               "largest_first": largest}
        ctx.set_tuning(**cfg)
        ms = _time(lambda: ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs), 10, stream)
        results.append((ms, cfg))
        print(json.dumps({"ms_per_batch": round(ms, 4), **cfg}), flush=True)
    # stage fusion: deblocking and CDEF as separate kernels, at the best shape so far
    results.sort(key=lambda r: r[0])
    unfused = dict(results[0][1], stage_fusion=0)
    ctx.set_tuning(**unfused)
    ms = _time(lambda: ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs), 10, stream)
    results.append((ms, unfused))
    print(json.dumps({"ms_per_batch": round(ms, 4), **unfused}), flush=True)
    ctx.set_tuning(stage_fusion=1)
    results.sort(key=lambda r: r[0])
    best_ms, best = results[0]
    best = dict(best, stage_fusion=best.get("stage_fusion", 1))
    del devs, jobs
    # per-frame chain: 4K 10-bit frames back to back (deferred status)
    k4 = [DeviceFrame(synth.make_frame(synth.CONFIG1, synth.seed_for(3, 6000 + i))) for i in range(8)]
    ctx.set_deferred_status(True)
    frame_results = []
    for threads in (256, 128):
        ctx.set_tuning(dbcdef_threads=threads)

        def run():
            for d in k4:
                ctx.postfilter_frame_dev(d, stream.cuda_stream)

        ms = _time(run, 50, stream) / len(k4)
        ctx.flush(stream.cuda_stream)
        frame_results.append((ms, {"dbcdef_threads": threads}))
        print(json.dumps({"frame_ms": round(ms, 5), "dbcdef_threads": threads}), flush=True)
    ctx.set_deferred_status(False)
    frame_results.sort(key=lambda r: r[0])
    out = {"gpu": torch.cuda.get_device_name(0), "workload": "64 mixed frames (synthetic batch mix)",
           "batch": best, "ms_per_batch": round(best_ms, 4),
           "frame": dict(frame_results[0][1], ms_per_4k_frame=round(frame_results[0][0], 5)),
           "sweep": [{"ms_per_batch": round(m, 4), **c} for m, c in results],
           "frame_sweep": [{"ms_per_4k_frame": round(m, 5), **c} for m, c in frame_results]}
    TUNED.mkdir(exist_ok=True)
    path = pathlib.Path(argv[0]) if argv else TUNED / f"{gpu_key()}.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(f"best {best} at {best_ms:.4f} ms/batch; per frame {frame_results[0][1]} -> {path}")
    ctx.close()


if __name__ == "__main__":
    main(sys.argv[1:])
