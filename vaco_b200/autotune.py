"""Launch-shape autotuner for the batched form.

Sweeps the persistent grid of both per-stage kernels (CTAs per SM), CUDA-graph
replay and the tile-queue order on the batch workload (64 mixed frames) with
CUDA-event timing, and writes the fastest setting to tuned/<gpu>.json, which
load_tuning() reads.  Run on the target GPU:

    python -m vaco_b200.autotune
"""
from __future__ import annotations

import itertools
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
TUNED = ROOT / "tuned"
DEFAULT = {"dbcdef_ctas_per_sm": 3, "lr_ctas_per_sm": 4, "use_graphs": 1, "largest_first": 1, "dbcdef_threads": 256}


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


def main(argv=None):
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
    for db, lr, graphs, largest in itertools.product((2, 3, 4), (2, 3, 4), (0, 1), (0, 1)):
        ctx.set_tuning(dbcdef_ctas_per_sm=db, lr_ctas_per_sm=lr, use_graphs=graphs, largest_first=largest)
        for _ in range(3):
            ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(10):
            ctx.postfilter_batch_dev(devs, stream=stream.cuda_stream, jobs=jobs)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        cfg = {"dbcdef_ctas_per_sm": db, "lr_ctas_per_sm": lr, "use_graphs": graphs, "largest_first": largest}
        results.append((ms, cfg))
        print(json.dumps({"ms_per_batch": round(ms, 4), **cfg}), flush=True)
    results.sort(key=lambda r: r[0])
    best_ms, best = results[0]
    out = {"gpu": torch.cuda.get_device_name(0), "workload": "64 mixed frames (synthetic batch mix)",
           "batch": best, "ms_per_batch": round(best_ms, 4),
           "sweep": [{"ms_per_batch": round(m, 4), **c} for m, c in results]}
    TUNED.mkdir(exist_ok=True)
    path = pathlib.Path(argv[0]) if argv else TUNED / f"{gpu_key()}.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(f"best {best} at {best_ms:.4f} ms/batch -> {path}")
    ctx.close()


if __name__ == "__main__":
    main(sys.argv[1:])
