"""Multi-process replica path on CPU (gloo, world size 2): each rank filters
its own frames independently, results equal a single-process run, and the
timing reduction returns the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import oracle
    from vaco_b200 import replicas, synth

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    seeds = replicas.frame_seeds(rank, 2, 1)
    checks = []
    for s in seeds:
        f = synth.make_small(s, 136, 72, 10)
        out, m = oracle.postfilter_frame(f)
        assert m == 0
        checks.append(int(sum(int(o.astype(np.int64).sum()) for o in out)))
    dist.barrier()
    elapsed = 10.0 * (rank + 1)  # a rank-dependent stand-in for the timed region
    mx = replicas.max_over_ranks(elapsed)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(checks + [mx]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_are_independent_and_time_is_max_over_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    import oracle
    from vaco_b200 import replicas, synth

    for rank in range(world):
        got = np.load(tmp_path / f"rank{rank}.npy")
        assert got[-1] == 20.0  # max over ranks of 10, 20
        for i, s in enumerate(replicas.frame_seeds(rank, 2, 1)):
            out, m = oracle.postfilter_frame(synth.make_small(s, 136, 72, 10))
            assert got[i] == sum(int(o.astype(np.int64).sum()) for o in out)
    assert replicas.aggregate_mpixels(2, 10, 1_000_000, 1000.0) == pytest.approx(20.0)
