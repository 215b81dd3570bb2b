"""bench.py's issue roofline: the committed per-launch instruction counts
(ncu smsp__inst_executed.sum) cover every bench workload's kernels, and the
fraction is instructions / launch time / (SMs x 4 sub-partitions x clock)."""
import pytest

import bench

STAGE_MS = {"deblock_cdef": 0.17, "unused": 0.0, "superres": 0.027, "restoration": 0.058}


@pytest.mark.parametrize("workload", sorted(bench.WORKLOADS))
def test_every_workload_has_counts(workload):
    r = bench.issue_roofline(workload, STAGE_MS, {"sm_mhz": 1965.0}, 0.26, 148)
    assert r is not None
    assert r["peak"] == pytest.approx(148 * 4 * 1965e6)
    assert "deblock_cdef" in r["kernels"]
    for stage, k in r["kernels"].items():
        n, t = k["warp_instructions_per_launch"], STAGE_MS[stage]
        assert k["frac"] == pytest.approx(n / (t / 1e3) / r["peak"], abs=1e-4)
        assert 0 < k["frac"] < 1.5


def test_no_counts_or_no_clock_gives_none():
    assert bench.issue_roofline("no_such_workload", STAGE_MS, {"sm_mhz": 1965.0}, 0.26, 148) is None
    assert bench.issue_roofline("chain_4k_10bit", STAGE_MS, None, 0.26, 148) is None


def test_algorithmic_bytes_of_the_4k_chain():
    """The HBM roofline's numerators for the 4K 10-bit chain: the planes read
    and written once (24.9 MB each), the side information, and for the
    kernels the boundary rows between them."""
    from vaco_b200 import synth

    f = synth.make_frame(synth.CONFIG1, synth.seed_for(1, 0))
    fin, fout, side = bench.frame_bytes(f)
    assert fin == fout == 3840 * 2160 * 3 // 2 * 2  # 24,883,200
    assert 0.5e6 < side < 3e6
    sb = bench.stage_bytes(f)
    assert sb["deblock_cdef"] == pytest.approx(53.03e6, rel=2e-3)
    assert sb["restoration"] == pytest.approx(51.92e6, rel=2e-3)
    assert sb["superres"] == 0
