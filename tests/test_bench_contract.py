"""Host-side pieces of bench.py that need no GPU: the clock record of a
short timed region, and the CPU legs' sample of the GPU arm's frames."""
import types

import numpy as np

import bench
import oracle
from vaco_b200 import synth


def _sampler(samples, t0, t1):
    nv = types.SimpleNamespace(nvmlClocksEventReasonSwPowerCap=0x4, nvmlClocksEventReasonHwSlowdown=0x8,
                               nvmlClocksEventReasonSwThermalSlowdown=0x20,
                               nvmlClocksEventReasonHwThermalSlowdown=0x40,
                               nvmlClocksEventReasonHwPowerBrakeSlowdown=0x80)
    c = bench.ClockSampler(0)
    c.nv, c.handle, c.max_mhz = nv, object(), 1965
    c.samples = samples
    c.t_start, c.t_end = t0, t1
    return c.summary()


def test_clock_record_of_a_region_shorter_than_the_sampling_period():
    # a 4 ms region with no periodic sample inside: the edge samples make the record
    rec = _sampler([(0.0, 1200, 0x1, 100.0), (1.000, 1965, 0, 700.0), (1.004, 1965, 0x4, 710.0),
                    (1.010, 1500, 0x8, 300.0)], 1.0005, 1.0035)
    assert rec["samples"] == 2 and rec["samples_inside_region"] == 0
    assert rec["sm_mhz"] == 1965 and rec["sm_max_mhz"] == 1965
    assert rec["reasons"] == ["sw_power_cap"]  # the idle sample before and the throttle after are outside


def test_clock_record_keeps_inside_samples_and_flags_throttling():
    samples = [(0.5, 1965, 0, 500.0)] + [(1.0 + 0.002 * i, 1900 + i, 0x40 if i == 3 else 0, 800.0) for i in range(6)]
    rec = _sampler(samples + [(2.0, 1965, 0, 500.0)], 1.0, 1.011)
    assert rec["samples_inside_region"] == 6 and rec["samples"] == 8
    assert rec["reasons"] == ["hw_thermal_slowdown"]


def test_cpu_band_is_the_top_of_the_gpu_arms_frame():
    frames = bench.workload_frames(1, synth.Workload("t", 640, 256, 10, 640, True), 0, count=2)
    assert [f.coded_height for f in frames] == [256, 256]
    band = bench.band_of(frames[1], 128)
    full, m = oracle.postfilter_frame(frames[1], threads=4)
    part, m2 = oracle.postfilter_frame(band, threads=4)
    assert m == m2 == 0
    for k, (a, b) in enumerate(zip(part, full)):
        rows = (128 - 24) >> (1 if k else 0)  # rows whose stripes and units do not reach the band's bottom
        assert np.array_equal(a[:rows], b[:rows]), k
