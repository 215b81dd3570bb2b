"""The batched form: many frames of different sizes and bit depths in one
launch set (one per-stage kernel launch over the tiles of all frames,
optionally replayed from a CUDA graph) give, frame by frame, exactly the
single-frame results and the oracle's."""
import numpy as np
import pytest
import torch

import oracle
from vaco_b200 import abi, synth
from vaco_b200.gpu import DeviceFrame

pytestmark = pytest.mark.gpu


def mixed_frames(seed0, small=True):
    geoms = [(200, 136, 10, None), (328, 200, 10, 400), (64, 64, 8, None), (520, 264, 12, None),
             (120, 72, 8, 136), (1280, 720, 8, None)]
    if not small:
        geoms.append((1920, 1080, 10, None))
    return [synth.make_small(seed0 + i, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=i % 2 == 1)
            for i, (w, h, bd, up) in enumerate(geoms)]


@pytest.mark.parametrize("graphs", [0, 1])
@pytest.mark.parametrize("largest_first", [0, 1])
def test_batch_matches_oracle_frame_by_frame(ctx, graphs, largest_first, oracle_threads):
    ctx.set_tuning(use_graphs=graphs, largest_first=largest_first)
    frames = mixed_frames(100, small=False)
    devs = [DeviceFrame(f) for f in frames]
    stream = torch.cuda.current_stream().cuda_stream
    st, ms = ctx.postfilter_batch_dev(devs, stream=stream)
    assert st == [0] * len(frames) and ms == [0] * len(frames)
    for f, d in zip(frames, devs):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        for g, w in zip(d.outputs_numpy(), want):
            np.testing.assert_array_equal(g, w)


def test_batch_mixed_chroma_layouts_match_oracle(ctx, oracle_threads):
    """One batch of 4:2:0, 4:2:2, 4:4:4 and monochrome frames: the batched
    fused kernel reads each frame's layout from its record."""
    layouts = [((1, 1), False), ((1, 0), False), ((0, 0), False), ((1, 1), True)]
    geoms = [(200, 136, 10, None), (328, 200, 10, 400), (60, 44, 8, None), (520, 264, 12, None),
             (120, 72, 8, 136), (96, 80, 12, None), (204, 130, 8, None), (256, 128, 10, 320)]
    frames = [synth.make_small(700 + i, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=i % 2 == 0,
                               subsampling=sub, monochrome=mono)
              for i, ((sub, mono), (w, h, bd, up)) in enumerate(zip(layouts * 2, geoms))]
    devs = [DeviceFrame(f) for f in frames]
    st, ms = ctx.postfilter_batch_dev(devs, stream=torch.cuda.current_stream().cuda_stream)
    assert st == [0] * len(frames) and ms == [0] * len(frames)
    for i, (f, d) in enumerate(zip(frames, devs)):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        for k, (g, w) in enumerate(zip(d.outputs_numpy(), want)):
            assert np.array_equal(g, w), f"frame {i} layout {layouts[i % 4]} plane {k} differs"


def test_batch_graph_replay_with_new_data(ctx, oracle_threads):
    ctx.set_tuning(use_graphs=1)
    stream = torch.cuda.current_stream().cuda_stream
    for seed0 in (200, 300, 400):  # same composition, different frames: one capture, two replays
        frames = mixed_frames(seed0)
        devs = [DeviceFrame(f) for f in frames]
        st, _ = ctx.postfilter_batch_dev(devs, stream=stream)
        assert st == [0] * len(frames)
        for f, d in zip(frames, devs):
            want, _ = oracle.postfilter_frame(f, threads=oracle_threads)
            for g, w in zip(d.outputs_numpy(), want):
                np.testing.assert_array_equal(g, w)


def test_batch_reports_errors_per_frame(ctx):
    frames = mixed_frames(500)
    frames[1].planes[0][3, 3] = 60000          # bad sample: deblocking check
    frames[3].lr_units[1][0] = (abi.LR_SGRPROJ, 0, (0, 0, 0), (0, 0, 0), (40, 0))  # bad coefficient in plane U
    devs = [DeviceFrame(f) for f in frames]
    st, ms = ctx.postfilter_batch_dev(devs, stream=torch.cuda.current_stream().cuda_stream)
    assert st[1] == abi.INVALID_DATA and ms[1] == abi.MSG["DB_SAMPLE"]
    assert st[3] == abi.INVALID_DATA and ms[3] == abi.MSG["LR_COEFFICIENT"]
    for i in (0, 2, 4, 5):
        assert st[i] == abi.OK
        want, _ = oracle.postfilter_frame(frames[i])
        for g, w in zip(devs[i].outputs_numpy(), want):
            np.testing.assert_array_equal(g, w)


def test_config3_full_mix_matches_oracle(ctx, oracle_threads):
    """Config 3 as specified: 64 frames, 16 each of 640x360 8-bit, 1280x720
    8-bit, 1920x1080 10-bit and 3840x2160 10-bit, independently seeded, in one
    launch set with the committed tuning; every frame bit-exact."""
    from vaco_b200 import autotune

    ctx.set_tuning(**autotune.load_tuning())
    stream = torch.cuda.current_stream().cuda_stream
    frames = []
    for wl, count in synth.BATCH_MIX:
        for i in range(count):
            frames.append(synth.make_frame(wl, synth.seed_for(3, 2000 + len(frames))))
    assert len(frames) == 64
    devs = [DeviceFrame(f) for f in frames]
    st, ms = ctx.postfilter_batch_dev(devs, stream=stream)
    assert st == [0] * 64 and ms == [0] * 64
    for i, (f, d) in enumerate(zip(frames, devs)):
        want, m = oracle.postfilter_frame(f, threads=oracle_threads)
        assert m == 0
        for k, (g, w) in enumerate(zip(d.outputs_numpy(), want)):
            assert np.array_equal(g, w), f"frame {i} ({f.coded_width}x{f.coded_height}) plane {k} differs"


@pytest.mark.parametrize("shape", [(256, 3, 1, 4), (256, 4, 1, 3), (128, 5, 1, 4), (256, 4, 0, 4)],
                         ids=["fused256x3", "fused256x4_lr3", "fused128", "unfused"])
def test_batch_launch_shapes_and_stage_fusion_match_oracle(ctx, shape, oracle_threads):
    """Every kernel body and stage-fusion choice the autotuner may pick gives
    the oracle's planes (superres frames and restoration included)."""
    threads, ctas, fusion, lr_ctas = shape
    ctx.set_tuning(dbcdef_threads=threads, dbcdef_ctas_per_sm=ctas, stage_fusion=fusion, use_graphs=1,
                   lr_ctas_per_sm=lr_ctas)
    try:
        frames = mixed_frames(900)
        devs = [DeviceFrame(f) for f in frames]
        st, ms = ctx.postfilter_batch_dev(devs, stream=torch.cuda.current_stream().cuda_stream)
        assert st == [0] * len(frames) and ms == [0] * len(frames)
        for f, d in zip(frames, devs):
            want, m = oracle.postfilter_frame(f, threads=oracle_threads)
            assert m == 0
            for g, w in zip(d.outputs_numpy(), want):
                np.testing.assert_array_equal(g, w)
    finally:
        ctx.set_tuning(dbcdef_threads=256, dbcdef_ctas_per_sm=3, stage_fusion=1, lr_ctas_per_sm=4)


def test_per_frame_128_thread_tiles_match_oracle(ctx, oracle_threads):
    """The per-frame chain with 128-thread tiles of the fused kernel."""
    ctx.set_tuning(dbcdef_threads=128)
    try:
        for f in mixed_frames(950, small=False):
            want, m = oracle.postfilter_frame(f, threads=oracle_threads)
            assert m == 0
            d = DeviceFrame(f)
            ctx.postfilter_frame_dev(d)
            for g, w in zip(d.outputs_numpy(), want):
                np.testing.assert_array_equal(g, w)
    finally:
        ctx.set_tuning(dbcdef_threads=256)
