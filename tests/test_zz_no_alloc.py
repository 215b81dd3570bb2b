"""vaco_av1_postfilter_frame_noalloc: the whole chain for callers that cannot
call cudaMalloc.

Such a caller might be a decoder plugin whose host application owns all
device memory and forbids plugins from allocating, or a real-time path that
cannot afford an allocation's device-wide synchronization.  The entry point
keeps its intermediates in a fixed 16 MiB device array inside the library,
so it must give exactly the same planes as the context-based
vaco_av1_postfilter_frame_dev.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from vaco_b200 import abi, synth
from vaco_b200._lib import lib
from vaco_b200.gpu import Context, DeviceFrame

pytestmark = pytest.mark.gpu


def _noalloc(dev: DeviceFrame):
    import torch

    m = C.c_int32(-1)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib().vaco_av1_postfilter_frame_noalloc(stream, C.byref(dev.job), C.byref(m))
    torch.cuda.synchronize()
    return st, m.value


def _fresh_device_frame(f):
    d = DeviceFrame(f)
    for o in d.outputs:
        o.fill_(-1)  # stale contents that a correct call overwrites
    return d


@pytest.mark.parametrize("geom", [(328, 200, 10, 400), (1280, 720, 8, None)])
def test_noalloc_matches_context_entry_point_on_two_calls_in_a_row(geom):
    import torch

    torch.cuda.init()
    w, h, bd, up = geom
    ctx = Context(0)
    try:
        for seed in (31, 32):  # two calls in a row share the scratch array
            f = synth.make_small(seed, w, h, bd, upscaled_width=up, sharpness=None, with_lvl_map=seed == 32)
            ref = DeviceFrame(f)
            ctx.postfilter_frame_dev(ref)
            want = ref.outputs_numpy()
            d = _fresh_device_frame(f)
            st, m = _noalloc(d)
            assert (st, m) == (abi.OK, 0), abi.MESSAGES.get(m)
            got = d.outputs_numpy()
            for k, (g, r) in enumerate(zip(got, want)):
                assert np.array_equal(g, r), f"seed {seed} plane {k} differs"
    finally:
        ctx.close()


def test_noalloc_rejects_frames_beyond_its_scratch():
    f = synth.make_frame(synth.CONFIG1, synth.seed_for(1, 0))  # 4K needs ~50 MB of intermediates
    d = DeviceFrame(f)
    st, m = _noalloc(d)
    assert st == abi.LIMIT_EXCEEDED and m == abi.MSG["SCRATCH_LIMIT"]


def test_noalloc_reports_data_errors_like_the_context_entry_point():
    f = synth.make_small(33, 200, 136, 10)
    f.planes[0][9, 9] = 4000  # above 10-bit
    st, m = _noalloc(DeviceFrame(f))
    assert st == abi.INVALID_DATA and m == abi.MSG["DB_SAMPLE"]
