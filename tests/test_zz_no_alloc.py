"""fg_record_synth_noalloc, the synthesis entry point that allocates nothing.

It exists for hosts that cannot call the CUDA allocator while they generate frames: code running inside another
program's frame callback under that program's memory budget, a presentation thread that must never block on
cudaMalloc / cudaFree (both can synchronise the device), or a plugin that is given buffers but no allocator. Such a
host keeps the pair's per-pixel field and scene-cut decision from an earlier estimate and passes them in together with
the frames and the output; the library's own scratch for this path is a fixed array inside the library.

The test computes one estimate and a synth through the usual Interpolator entry points, then feeds the same frames,
the estimate's field and its cut decision to fg_record_synth_noalloc twice in a row, and checks that both calls give
the usual entry point's frame, bit for bit (both run the same synthesis kernel on the same field). The second call
must not change the device's free memory: after the first call on a device has placed the library's fixed array,
nothing further is allocated. It also checks that a frame too large for the fixed scratch is refused with a clear
message and that nothing is launched for it (the stream stays clean). This file is collected last so that a failure
here cannot hide other tests' results.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import workloads
from gpu_util import frame_diff, new_out, to_dev

pytestmark = pytest.mark.gpu
TOL = 1


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def reference_synth(prev, curr, t, settings):
    """The usual path: Interpolator estimate + synth; returns (frame, per-pixel field on the device, cut decision)."""
    H, W = prev.shape[:2]
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=settings), I.init_error()
    a, c = to_dev(prev), to_dev(curr)
    o = new_out(a)
    I.begin_frame()
    assert I.record_estimate(a, c)
    assert I.record_synth(a, c, o, t)
    tr = fg.read_trace(I)
    torch.cuda.synchronize()
    field = torch.from_numpy(np.ascontiguousarray(tr["pf"])).cuda()
    I.close()
    return o.cpu().numpy(), field, tr["cut"]


@pytest.mark.parametrize("kind,t", [("normal", 0.5), ("normal", 0.25), ("fresh", float(np.float32(2 / 3))),
                                    ("cut", 0.75)])
def test_noalloc_matches_synth_twice(kind, t):
    if kind == "cut":
        prev, curr = workloads.contrast_pair(320, 192, seed=3, kind="cut")
    else:
        prev, curr, _ = workloads.flow_pair(640, 360, seed=77, kind=kind)
    settings = fg.Settings()
    ref, field, cut = reference_synth(prev, curr, t, settings)
    a, c = to_dev(prev), to_dev(curr)
    outs = [new_out(a) for _ in range(2)]
    for call in range(2):   # two calls in a row on the shared scratch
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        ok, err = fg.record_synth_noalloc(a, c, outs[call], field, cut, t, settings)
        assert ok, err
        torch.cuda.synchronize()
        if call == 1:   # the first call may place the fixed array; the next one allocates nothing at all
            assert torch.cuda.mem_get_info()[0] == free_before, "the second call changed the device's free memory"
        got = outs[call].cpu().numpy()
        mx, mean, nd = frame_diff(got, ref)
        assert mx <= TOL and nd == 0, f"call {call}: max diff {mx}, mean {mean}, {nd} bytes differ"


def test_noalloc_refuses_frames_beyond_its_scratch():
    small = torch.zeros((16, 16, 4), dtype=torch.uint8, device="cuda")
    field = torch.zeros((8, 8, 2), dtype=torch.float32, device="cuda")
    # 4096 x 3080 at flowScale 2 needs 2048 x 1540 = 3,153,920 flow pixels, above the 3,145,728 the scratch holds; the
    # size is checked before anything else, so these small stand-in buffers are never touched
    err = fg.ctypes.c_char_p()
    ok = fg.lib().fg_record_synth_noalloc(fg._stream(None), fg.VK_R8G8B8A8_UNORM, 4096, 3080,
                                          fg.ctypes.byref(fg.frame_of(small)), fg.ctypes.byref(fg.frame_of(small)),
                                          fg.ctypes.byref(fg.frame_of(small)), field.data_ptr(), 0, 0.5,
                                          fg.ctypes.byref(fg.Settings().to_c()), fg.ctypes.byref(err))
    assert ok == 0 and b"no-allocation scratch" in err.value
    # t outside (0, 1) is refused too, with its own reason
    ok, msg = fg.record_synth_noalloc(small, small, small, field, 0, 1.0)
    assert not ok and "outside" in msg
    # nothing was launched for either call: the device is idle, and a valid call right after succeeds (the entry point
    # reads cudaGetLastError after its first launch, so an error left pending by the refused calls would fail it)
    torch.cuda.synchronize()
    prev, curr = workloads.pan_pair(32, 32, seed=5)
    a, c = to_dev(prev), to_dev(curr)
    f16 = torch.zeros((16, 16, 2), dtype=torch.float32, device="cuda")
    ok, msg = fg.record_synth_noalloc(a, c, new_out(a), f16, 0, 0.5)
    assert ok, msg
    torch.cuda.synchronize()
