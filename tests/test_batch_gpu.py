"""framegen::Batch (fg_batch_*): many frame pairs of mixed sizes, formats and multipliers recorded together, the
8-bit RGBA syntheses of all slots in one persistent launch, the estimates forked over streams or merged into one launch
per pass for all slots. Every slot's outputs must equal, byte for byte, those of a standalone Interpolator on the same
pair (whose parity with the oracle the other test files establish), for every launch shape the autotuner chooses from,
after tune(), and through a CUDA graph.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import workloads

pytestmark = pytest.mark.gpu

VK = {"rgba8": fg.VK_R8G8B8A8_UNORM, "rgb10": fg.VK_A2B10G10R10_UNORM, "nv12": fg.VK_R8_UNORM,
      "p010": fg.VK_R16_UNORM}


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def convert(fmt, rgba):
    if fmt == "rgba8":
        return rgba
    if fmt == "rgb10":
        return workloads.to_rgb10(rgba)
    return workloads.to_yuv(rgba, 8 if fmt == "nv12" else 10, "bt709")


def dev(frame):
    def plane(a):
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        elif a.dtype == np.uint16:
            a = a.view(np.int16)
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return tuple(plane(a) for a in frame) if isinstance(frame, tuple) else plane(frame)


def like(d):
    return tuple(torch.zeros_like(x) for x in d) if isinstance(d, tuple) else torch.zeros_like(d)


def host(d):
    return tuple(x.cpu().numpy() for x in d) if isinstance(d, tuple) else d.cpu().numpy()


def same(a, b):
    if isinstance(a, tuple):
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return np.array_equal(a, b)


def c3_slots(scale=4, n=64):
    """the mixed batch's structure at 1/scale resolution: sizes 1280x720 / 1920x1080 / 2560x1440 / 3840x2160 in ratio
    8:4:2:1 (34 / 17 / 9 / 4 of 64), formats cycling Rgba8 / Rgb10 / Nv12 / P010, multipliers cycling 2 / 3 / 4"""
    sizes = [(1280, 720)] * 34 + [(1920, 1080)] * 17 + [(2560, 1440)] * 9 + [(3840, 2160)] * 4
    fmts = ["rgba8", "rgb10", "nv12", "p010"]
    out = []
    for i, (w, h) in enumerate(sizes[:n]):
        out.append((w // scale, h // scale, fmts[i % 4], 2 + i % 3))
    return out


def build_case(slots, seed=0):
    B = fg.Batch()
    prev, curr, outs, ref = [], [], [], []
    for i, (w, h, fmt, m) in enumerate(slots):
        assert B.add(w, h, VK[fmt], multiplier=m) == i, B.error()
        p, c, _ = workloads.flow_pair(w, h, seed=seed + i)
        prev.append(dev(convert(fmt, p)))
        curr.append(dev(convert(fmt, c)))
        for _ in range(m - 1):
            outs.append(like(prev[-1]))
    # the standalone references
    for i, (w, h, fmt, m) in enumerate(slots):
        I = fg.Interpolator()
        assert I.init(w, h, VK[fmt]), I.init_error()
        I.begin_frame()
        assert I.record_estimate(prev[i], curr[i])
        for t in fg.Batch.times(m):
            o = like(prev[i])
            assert I.record_synth(prev[i], curr[i], o, t)
            ref.append(o)
        torch.cuda.synchronize()
        I.close()
    return B, prev, curr, outs, [host(r) for r in ref]


@pytest.fixture(scope="module")
def case():
    return build_case(c3_slots(scale=8, n=24))


@pytest.mark.parametrize("shape", [(0, 0, 1), (3, 1, 1), (0, 0, 4), (2, 0, 8), (2, 1, 8), (3, 0, 8), (3, 1, 8),
                                   (0, 0, 1, 1), (3, 1, 1, 1), (0, 0, 8, 1), (3, 1, 8, 1), (0, 0, 8, 4), (3, 1, 8, 8)])
def test_batch_matches_standalone(case, shape):
    B, prev, curr, outs, ref = case
    assert B.set_shape(*shape)
    for o in outs:   # poison the outputs
        for x in (o if isinstance(o, tuple) else (o,)):
            x.fill_(7)
    for _ in range(2):   # twice: the counters and the work list start from scratch each record
        assert B.record(prev, curr, outs), B.error()
        torch.cuda.synchronize()
        bad = [j for j, (o, r) in enumerate(zip(outs, ref)) if not same(host(o), r)]
        assert not bad, f"shape {shape}: outputs {bad} differ"


def test_tune_then_record(case):
    B, prev, curr, outs, ref = case
    best = B.tune(prev, curr, outs, reps=2)
    assert 0 <= best < 16
    assert B.record(prev, curr, outs)
    torch.cuda.synchronize()
    assert all(same(host(o), r) for o, r in zip(outs, ref))


@pytest.mark.parametrize("shape", [(3, 1, 8), (3, 1, 8, 1), (3, 1, 8, 4)])
def test_batch_graph_capture(case, shape):
    B, prev, curr, outs, ref = case
    assert B.set_shape(*shape)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        assert B.record(prev, curr, outs, stream=s)   # warm (parameter upload ring, lazy module loads)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            assert B.record(prev, curr, outs, stream=s)
    for o in outs:
        for x in (o if isinstance(o, tuple) else (o,)):
            x.fill_(3)
    g.replay()
    torch.cuda.synchronize()
    assert all(same(host(o), r) for o, r in zip(outs, ref))
    del g


def test_merged_estimates_mixed_settings():
    """merged estimates over slots whose passes take different kernel variants in the same launch step: radii 1 / 3 /
    6 / 9 (the runtime-radius search), subpixel off (the scene-cut mean instead of the sub-pixel pass), flowScale 1 /
    4, sizes from 96 x 200 to 1280 x 720 and more slots than one merged launch takes (kMergeMax 48)"""
    kinds = [dict(searchRadius=1), dict(searchRadius=3, searchRadiusTop=4), dict(searchRadius=6),
             dict(searchRadius=9, searchRadiusTop=9), dict(subpixel=False), dict(flowScale=1), dict(flowScale=4), {}]
    sizes = [(128, 96), (160, 90), (320, 180), (640, 360), (1280, 720), (96, 200)]
    B = fg.Batch()
    prev, curr, outs, ref = [], [], [], []
    for i in range(52):
        w, h = sizes[i % len(sizes)]
        fmt = ["rgba8", "rgb10", "nv12", "p010"][i % 4]
        st = fg.Settings(**kinds[i % len(kinds)])
        assert B.add(w, h, VK[fmt], multiplier=2, settings=st) == i, B.error()
        p, c, _ = workloads.flow_pair(w, h, seed=500 + i)
        prev.append(dev(convert(fmt, p)))
        curr.append(dev(convert(fmt, c)))
        outs.append(like(prev[-1]))
        I = fg.Interpolator()
        assert I.init(w, h, VK[fmt], settings=st), I.init_error()
        I.begin_frame()
        assert I.record_estimate(prev[i], curr[i])
        o = like(prev[i])
        assert I.record_synth(prev[i], curr[i], o, 0.5)
        torch.cuda.synchronize()
        ref.append(host(o))
        I.close()
    for shape in [(0, 0, 1, 1), (3, 1, 8, 1), (0, 0, 8, 3)]:
        assert B.set_shape(*shape)
        assert B.shape() == shape
        for o in outs:
            for x in (o if isinstance(o, tuple) else (o,)):
                x.fill_(7)
        assert B.record(prev, curr, outs), B.error()
        torch.cuda.synchronize()
        bad = [j for j, (o, r) in enumerate(zip(outs, ref)) if not same(host(o), r)]
        assert not bad, f"shape {shape}: outputs {bad} differ"


@pytest.mark.parametrize("shape", [(3, 1, 8), (0, 0, 1), (3, 1, 1, 1), (0, 0, 8, 2)])
def test_batch_whole_frame_fallbacks(shape):
    """every synthesis flicks (a tiny globalFallback with a steep trust ramp): the batch's fallback launches must see
    the complete untrusted counts of their syntheses and copy the nearer frame, as standalone Interpolators do"""
    st = fg.Settings(globalFallback=1e-6, trustLow=0.0, trustHigh=1.0)
    assert fg.validate(st)
    slots = [(160, 96, "rgba8", 3), (320, 180, "rgb10", 2), (200, 120, "nv12", 4), (128, 96, "p010", 2),
             (320, 180, "rgba8", 4), (96, 64, "rgba8", 2)]
    B = fg.Batch()
    prev, curr, outs, ref, near = [], [], [], [], []
    for i, (w, h, fmt, m) in enumerate(slots):
        assert B.add(w, h, VK[fmt], multiplier=m, settings=st) == i, B.error()
        p, c, _ = workloads.flow_pair(w, h, seed=900 + i)
        prev.append(dev(convert(fmt, p)))
        curr.append(dev(convert(fmt, c)))
        I = fg.Interpolator()
        assert I.init(w, h, VK[fmt], settings=st), I.init_error()
        I.begin_frame()
        assert I.record_estimate(prev[i], curr[i])
        for t in fg.Batch.times(m):
            outs.append(like(prev[i]))
            o = like(prev[i])
            assert I.record_synth(prev[i], curr[i], o, t)
            torch.cuda.synchronize()
            ref.append(host(o))
            near.append(host(curr[i] if t > 0.5 else prev[i]))
        I.close()
    assert sum(same(r, n) for r, n in zip(ref, near)) >= len(ref) // 2, "the settings should make the syntheses flick"
    assert B.set_shape(*shape)
    for _ in range(2):
        for o in outs:
            for x in (o if isinstance(o, tuple) else (o,)):
                x.fill_(7)
        assert B.record(prev, curr, outs), B.error()
        torch.cuda.synchronize()
        bad = [j for j, (o, r) in enumerate(zip(outs, ref)) if not same(host(o), r)]
        assert not bad, f"shape {shape}: outputs {bad} differ"


@pytest.mark.parametrize("shape", [(3, 1, 8), (0, 0, 1), (3, 1, 1, 1)])
def test_batch_with_a_crosshair_slot(shape):
    """a CrosshairV2 slot in a batch synthesizes through recordSynth (tap rejection, paste-back) whatever the launch
    shape, next to plain slots: over a sequence of records (the implicit observe of each pair), its outputs equal a
    standalone Interpolator's on the same sequence"""
    from test_ui_v2_gpu import grain_scene, v2_settings
    W, H = 320, 192
    frames, _ = grain_scene(W, H, 10)
    st = v2_settings()
    dframes = [torch.from_numpy(f).cuda() for f in frames]
    B = fg.Batch()
    assert B.add(W, H, fg.VK_R8G8B8A8_UNORM, multiplier=2, settings=st) == 0, B.error()
    assert B.add(W, H, fg.VK_R8G8B8A8_UNORM, multiplier=2) == 1, B.error()
    assert B.set_shape(*shape)
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=st), I.init_error()
    outs = [torch.zeros_like(dframes[0]) for _ in range(2)]
    ref = torch.zeros_like(dframes[0])
    for k in range(1, len(frames)):
        assert B.record([dframes[k - 1], dframes[k - 1]], [dframes[k], dframes[k]], outs), B.error()
        I.begin_frame()
        assert I.record_estimate(dframes[k - 1], dframes[k])
        assert I.record_synth(dframes[k - 1], dframes[k], ref, 0.5)
        torch.cuda.synchronize()
        assert np.array_equal(outs[0].cpu().numpy(), ref.cpu().numpy()), f"record {k}: the CrosshairV2 slot differs"
    assert fg.read_ui(I, dframes[-1], st, W, H)["mask"].max() == 255, "the plus should be protected by the end"
    I.close()


def test_rgba8_slot_against_the_oracle():
    """one batched 8-bit RGBA slot straight against the oracle (interp.py's restatement)"""
    p, c, _ = workloads.flow_pair(320, 180, seed=99)
    B = fg.Batch()
    assert B.add(320, 180, fg.VK_R8G8B8A8_UNORM, multiplier=4) == 0
    outs = [torch.zeros((180, 320, 4), dtype=torch.uint8, device="cuda") for _ in range(3)]
    assert B.record([dev(p)], [dev(c)], outs)
    torch.cuda.synchronize()
    est = oracle.estimate(p, c)
    for o, t in zip(outs, fg.Batch.times(4)):
        ref, _ = oracle.synth(p, c, est, t)
        assert np.array_equal(o.cpu().numpy(), ref), t


def test_batch_refusals():
    B = fg.Batch()
    assert B.add(64, 48, fg.VK_R8G8B8A8_UNORM, multiplier=1) == -1 and "multiplier" in B.error()
    assert B.add(8, 8, fg.VK_R8G8B8A8_UNORM, multiplier=2) == -1
    assert B.add(64, 48, fg.VK_R8G8B8A8_UNORM, multiplier=2) == 0
    x = torch.zeros((48, 64, 4), dtype=torch.uint8, device="cuda")
    narrow = torch.zeros((48, 60, 4), dtype=torch.uint8, device="cuda")   # a pitch below the slot's 64 pixels
    assert not B.record([x], [x], [narrow])
    assert B.record([x], [x], [torch.zeros_like(x)])
