"""Motion blur (recordSynthBlur, fg_record_synth_blur) on the GPU against the oracle (oracle.synth_blur: the
sub-frames are the oracle's syntheses, whose parity with proto/interp.py the other test files establish).

Bar: byte-exact. Cases follow the reference's own check (gpu/blurtest.cpp:757-806): N = 2..8, the windows [.5, 1],
[.25, .75], [0, 1], [.1, .4], [.6, .9], even and Gaussian weights, the scene cut forced, the whole-frame flick forced
on every sample and on some samples only (the fix-up pass); the single-instant cases, refusals, a CUDA graph, and at
4K (too large for the oracle in seconds) the size-independent identity blur == the rounded mean of recordSynth
outputs at the sample times. The other formats (Rgb10, RgbaF16 linear and encoded, Nv12, P010) against
oracle.synth_blur_fmt, with the cut and the flick forced.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import workloads
from gpu_util import ORDER_VK, new_out, to_dev

pytestmark = pytest.mark.gpu
WINDOWS = [(0.5, 1.0), (0.25, 0.75), (0.0, 1.0), (0.1, 0.4), (0.6, 0.9)]


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def to_fg(s):
    return fg.Settings(**{k: getattr(s, k) for k in oracle.Settings.__dataclass_fields__})


class Ctx:
    """one Interpolator with the pair's estimate recorded"""

    def __init__(self, prev, curr, s=None, order="rgba", pad=0):
        self.s = s or oracle.Settings()
        self.prev, self.curr, self.order, self.pad = prev, curr, order, pad
        H, W = prev.shape[:2]
        self.I = fg.Interpolator()
        assert self.I.init(W, H, ORDER_VK[order], settings=to_fg(self.s)), self.I.init_error()
        self.a, self.c = to_dev(prev, pad), to_dev(curr, pad)
        self.I.begin_frame()
        assert self.I.record_estimate(self.a, self.c)
        self.est = oracle.estimate(prev, curr, settings=self.s, order=order, trace=False)
        self.subs = {}

    def blur(self, t0, t1, n, gaussian, stream=None):
        fs = to_fg(self.s)
        fs.blurSamples, fs.blurWeights = n, int(gaussian)
        assert self.I.set_settings(fs)
        self.I.begin_frame()
        o = new_out(self.a, self.pad)
        ok = self.I.record_synth_blur(self.a, self.c, o, t0, t1, stream=stream)
        torch.cuda.synchronize()
        return ok, o.cpu().numpy()

    def synth(self, t):
        self.I.begin_frame()
        o = new_out(self.a, self.pad)
        assert self.I.record_synth(self.a, self.c, o, t)
        torch.cuda.synchronize()
        return o.cpu().numpy()

    def want(self, t0, t1, n, gaussian):
        """the oracle's blur, its syntheses cached by time"""
        times, q = oracle.blur_plan(n, gaussian, t0, t1)
        acc = np.zeros(self.prev.shape, np.int64)
        for tk, qk in zip(times.tolist(), q):
            if tk <= 0:
                f = self.prev
            elif tk >= 1:
                f = self.curr
            else:
                if tk not in self.subs:
                    self.subs[tk] = oracle.synth(self.prev, self.curr, self.est, tk, self.s, self.order)[0]
                f = self.subs[tk]
            acc += qk * f.astype(np.int64)
        return ((acc + 32768) >> 16).astype(np.uint8)

    def close(self):
        self.I.close()


def check_all(ctx, ns, label):
    bad = []
    for n in ns:
        for t0, t1 in WINDOWS:
            for gaussian in (False, True):
                ok, got = ctx.blur(t0, t1, n, gaussian)
                assert ok, ctx.I.last_error()
                want = ctx.want(t0, t1, n, gaussian)
                if not np.array_equal(got, want):
                    d = np.abs(got.astype(int) - want.astype(int))
                    bad.append((n, t0, t1, gaussian, int(d.max()), int((d > 0).sum())))
    assert not bad, f"{label}: {bad}"


@pytest.mark.parametrize("size,order,pad", [((320, 180), "rgba", 0), ((203, 117), "bgra", 3)])
def test_blur_matches_oracle(size, order, pad):
    W, H = size
    p, c, _ = workloads.flow_pair(W, H, seed=11)
    ctx = Ctx(p, c, order=order, pad=pad)
    check_all(ctx, range(2, 9), f"{W}x{H} {order}")
    ctx.close()


def flick_threshold(prev, curr, s, n, t0, t1):
    """a globalFallback that flicks some, not all, of the window's samples (the median untrusted count)"""
    est = oracle.estimate(prev, curr, settings=s, trace=False)
    times, _ = oracle.blur_plan(n, False, t0, t1)
    cnt = sorted(oracle.synth(prev, curr, est, float(t), s, trace=True)["untrusted"] for t in times.tolist())
    H, W = prev.shape[:2]
    lo, hi = cnt[0], cnt[-1]
    assert hi > lo, "the samples' untrusted counts do not spread"
    mid = cnt[len(cnt) // 2]
    return float(np.float32((mid - 0.5) / (W * H))) if mid > lo else float(np.float32((lo + 0.5) / (W * H)))


@pytest.mark.parametrize("variant", ["cut", "flick all", "flick some"])
def test_blur_fallbacks(variant):
    p, c, _ = workloads.flow_pair(256, 144, seed=5)
    if variant == "cut":
        s = oracle.Settings(sceneCutSad=0.5)
    elif variant == "flick all":
        s = oracle.Settings(globalFallback=0.0005)
    else:
        s = oracle.Settings(globalFallback=flick_threshold(p, c, oracle.Settings(), 7, 0.0, 1.0))
    ctx = Ctx(p, c, s)
    if variant == "cut":
        assert ctx.est["cut"]
    check_all(ctx, (3, 4, 7), variant)
    ctx.close()


def test_blur_instants_and_refusals():
    p, c, _ = workloads.flow_pair(160, 96, seed=3)
    ctx = Ctx(p, c)
    s30 = ctx.synth(0.3)
    assert np.array_equal(ctx.blur(0.3, 0.3, 8, True)[1], s30)      # t0 == t1: recordSynth(t1)
    assert np.array_equal(ctx.blur(0.1, 0.3, 1, True)[1], s30)      # blur off: the window's end
    assert np.array_equal(ctx.blur(0.1, 0.3, 0, False)[1], s30)
    assert np.array_equal(ctx.blur(1.0, 1.0, 4, False)[1], c)       # real-frame instants
    assert np.array_equal(ctx.blur(0.0, 0.0, 4, False)[1], p)
    assert np.array_equal(ctx.blur(0.0, 1.0, 1, False)[1], c)
    for t0, t1 in [(0.6, 0.5), (-0.1, 0.5), (0.2, 1.5), (float("nan"), 0.5), (0.2, float("nan"))]:
        ok, o = ctx.blur(t0, t1, 4, False)
        assert not ok and (o == 7).all(), (t0, t1)
    # prev / curr not the estimate's frames
    o = new_out(ctx.a)
    assert not ctx.I.record_synth_blur(ctx.c, ctx.a, o, 0.2, 0.8)
    ctx.close()
    # no estimate yet
    I = fg.Interpolator()
    fs = fg.Settings()
    fs.blurSamples = 4
    assert I.init(160, 96, fg.VK_R8G8B8A8_UNORM, settings=fs)
    a = to_dev(p)
    assert not I.record_synth_blur(a, a, new_out(a), 0.2, 0.8)
    I.close()


BLUR_CASES = [(2, 0.0, 1.0, False), (3, 0.25, 0.75, True), (4, 0.1, 0.4, True), (5, 0.6, 0.9, False),
              (8, 0.0, 1.0, True)]


@pytest.mark.parametrize("variant", ["default", "cut", "flick"])
@pytest.mark.parametrize("name", ["rgb10_argb", "f16_linear", "f16_encoded", "nv12_709_limited", "p010_2020_limited"])
def test_blur_formats_match_oracle(name, variant):
    """the other formats (odd size: ragged chroma), byte for byte against oracle.synth_blur_fmt: integer formats'
    codes averaged with the 2^-16 weights, RgbaF16 float32 sums in sample order rounded to half; with the scene cut
    forced and with every synthesis flicked (the fix-up pass)"""
    from test_formats_gpu import SPEC, new_out as fmt_out, to_dev as fmt_dev, to_host
    _, vk, spec, conv, extra = SPEC[name]
    p8, c8, _ = workloads.flow_pair(203, 117, seed=17)
    a, c = conv(p8), conv(c8)
    s = {"default": oracle.Settings(), "cut": oracle.Settings(sceneCutSad=0.5),
         "flick": oracle.Settings(globalFallback=0.0005)}[variant]
    fs = to_fg(s)
    I = fg.Interpolator()
    assert I.init(203, 117, vk, settings=fs, **extra), I.init_error()
    da, dc = fmt_dev(a), fmt_dev(c)
    I.begin_frame()
    assert I.record_estimate(da, dc)
    est = oracle.estimate_fmt(a, c, spec, settings=s, trace=False)
    assert bool(est["cut"]) == (variant == "cut")
    bad = []
    for n, t0, t1, g in BLUR_CASES:
        fs.blurSamples, fs.blurWeights = n, int(g)
        assert I.set_settings(fs)
        I.begin_frame()
        o = fmt_out(da)
        assert I.record_synth_blur(da, dc, o, t0, t1), (n, t0, t1)
        torch.cuda.synchronize()
        got, want = to_host(o, a), oracle.synth_blur_fmt(a, c, est, t0, t1, n, g, spec, s)
        planes = zip(got, want) if isinstance(got, tuple) else [(got, want)]
        for gp, wp in planes:
            if not np.array_equal(gp.view(np.uint8), wp.view(np.uint8)):
                bad.append((n, t0, t1, g, int(np.count_nonzero(gp != wp))))
    assert not bad, f"{name} {variant}: {bad}"
    I.close()


def test_blur_graph_capture_and_profiling():
    p, c, _ = workloads.flow_pair(320, 180, seed=21)
    ctx = Ctx(p, c)
    ok, eager = ctx.blur(0.2, 0.9, 6, True)
    assert ok and np.array_equal(eager, ctx.want(0.2, 0.9, 6, True))
    s = torch.cuda.Stream()
    o = new_out(ctx.a)
    with torch.cuda.stream(s):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            ctx.I.begin_frame()
            assert ctx.I.record_synth_blur(ctx.a, ctx.c, o, 0.2, 0.9, stream=s)
    o.fill_(3)
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(o.cpu().numpy(), eager)
    del g
    assert ctx.I.set_profiling(True)
    ctx.blur(0.2, 0.9, 6, True)
    names = [name for name, _ in ctx.I.read_timings()]
    assert names[-2:] == ["blur samples", "blur blend"], names   # 8-bit RGBA: the stored sub-frames and their blend
    c = ctx.I.read_costs()
    assert c["synths"] == 1 and c["synth_ms"] > 0, c
    ctx.close()


def test_blur_4k_is_the_rounded_mean_of_the_syntheses():
    """3840x2160: with even weights and N a power of two, blur == (sum of recordSynth(t_k) + N/2) / N exactly"""
    p, c, _ = workloads.flow_pair(3840, 2160, seed=1)
    I = fg.Interpolator()
    assert I.init(3840, 2160, fg.VK_R8G8B8A8_UNORM), I.init_error()
    a, cc = to_dev(p), to_dev(c)
    I.begin_frame()
    assert I.record_estimate(a, cc)
    for n, (t0, t1) in [(2, (0.0, 1.0)), (8, (0.0, 1.0)), (4, (0.25, 0.75))]:
        times, q = oracle.blur_plan(n, False, t0, t1)
        acc = torch.zeros((2160, 3840, 4), dtype=torch.int32, device="cuda")
        o = torch.empty_like(a)
        for t in times.tolist():
            I.begin_frame()
            assert I.record_synth(a, cc, o, t)
            acc += o.int()
        want = ((acc + n // 2) // n).to(torch.uint8)
        fs = fg.Settings()
        fs.blurSamples, fs.blurWeights = n, 0
        assert I.set_settings(fs)
        I.begin_frame()
        assert I.record_synth_blur(a, cc, o, t0, t1)
        torch.cuda.synchronize()
        assert torch.equal(o, want), f"N={n} [{t0},{t1}]: {int((o != want).sum())} bytes differ"
    I.close()


def test_blur_fused_and_stored_sub_frames_agree_8k():
    """7680x4320 (a 4K pair tiled 2 x 2): 16 samples would take 2.1 GB of sub-frames, past the library's 1 GiB cap,
    so the fused kernel (k_synth_blur_t, main and fix-up passes) runs; 4 samples fit and run as stored sub-frames and
    their blend. Both equal the rounded mean of recordSynth at the sample times (even weights, N a power of two), and
    the profile names show which path ran."""
    p, c, _ = workloads.flow_pair(3840, 2160, seed=3)
    p, c = np.tile(p, (2, 2, 1)), np.tile(c, (2, 2, 1))
    W, H = 7680, 4320
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM), I.init_error()
    a, cc = to_dev(p), to_dev(c)
    I.begin_frame()
    assert I.record_estimate(a, cc)
    o = torch.empty_like(a)
    for n, (t0, t1), names in [(16, (0.0, 1.0), ["blur resolve", "blur fixup"]),
                               (4, (0.125, 0.875), ["blur samples", "blur blend"])]:
        times, _ = oracle.blur_plan(n, False, t0, t1)
        acc = torch.zeros((H, W, 4), dtype=torch.int32, device="cuda")
        for t in times.tolist():
            I.begin_frame()
            assert I.record_synth(a, cc, o, t)
            acc += o.int()
        want = ((acc + n // 2) // n).to(torch.uint8)
        del acc
        fs = fg.Settings()
        fs.blurSamples, fs.blurWeights = n, 0
        assert I.set_settings(fs)
        assert I.set_profiling(True)
        I.begin_frame()
        assert I.record_synth_blur(a, cc, o, t0, t1)
        torch.cuda.synchronize()
        got = [name for name, _ in I.read_timings()]
        assert I.set_profiling(False)
        assert got[-2:] == names, (n, got)
        assert torch.equal(o, want), f"N={n} [{t0},{t1}]: {int((o != want).sum())} bytes differ"
    I.close()
