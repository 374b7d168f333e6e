"""Parity of the CUDA path (through the C ABI) with the reference's proto/interp.py: against its golden fixtures
directly, and against the oracle (its CPU restatement) on further seeded inputs, settings, sizes and layouts.

Bar: every intermediate vector field, SAD, the scene-cut mean and every whole-frame decision bit-exact; output pixels
within TOL = 1 level per channel (the kernels are designed to be byte-exact, which the golden tests assert)."""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import workloads
from golden_io import golden, scene_inputs, scene_names, sha, times
from gpu_util import assert_estimate_equal, decision, frame_diff, new_out, run_gpu, to_dev

pytestmark = pytest.mark.gpu
TOL = 1
WHY = {None: 0, "cut": 1, "untrusted": 2}


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def check_against_oracle(prev, curr, ts, settings=None, order="rgba", pad=0, exact=True):
    s = settings or oracle.Settings()
    fs = fg.Settings(**{k: getattr(s, k) for k in oracle.Settings.__dataclass_fields__})
    tr, outs, unt, _, I = run_gpu(prev, curr, ts, fs, order, pad)
    est = oracle.estimate(prev, curr, settings=s, order=order)
    if not s.subpixel:
        est.pop("sub")
    assert_estimate_equal(tr, est)
    H, W = prev.shape[:2]
    for t, o, u in zip(ts, outs, unt):
        ref = oracle.synth(prev, curr, est, t, settings=s, order=order, trace=True)
        assert decision(tr["cut"], u, W, H, s.globalFallback) == ref["reason"], f"decision at t={t}"
        if not tr["cut"]:
            assert u == ref["untrusted"], f"untrusted count at t={t}"
        mx, mean, nd = frame_diff(o, ref["out"])
        assert mx <= TOL, f"t={t}: max diff {mx}, mean {mean}"
        if exact:
            assert nd == 0, f"t={t}: {nd} bytes differ (max {mx})"
    I.close()


@pytest.mark.parametrize("name", scene_names())
def test_golden_scene(name):
    """GPU vs the reference's own bytes (tests/golden, made by proto/interp.py)."""
    g = golden()
    p, c = scene_inputs(name)
    ts = times()
    tr, outs, unt, _, I = run_gpu(p, c, ts)
    n = len(tr["fields"])
    for l in range(n):
        assert np.array_equal(tr["fields"][l][0], g[f"{name}/search{l}"]), f"search level {l}"
        assert np.array_equal(tr["fields"][l][1], g[f"{name}/median{l}"]), f"median3 level {l}"
    for k in range(2):
        assert np.array_equal(tr["sub"][k], g[f"{name}/sub{k}"]), f"subpixel step {k}"
    assert np.array_equal(tr["sads"], g[f"{name}/sads"])
    assert tr["sad"] == float(g[f"{name}/sad"][0])
    if f"{name}/pf" in g:
        assert not tr["cut"] and np.array_equal(tr["pf"], g[f"{name}/pf"])
    else:
        assert tr["cut"]
    H, W = p.shape[:2]
    for k, (t, o, u) in enumerate(zip(ts, outs, unt)):
        assert WHY[decision(tr["cut"], u, W, H)] == int(g[f"{name}/why_t{k}"][0]), f"decision at t={t}"
        bgr = np.ascontiguousarray(o[..., [2, 1, 0]])
        if f"{name}/out_t{k}" in g:
            mx, mean, nd = frame_diff(bgr, g[f"{name}/out_t{k}"])
            assert nd == 0, f"t={t}: {nd} bytes differ, max {mx}, mean {mean}"
        else:
            assert np.array_equal(sha(bgr), g[f"{name}/outsha_t{k}"]), f"t={t}: frame digest differs"
        assert np.all(o[..., 3] == (p if t <= 0.5 else c)[..., 3])
    I.close()


@pytest.mark.parametrize("settings", [
    oracle.Settings(subpixel=False),
    oracle.Settings(flowScale=1),
    oracle.Settings(flowScale=4),
    oracle.Settings(searchRadius=1, searchRadiusTop=3),
    oracle.Settings(searchRadius=5, searchRadiusTop=12),
    oracle.Settings(searchRadius=12, searchRadiusTop=1),
    oracle.Settings(pyramidMinSide=16),
    oracle.Settings(trustLow=6.0, trustHigh=20.5, globalFallback=0.02),
    oracle.Settings(searchPenalty=0.3, hudBonus=0.0, smoothBonus=2.0),
    oracle.Settings(sceneCutSad=1.0),
], ids=["nosubpix", "fs1", "fs4", "r1t3", "r5t12", "r12t1", "minside16", "trust", "penalties", "cutlow"])
def test_settings_variants(settings):
    p, c, _ = workloads.flow_pair(208, 120, seed=21)
    check_against_oracle(p, c, [0.5, 0.25, float(np.float32(2 / 3))], settings)


@pytest.mark.parametrize("W,H", [(16, 16), (17, 16), (45, 33), (333, 211), (1001, 563)])
def test_odd_sizes(W, H):
    p, c = workloads.pan_pair(W, H, seed=W + H)
    check_against_oracle(p, c, [0.5, 0.75])


def test_bgra_order_and_padded_pitch():
    p, c = workloads.pan_pair(250, 140, seed=3)
    check_against_oracle(p, c, [0.5, 0.25], order="bgra", pad=13)


@pytest.mark.parametrize("kind", ["normal", "fresh", "cut"])
def test_1080p(kind):
    p, c, _ = workloads.flow_pair(1920, 1080, seed=100, kind=kind)
    check_against_oracle(p, c, [0.25, 0.5, 0.75])


def test_4k_pair():
    p, c, _ = workloads.flow_pair(3840, 2160, seed=4000)
    check_against_oracle(p, c, [0.25, 0.5, 0.75])


@pytest.mark.parametrize("n,W,H", [(96, 640, 360), (24, 1920, 1080)])
def test_flow_pairs_many(n, W, H):
    """A smooth-flow sequence, many pairs: smooth flows with scene cuts and fresh content mixed in (15 % each
    here, so that every batch has some), each pair checked stage by stage and at t = 1/4, 1/2, 3/4"""
    import workloads_gpu
    gen = torch.Generator(device="cuda")
    gen.manual_seed(10 ** 6 + n)
    d = workloads_gpu.flow_batch(n, W, H, gen, cut_frac=0.15, fresh_frac=0.15)
    kinds = d["kind"].tolist()
    for i in range(n):
        p, c = d["prev"][i].cpu().numpy(), d["curr"][i].cpu().numpy()
        check_against_oracle(p, c, [0.25, 0.5, 0.75])
    if n >= 24:
        assert 1 in kinds and 2 in kinds and 0 in kinds, kinds


def test_8k_pair():
    """7680x4320: six pyramid levels, the multi-CTA median3 on levels 2 and 1, the widest histograms (+-372 bins)"""
    import workloads_gpu   # the CPU generator takes minutes at this size; the GPU one the same kind of content
    gen = torch.Generator(device="cuda")
    gen.manual_seed(8000)
    d = workloads_gpu.flow_batch(1, 7680, 4320, gen)
    p, c = d["prev"][0].cpu().numpy(), d["curr"][0].cpu().numpy()
    check_against_oracle(p, c, [0.25, 0.5])


def test_hard_cut_and_repeat_determinism():
    """A scene cut then a normal pair on the same interpolator: state resets between estimates (histograms,
    counters), and the same pair twice gives identical bytes."""
    I = fg.Interpolator()
    a1, c1 = workloads.contrast_pair(320, 192, seed=9, kind="cut")
    a2, c2, _ = workloads.flow_pair(320, 192, seed=10)
    assert I.init(320, 192, fg.VK_R8G8B8A8_UNORM)
    res = []
    for a, c in ((a1, c1), (a2, c2), (a2, c2)):
        da, dc = to_dev(a), to_dev(c)
        o = new_out(da)
        I.begin_frame()
        assert I.record(da, dc, o, 0.5)
        torch.cuda.synchronize()
        res.append(o.cpu().numpy())
    assert np.array_equal(res[0], a1)   # cut: the nearer frame (prev at t = 0.5)
    assert np.array_equal(res[1], res[2])
    est = oracle.estimate(a2, c2, trace=False)
    assert np.array_equal(res[1], oracle.synth(a2, c2, est, 0.5)[0])
    I.close()


def test_record_refusals():
    """gpu/framegen.h:532-549: false and nothing recorded for t outside (0, 1), no estimate, other frames, ring
    overflow, a frame whose plane spans more than 2^34 bytes; beginFrame() resets the rings."""
    p, c = workloads.pan_pair(64, 48, seed=1)
    I = fg.Interpolator()
    assert I.init(64, 48, fg.VK_R8G8B8A8_UNORM)
    a, cc = to_dev(p), to_dev(c)
    o = new_out(a)
    before = o.clone()
    assert not I.record_synth(a, cc, o, 0.5)            # no estimate yet
    for t in (0.0, 1.0, -0.5, 1.5, float("nan")):
        assert not I.record(a, cc, o, t)
    big = fg.frame_of(a)
    big.pitch = 1 << 29                                  # 47 rows of 512 MiB: the plane spans more than 2^34 bytes
    assert not fg.lib().fg_record_estimate(I._h, fg._stream(None), fg.ctypes.byref(big), fg.ctypes.byref(big))
    I.begin_frame()
    assert I.record_estimate(a, cc)
    other = to_dev(c)
    assert not I.record_synth(other, cc, o, 0.5)        # not the estimate's frames
    torch.cuda.synchronize()
    assert torch.equal(o, before)
    for _ in range(fg.SET_RING - 1):
        assert I.record_estimate(a, cc)
    assert not I.record_estimate(a, cc)                  # ring overflow
    I.begin_frame()
    assert I.record_estimate(a, cc)
    for _ in range(fg.SET_RING):
        assert I.record_synth(a, cc, o, 0.5)
    assert not I.record_synth(a, cc, o, 0.5)
    I.close()


def test_profiling_timings():
    p, c, _ = workloads.flow_pair(640, 360, seed=2)
    I = fg.Interpolator()
    assert I.init(640, 360, fg.VK_R8G8B8A8_UNORM) and I.set_profiling(True)
    a, cc = to_dev(p), to_dev(c)
    o = new_out(a)
    assert I.record_estimate(a, cc)
    for t in (0.25, 0.5, 0.75):
        assert I.record_synth(a, cc, o, t)
    tm = I.read_timings()
    names = [n for n, _ in tm]
    assert names[:2] == ["luma", "pyramid"] and "subpixel" in names and "pixel field" in names
    assert names.count("synth") == 3 and names.count("fallback") == 3
    assert sum(ns for _, ns in tm) > 0
    # the pacer's cost-guard inputs from the same profile (gpu/pacing.h:869-871)
    c = I.read_costs()
    est_ns = sum(ns for n, ns in tm if n in ("luma", "pyramid", "subpixel", "pixel field") or n.startswith("level "))
    syn_ns = sum(ns for n, ns in tm if n in ("synth", "fallback"))
    assert c["synths"] == 3 and abs(c["estimate_ms"] - est_ns * 1e-6) < 1e-6 and abs(c["synth_ms"] - syn_ns * 1e-6 / 3) < 1e-6
    assert I.read_costs()["seq"] == c["seq"], "same profile, same sequence number"
    assert I.record_estimate(a, cc)
    assert I.read_costs()["seq"] == c["seq"] + 1 and I.read_costs()["synths"] == 0
    I.close()


def test_debug_maps_and_counters():
    p, c, _ = workloads.flow_pair(320, 180, seed=31, kind="fresh")
    tr, outs, unt, emaps, I = run_gpu(p, c, [0.25, 0.5], capture=True)
    est = oracle.estimate(p, c)
    for k, t in enumerate([0.25, 0.5]):
        ref = oracle.synth(p, c, est, t, trace=True)
        assert np.array_equal(emaps[k], ref["e"])
        assert unt[k] == ref["untrusted"]
    l = I.debug_map_layout()
    assert (l.W, l.H, l.fw, l.fh, l.bw, l.bh, l.fscale, l.eStride) == (320, 180, 160, 90, 20, 12, 2, 80)
    assert I.debug_sad_blocks() == 240
    assert tr["sadSum256"] == int(np.rint(est["sads"].astype(np.float64) * 256).sum())
    I.close()


def test_cuda_graph_capture():
    """Records are plain launches: estimate + 3 synths captured in a CUDA graph replay to the eager bytes."""
    p, c, _ = workloads.flow_pair(640, 360, seed=5)
    I = fg.Interpolator()
    assert I.init(640, 360, fg.VK_R8G8B8A8_UNORM)
    a, cc = to_dev(p), to_dev(c)
    outs = [new_out(a) for _ in range(3)]
    ts = (0.25, 0.5, 0.75)
    I.begin_frame()
    assert I.record_estimate(a, cc)
    for o, t in zip(outs, ts):
        assert I.record_synth(a, cc, o, t)
    torch.cuda.synchronize()
    eager = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        I.begin_frame()
        assert I.record_estimate(a, cc, stream=s)
        for o, t in zip(outs, ts):
            assert I.record_synth(a, cc, o, t, stream=s)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for o, e in zip(outs, eager):
        assert torch.equal(o, e)
    del g
    I.close()
