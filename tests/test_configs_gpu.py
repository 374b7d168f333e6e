"""The path's workload configurations at their stated sizes, on the GPU through the C ABI, each against the oracle.

  config 0  640x360 Rgba8 2x (t = 1/2): the panning value-noise pair with a moving sprite and a static HUD box;
  config 1  1920x1080 Rgba8 4x (t = 1/4, 1/2, 3/4), 500 pairs of the smooth-flow generator (5 % scene cuts, 5 % with
            20 % fresh content), generated on the device (workloads_gpu.flow_batch, seeded per batch of 10);
  config 2  3840x2160 RgbaF16 linear scRGB 3x (t = 1/3, 2/3): 16 of the 200 pairs of the HDR generator
            (workloads_gpu.hdr_pair; the oracle's float-format restatement takes ~2.5 s per pair on the host);
  config 3  the 64-pair mixed batch at full size (34 x 720p, 17 x 1080p, 9 x 1440p, 4 x 2160p; Rgba8 / Rgb10 / Nv12 /
            P010; 2x / 3x / 4x), every slot against a standalone Interpolator and every Rgba8 slot against the oracle.
Bar: outputs byte-identical (the tests print max and mean absolute difference and the bytes that differ), identical
whole-frame decisions and untrusted-pixel counts, identical per-pixel fields.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import workloads
import workloads_gpu
from gpu_util import assert_estimate_equal, decision

pytestmark = pytest.mark.gpu
TOL = 1


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


class Diff:
    """running max / mean absolute difference and count of differing bytes over many frames"""

    def __init__(self):
        self.mx, self.sum, self.n, self.nd, self.frames = 0, 0.0, 0, 0, 0

    def add(self, got, ref):
        d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
        self.mx = max(self.mx, int(d.max()))
        self.sum += float(d.sum())
        self.n += d.size
        self.nd += int(np.count_nonzero(d))
        self.frames += 1

    def __str__(self):
        return f"{self.frames} frames: max abs diff {self.mx}, mean {self.sum / max(self.n, 1):.3g}, {self.nd} bytes differ"


def run_pair(I, a, c, ts, cnt):
    """estimate + syntheses through the C ABI: (outputs on the host, trace, untrusted counts)"""
    I.begin_frame()
    assert I.record_estimate(a, c), I.last_error()
    tr = fg.read_trace(I)
    outs, unt = [], []
    for t in ts:
        o = torch.empty_like(a)
        assert I.record_synth(a, c, o, t), I.last_error()
        assert I.record_debug_counters(cnt)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        unt.append(int(cnt[0]))
    return outs, tr, unt


def check_against_oracle(p, c, outs, tr, unt, ts, diff, full_trace=False):
    H, W = p.shape[:2]
    est = oracle.estimate(p, c, trace=full_trace)
    if full_trace:
        assert_estimate_equal(tr, est)
    else:
        assert tr["cut"] == est["cut"] and tr["sad"] == est["sad"]
        if est["pf"] is not None:
            assert np.array_equal(tr["pf"], est["pf"]), "per-pixel field differs"
    for o, u, t in zip(outs, unt, ts):
        ref, why = oracle.synth(p, c, est, t)
        assert decision(tr["cut"], u, W, H) == why, f"decision at t={t}"
        diff.add(o, ref)


def test_config0_pan_640x360():
    p, c = workloads.pan_pair()
    I = fg.Interpolator()
    assert I.init(640, 360, fg.VK_R8G8B8A8_UNORM), I.init_error()
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    outs, tr, unt = run_pair(I, torch.from_numpy(p).cuda(), torch.from_numpy(c).cuda(), [0.5], cnt)
    d = Diff()
    check_against_oracle(p, c, outs, tr, unt, [0.5], d, full_trace=True)
    print("config 0:", d)
    assert d.mx <= TOL and d.nd == 0
    I.close()


def test_config1_500_pairs_1080p():
    ts = (0.25, 0.5, 0.75)
    I = fg.Interpolator()
    assert I.init(1920, 1080, fg.VK_R8G8B8A8_UNORM), I.init_error()
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    gen = torch.Generator(device="cuda")
    d = Diff()
    kinds = [0, 0, 0]
    for b in range(50):
        gen.manual_seed(1 * 10 ** 6 + b)
        batch = workloads_gpu.flow_batch(10, 1920, 1080, gen)
        for k in range(10):
            a, c = batch["prev"][k].contiguous(), batch["curr"][k].contiguous()
            kinds[int(batch["kind"][k])] += 1
            outs, tr, unt = run_pair(I, a, c, ts, cnt)
            check_against_oracle(a.cpu().numpy(), c.cpu().numpy(), outs, tr, unt, ts, d)
    I.close()
    print(f"config 1: 500 pairs ({kinds[1]} cuts, {kinds[2]} fresh), {d}")
    assert d.frames == 1500 and d.mx <= TOL and d.nd == 0
    assert kinds[1] > 0 and kinds[2] > 0


def test_config2_hdr_4k_f16():
    ts = (float(np.float32(1 / 3)), float(np.float32(2 / 3)))
    spec = oracle.FormatSpec("f16", linear=True, white=80.0)
    I = fg.Interpolator()
    assert I.init(3840, 2160, fg.VK_R16G16B16A16_SFLOAT, transfer=1, linear_white_nits=80.0), I.init_error()
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    gen = torch.Generator(device="cuda")
    worst = 0.0
    ndiff = 0
    for k in range(16):
        gen.manual_seed(2 * 10 ** 6 + k)
        a, c = workloads_gpu.hdr_pair(3840, 2160, gen)
        I.begin_frame()
        assert I.record_estimate(a, c), I.last_error()
        tr = fg.read_trace(I)
        ah, ch = a.cpu().numpy(), c.cpu().numpy()
        est = oracle.estimate_fmt(ah, ch, spec)
        assert tr["cut"] == est["cut"] and np.array_equal(tr["pf"], est["pf"]), f"pair {k}: estimate differs"
        for t in ts:
            o = torch.empty_like(a)
            assert I.record_synth(a, c, o, t), I.last_error()
            assert I.record_debug_counters(cnt)
            torch.cuda.synchronize()
            ref = oracle.synth_fmt(ah, ch, est, t, spec, trace=True)
            assert decision(tr["cut"], int(cnt[0]), 3840, 2160) == ref["reason"], f"pair {k}: decision at t={t}"
            got = o.cpu().numpy()
            nd = got.view(np.uint16) != ref["out"].view(np.uint16)
            ndiff += int(np.count_nonzero(nd))
            if nd.any():   # in PQ levels, the unit of the mismatch metric
                pq = np.vectorize(lambda v: oracle.pq255(v, 80.0))
                worst = max(worst, float(np.abs(pq(got[nd].astype(np.float32)) - pq(ref["out"][nd].astype(np.float32))).max()))
    I.close()
    print(f"config 2: 16 pairs, 32 frames: max diff {worst} PQ levels, {ndiff} half floats differ")
    assert worst <= TOL and ndiff == 0


def test_config3_full_batch():
    import batch_bench
    slots = batch_bench.slots()
    B = fg.Batch()
    prev, curr, outs, rgba = [], [], [], {}
    gen = torch.Generator(device="cuda")
    for i, (w, h, fmt, m) in enumerate(slots):
        assert B.add(w, h, batch_bench.VK[fmt], multiplier=m) == i, B.error()
        gen.manual_seed(3 * 10 ** 6 + i)
        d = workloads_gpu.flow_batch(1, w, h, gen)
        if fmt == "rgba8":
            rgba[i] = (d["prev"][0].cpu().numpy(), d["curr"][0].cpu().numpy())
        prev.append(batch_bench.to_dev(fmt, d["prev"][0].contiguous()))
        curr.append(batch_bench.to_dev(fmt, d["curr"][0].contiguous()))
        outs += [batch_bench.like(prev[-1]) for _ in range(m - 1)]
    assert B.record(prev, curr, outs), B.error()
    torch.cuda.synchronize()
    got = [tuple(x.cpu().numpy() for x in o) if isinstance(o, tuple) else o.cpu().numpy() for o in outs]
    dstand, dor = Diff(), Diff()
    j = 0
    for i, (w, h, fmt, m) in enumerate(slots):
        I = fg.Interpolator()
        assert I.init(w, h, batch_bench.VK[fmt]), I.init_error()
        I.begin_frame()
        assert I.record_estimate(prev[i], curr[i])
        est = oracle.estimate(*rgba[i], trace=False) if fmt == "rgba8" else None
        for t in fg.Batch.times(m):
            o = batch_bench.like(prev[i])
            assert I.record_synth(prev[i], curr[i], o, t)
            torch.cuda.synchronize()
            for x, y in zip(o if isinstance(o, tuple) else (o,), got[j] if isinstance(got[j], tuple) else (got[j],)):
                dstand.add(y, x.cpu().numpy())
            if est is not None:
                ref, _ = oracle.synth(*rgba[i], est, t)
                dor.add(got[j], ref)
            j += 1
        I.close()
    print(f"config 3: every slot against a standalone Interpolator, {dstand}; Rgba8 slots against the oracle, {dor}")
    assert j == len(outs) == 127
    assert dor.frames == sum(m - 1 for _, _, f, m in slots if f == "rgba8") == 31
    assert dstand.nd == 0 and dor.nd == 0
