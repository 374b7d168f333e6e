#!/usr/bin/env python3
"""Benchmark of the V1 path: 4K ms per real pair (estimate + 3 synths at t = 1/4, 1/2, 3/4), 3840x2160 Rgba8.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one real pair: recordEstimate + 3 recordSynth. `value` is device time with the inputs resident in HBM:
each step's pair comes from a pool of distinct pairs larger than L2 (so no step reads a cached pair), and each
pool slot's step is a CUDA graph of the library's own launches; `value` = max-over-ranks time / pairs of all ranks.
`e2e` is the same metric through the public API with host buffers: every step copies its pair host -> device from
pinned memory, records the estimate and 3 synths, and copies the 3 frames back.
`roofline` is the dominant kernel (the fused synth) against the measured HBM copy bandwidth, its duration from the
library's own per-pass CUDA events. `cpu_baseline` is the oracle (a plain-C restatement of proto/interp.py) on this
host's cores. --impl reference times that CPU implementation itself (rank 0 only); where FGR_REF names a checkout
of the reference, it times the reference's own proto/interp.py (NumPy + OpenCV) on the same pairs instead and keeps
the port as a second row.
Multi-GPU: every rank runs its own pairs (weak scaling, no collective on the data path). `--gpus N` without a
launcher starts the N ranks itself (one process per GPU, the launcher's environment variables, rendezvous on
127.0.0.1); under torchrun the launcher's ranks are used and must number N. `value` is then the whole job's time per
pair (the slowest rank's span over the pairs of all ranks) and `per_rank_ms_per_pair` the slowest rank's latency.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(REPO, "frame-gen-ritz_b200"), os.path.join(REPO, "oracle")):
    sys.path.insert(0, _p)

METRIC = "4K ms per real pair (estimate+3 synths), CNN-seeded vs plain, PSNR within 0.1 dB"
W4K, H4K = 3840, 2160
TS = (0.25, 0.5, 0.75)
FW, FH = W4K // 2, H4K // 2
# algorithmic bytes of one fused synth launch: both frames read, the per-pixel field read, the output written
SYNTH_BYTES = 2 * 4 * W4K * H4K + 8 * FW * FH + 4 * W4K * H4K
PAIR_BYTES = 2 * 4 * W4K * H4K + 8 * FW * FH + 3 * SYNTH_BYTES     # (A): 431,308,800 B per pair


def args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pool", type=int, default=8, help="distinct 4K pairs cycled through (8 x 66 MB > L2)")
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--interp-pairs", type=int, default=5,
                    help="--impl reference with FGR_REF set: 4K pairs of proto/interp.py timed (median)")
    ap.add_argument("--copy-streams", type=int, default=1,
                    help="e2e: streams per copy direction, each frame split into that many row bands (on a B200 one "
                         "stream already fills the PCIe link: 1.96 ms per pair with 1, 2.00-2.02 with 2-4)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU leg (the oracle's timing and the parity checks)")
    ap.add_argument("--parity-c1-pairs", type=int, default=100, help="1080p pairs of the parity check (config 1)")
    ap.add_argument("--parity-c2-pairs", type=int, default=2, help="4K RgbaF16 pairs of the parity check (config 2)")
    ap.add_argument("--batch-reps", type=int, default=10, help="graph replays of the config-3 batch per shape (0: no line)")
    ap.add_argument("--eager", type=int, default=0,
                    help="profiling mode: run this many eager steps (no graphs, no timing, no JSON) and exit")
    ap.add_argument("--seed-net", default=os.path.join(REPO, "frame-gen-ritz_b200", "seednet_l1.bin"),
                    help="seed-net weights of the CNN-seeded arm (reported beside the plain path)")
    ap.add_argument("--seed-level", type=int, default=1)
    ap.add_argument("--no-seed-net", action="store_true")
    ap.add_argument("--psnr-pairs", type=int, default=8, help="held-out 4K pairs of the CNN-vs-plain PSNR check")
    ap.add_argument("--blur-samples", type=int, default=4, help="sub-frames of the motion-blur line (0: no line)")
    ap.add_argument("--dry-run", action="store_true",
                    help="the rank plumbing only, on CPU with gloo: a stand-in host step, no GPU (for the CPU tests)")
    return ap.parse_args()


def dry_run(a, world, rank):
    """The rank logic of the timed region without a GPU: gloo, a barrier on both sides, a stand-in host step per pair,
    the max of the ranks' spans; rank 0 prints a line shaped like the real one."""
    import datetime
    import torch.distributed as dist
    import replicas
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    x = np.arange(1 << 16, dtype=np.float64)
    for _ in range(a.warmup):
        np.sort(x[::-1])
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        np.sort(x[::-1])
    span = (time.perf_counter() - t0) * 1e3
    if world > 1:
        dist.barrier()
    t_ms = replicas.max_over_ranks(span)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": round(t_ms / (a.steps * world), 6), "unit": "ms",
                          "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                          "per_rank_ms_per_pair": round(t_ms / a.steps, 6), "dry_run": True}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def workload_pair():
    import workloads
    p, c, _ = workloads.flow_pair(W4K, H4K, seed=4 * 10 ** 6)
    return p, c


def frame_stats(got, ref):
    d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
    return int(d.max()), float(d.sum()), d.size, int(np.count_nonzero(d))


class ParityTally:
    """max / mean absolute difference, differing bytes and decision agreement over many frames"""

    def __init__(self):
        self.mx, self.sum, self.n, self.nd, self.frames, self.pairs, self.dec_ok, self.dec_n = 0, 0.0, 0, 0, 0, 0, 0, 0

    def add(self, got, ref):
        mx, sm, n, nd = frame_stats(got, ref)
        self.mx, self.sum, self.n, self.nd, self.frames = max(self.mx, mx), self.sum + sm, self.n + n, self.nd + nd, \
            self.frames + 1

    def decision(self, same):
        self.dec_n += 1
        self.dec_ok += int(bool(same))

    def report(self, **extra):
        return dict({"pairs": self.pairs, "frames": self.frames, "max_abs_diff": self.mx,
                     "mean_abs_diff": round(self.sum / max(self.n, 1), 9), "bytes_differing": self.nd,
                     "decisions_agree": f"{self.dec_ok}/{self.dec_n}"}, **extra)


def gpu_decision(cut, untrusted, W, H, frac=0.15):
    if cut:
        return "cut"
    return "untrusted" if untrusted / (W * H) > float(np.float32(frac)) else None


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_leg(pool, outs, seconds):
    """The CPU baseline on the metric's own workload: the oracle (the plain-C port of proto/interp.py, all host
    threads) runs estimate + 3 synths on full 3840x2160 pairs of the pool, for about `seconds` (at least every pool
    pair once); returns (median ms per pair, pairs timed, parity of the GPU's outputs of those pairs against the
    oracle's: the oracle is the checker here, its outputs are compared with what the graphs left in `outs`)."""
    import oracle
    times = []
    tally = ParityTally()
    host = [(pool[k][0].cpu().numpy(), pool[k][1].cpu().numpy()) for k in range(len(pool))]
    got = [[o.cpu().numpy() for o in outs[k]] for k in range(len(pool))]
    t_end = time.perf_counter() + seconds
    k = 0
    while True:
        j = k % len(pool)
        p, c = host[j]
        t0 = time.perf_counter()
        est = oracle.estimate(p, c, trace=False)
        res = [oracle.synth(p, c, est, t) for t in TS]
        times.append(time.perf_counter() - t0)
        if k < len(pool):
            tally.pairs += 1
            for (ref, _), g in zip(res, got[j]):
                tally.add(g, ref)
        k += 1
        if time.perf_counter() > t_end and k >= len(pool):
            break
    return statistics.median(times) * 1e3, k, tally


def config3_inputs(fg):
    """the 64-pair mixed batch at full size (34 x 720p, 17 x 1080p, 9 x 1440p, 4 x 2160p; Rgba8 / Rgb10 / Nv12 / P010;
    2x / 3x / 4x), content from the smooth-flow generator seeded per pair: (slots, Batch, prev, curr, outs, rgba pairs)"""
    import torch
    import batch_bench
    import workloads_gpu
    slots = batch_bench.slots()
    B = fg.Batch()
    prev, curr, outs, rgba = [], [], [], {}
    gen = torch.Generator(device="cuda")
    for i, (w, h, fmt, m) in enumerate(slots):
        assert B.add(w, h, batch_bench.VK[fmt], multiplier=m) == i, B.error()
        gen.manual_seed(3 * 10 ** 6 + i)
        d = workloads_gpu.flow_batch(1, w, h, gen)
        if fmt == "rgba8":
            rgba[i] = (d["prev"][0], d["curr"][0])
        prev.append(batch_bench.to_dev(fmt, d["prev"][0].contiguous()))
        curr.append(batch_bench.to_dev(fmt, d["curr"][0].contiguous()))
        outs += [batch_bench.like(prev[-1]) for _ in range(m - 1)]
    return slots, B, prev, curr, outs, rgba


def batch_arm(a, b3):
    """Config 3 timed: one Batch record of all 64 pairs (127 generated frames, 259 megapixels) as a CUDA graph, device
    time (CUDA events), median of --batch-reps replays, in the single-stream per-synthesis shape and in the shape
    Batch::tune picks on the device"""
    import torch
    slots, B, prev, curr, outs, _ = b3
    s = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed():
        with torch.cuda.stream(s):
            assert B.record(prev, curr, outs, stream=s), B.error()
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                assert B.record(prev, curr, outs, stream=s)
            for _ in range(2):
                g.replay()
            torch.cuda.synchronize()
            ts = []
            for _ in range(a.batch_reps):
                e0.record(s)
                g.replay()
                e1.record(s)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
        del g
        return statistics.median(ts)

    assert B.set_shape(0, 0, 1)
    base = timed()
    with torch.cuda.stream(s):
        best = B.tune(prev, curr, outs, reps=3, stream=s)
    shape = B.shape()
    tuned = timed()
    px = sum(w * h * (m - 1) for w, h, _, m in slots)
    return {"workload": "config 3: 64 pairs, 34 x 720p / 17 x 1080p / 9 x 1440p / 4 x 2160p, Rgba8 / Rgb10 / Nv12 / "
                        "P010, 2x / 3x / 4x; one Batch record per step, graph-replayed",
            "generated_frames": len(outs), "generated_megapixels": round(px / 1e6, 1),
            "ms_per_batch_per_synthesis_1_stream": round(base, 3), "ms_per_batch_tuned": round(tuned, 3),
            "tuned_shape": {"ctas_per_sm": shape[0], "order": shape[1], "streams": shape[2],
                            "merge_estimates": shape[3], "index": best},
            "megapixels_per_s_tuned": round(px / 1e6 / (tuned * 1e-3), 1), "reps": a.batch_reps}


def parity_configs(a, fg, b3):
    """Every workload configuration of the path against the oracle (rank 0, N = 1; part of the CPU leg: the oracle
    runs on the host for each): config 0 (640x360, 2x, one pair, also its device latency), config 1 (1080p 4x, a sample
    of --parity-c1-pairs of the 500), config 2 (4K RgbaF16 linear 3x, --parity-c2-pairs of the 200), config 3 (the
    full 64-pair mixed batch: every slot against a standalone Interpolator, the Rgba8 slots against the oracle)."""
    import torch
    import oracle
    import workloads
    import workloads_gpu
    out = {}
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")

    def pair_through(I, da, dc, ts):
        I.begin_frame()
        assert I.record_estimate(da, dc)
        tr = fg.read_trace(I)
        res = []
        for t in ts:
            o = torch.empty_like(da)
            assert I.record_synth(da, dc, o, t)
            assert I.record_debug_counters(cnt)
            torch.cuda.synchronize()
            res.append((o.cpu().numpy(), int(cnt[0])))
        return tr, res

    # config 0
    p, c = workloads.pan_pair()
    I = fg.Interpolator()
    assert I.init(640, 360, fg.VK_R8G8B8A8_UNORM), I.init_error()
    da, dc = torch.from_numpy(p).cuda(), torch.from_numpy(c).cuda()
    tr, res = pair_through(I, da, dc, [0.5])
    tally = ParityTally()
    tally.pairs = 1
    est = oracle.estimate(p, c, trace=False)
    ref, why = oracle.synth(p, c, est, 0.5)
    tally.add(res[0][0], ref)
    tally.decision(gpu_decision(tr["cut"], res[0][1], 640, 360) == why and tr["sad"] == est["sad"])
    o = torch.empty_like(da)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        I.begin_frame()
        I.record_estimate(da, dc, stream=s)
        I.record_synth(da, dc, o, 0.5, stream=s)
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            I.begin_frame()
            I.record_estimate(da, dc, stream=s)
            I.record_synth(da, dc, o, 0.5, stream=s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lat = []
        for _ in range(50):
            e0.record(s)
            g.replay()
            e1.record(s)
            torch.cuda.synchronize()
            lat.append(e0.elapsed_time(e1) * 1e3)
    del g
    I.close()
    out["config0"] = tally.report(workload="640x360 Rgba8 2x (t = 1/2), the panning pair with sprite and HUD",
                                  latency_us=round(statistics.median(lat), 2),
                                  latency_method="median of 50 CUDA-graph replays of estimate + synth, device time")
    # config 1
    tally = ParityTally()
    I = fg.Interpolator()
    assert I.init(1920, 1080, fg.VK_R8G8B8A8_UNORM), I.init_error()
    gen = torch.Generator(device="cuda")
    kinds = [0, 0, 0]
    n1 = a.parity_c1_pairs
    for b in range((n1 + 9) // 10):
        gen.manual_seed(1 * 10 ** 6 + b)
        d = workloads_gpu.flow_batch(10, 1920, 1080, gen)
        for k in range(min(10, n1 - 10 * b)):
            da, dc = d["prev"][k].contiguous(), d["curr"][k].contiguous()
            kinds[int(d["kind"][k])] += 1
            tr, res = pair_through(I, da, dc, TS)
            p, c = da.cpu().numpy(), dc.cpu().numpy()
            est = oracle.estimate(p, c, trace=False)
            tally.pairs += 1
            for (g_out, u), t in zip(res, TS):
                ref, why = oracle.synth(p, c, est, t)
                tally.add(g_out, ref)
                tally.decision(gpu_decision(tr["cut"], u, 1920, 1080) == why and tr["sad"] == est["sad"])
    I.close()
    out["config1"] = tally.report(workload=f"1920x1080 Rgba8 4x, {n1} of the 500 smooth-flow pairs ({kinds[1]} cuts, "
                                           f"{kinds[2]} fresh); all 500 run in tests/test_configs_gpu.py")
    # config 2
    spec = oracle.FormatSpec("f16", linear=True, white=80.0)
    ts2 = (float(np.float32(1 / 3)), float(np.float32(2 / 3)))
    I = fg.Interpolator()
    assert I.init(3840, 2160, fg.VK_R16G16B16A16_SFLOAT, transfer=1, linear_white_nits=80.0), I.init_error()
    worst, ndiff, frames, dec_ok, dec_n = 0.0, 0, 0, 0, 0
    for k in range(a.parity_c2_pairs):
        gen.manual_seed(2 * 10 ** 6 + k)
        da, dc = workloads_gpu.hdr_pair(3840, 2160, gen)
        tr, res = pair_through(I, da, dc, ts2)
        ah, ch = da.cpu().numpy(), dc.cpu().numpy()
        est = oracle.estimate_fmt(ah, ch, spec)
        for (got, u), t in zip(res, ts2):
            ref = oracle.synth_fmt(ah, ch, est, t, spec, trace=True)
            nd = got.view(np.uint16) != ref["out"].view(np.uint16)
            ndiff += int(np.count_nonzero(nd))
            frames += 1
            dec_n += 1
            dec_ok += int(gpu_decision(tr["cut"], u, 3840, 2160) == ref["reason"])
            if nd.any():
                pq = np.vectorize(lambda v: oracle.pq255(v, 80.0))
                worst = max(worst, float(np.abs(pq(got[nd].astype(np.float32)) - pq(ref["out"][nd].astype(np.float32))).max()))
    I.close()
    out["config2"] = {"pairs": a.parity_c2_pairs, "frames": frames, "max_abs_diff_pq_levels": worst,
                      "half_floats_differing": ndiff, "decisions_agree": f"{dec_ok}/{dec_n}",
                      "workload": f"3840x2160 RgbaF16 linear 3x, {a.parity_c2_pairs} of the 200 HDR pairs; 16 run in "
                                  "tests/test_configs_gpu.py"}
    # config 3: the batch as the batch arm left it (its tuned shape); every slot against a standalone Interpolator
    import batch_bench
    slots, B, prev, curr, bouts, rgba = b3
    rgba = {k: (p.cpu().numpy(), c.cpu().numpy()) for k, (p, c) in rgba.items()}
    assert B.record(prev, curr, bouts), B.error()
    torch.cuda.synchronize()
    st, orc = ParityTally(), ParityTally()
    j = 0
    for i, (w, h, fmt, m) in enumerate(slots):
        I = fg.Interpolator()
        assert I.init(w, h, batch_bench.VK[fmt]), I.init_error()
        I.begin_frame()
        assert I.record_estimate(prev[i], curr[i])
        st.pairs += 1
        est = oracle.estimate(*rgba[i], trace=False) if fmt == "rgba8" else None
        orc.pairs += est is not None
        for t in fg.Batch.times(m):
            o = batch_bench.like(prev[i])
            assert I.record_synth(prev[i], curr[i], o, t)
            torch.cuda.synchronize()
            for x, y in zip(o if isinstance(o, tuple) else (o,), bouts[j] if isinstance(bouts[j], tuple) else (bouts[j],)):
                st.add(y.cpu().numpy(), x.cpu().numpy())
            if est is not None:
                ref, _ = oracle.synth(*rgba[i], est, t)
                orc.add(bouts[j].cpu().numpy(), ref)
            j += 1
        I.close()
    rs, ro = st.report(), orc.report()
    rs.pop("decisions_agree")
    ro.pop("decisions_agree")
    out["config3"] = {"workload": "the 64-pair mixed batch at full size, one Batch record in the tuned shape",
                      "vs_standalone": rs, "rgba8_vs_oracle": ro}
    return out


def clock_sampler(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    idx = str(local_rank)
    if vis:
        parts = [v.strip() for v in vis.split(",")]
        if local_rank < len(parts):
            idx = parts[local_rank]
    q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", "-i", idx, f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None


def clock_summary(proc):
    if proc is None:
        return None
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 8:
            continue
        try:
            sm.append(float(f[0]))
            mx.append(float(f[1]))
        except ValueError:
            continue
        for n, v in zip(names, f[4:8]):
            if v.lower().startswith("active"):
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def sources_sha(paths):
    import hashlib
    h = hashlib.sha256()
    for rel in paths:
        with open(os.path.join(REPO, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def ncu_synth():
    """the committed ncu summary of one 4K synth launch (profiles/synth_4k.json): dram bytes, warp instructions. It
    records the sha256 of the kernel sources it was captured from; when they have changed since, the figures are
    stale and are not reported ({"stale": True})."""
    try:
        with open(os.path.join(REPO, "profiles", "synth_4k.json")) as f:
            prof = json.load(f)
    except (OSError, ValueError):
        return {}
    try:
        if sources_sha(prof["sources"]) != prof["source_sha256"]:
            return {"stale": True}
    except (KeyError, OSError):
        return {"stale": True}
    return prof


def issue_roofline(prof, synth_us, clocks):
    """the synth against the instruction-issue ceiling, the roofline that binds it: its ncu warp-instruction count
    over its live duration, against one warp instruction per scheduler (4 per SM) per SM clock at the sampled clock"""
    n, sms = prof.get("warp_instructions_per_launch"), prof.get("sms")
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
    if not n or not sms or not mhz or not synth_us:
        return None
    achieved = n / (synth_us * 1e-6) / 1e12
    peak = sms * 4 * mhz * 1e6 / 1e12
    return {"kernel": "k_synth", "achieved": round(achieved, 4), "peak": round(peak, 4),
            "unit": "T warp instructions/s", "frac": round(achieved / peak, 4), "warp_instructions": n,
            "source": "ncu smsp__inst_executed of one 4K launch (profiles/synth_4k.json), live duration, sampled clock"}


def run_reference(a):
    """The reference arm: the CPU implementation of the path (the oracle port of proto/interp.py, all host threads) on
    the metric's workload itself, full 3840x2160 pairs, estimate + 3 synths per step (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    p, c = workload_pair()
    cores = os.cpu_count()
    step_ms = []
    for i in range(a.warmup + a.steps):
        k = i % 4   # four distinct pairs: the same content rolled, as the GPU arm's pool
        pa, pc = np.roll(p, (53 * k, 97 * k), axis=(0, 1)), np.roll(c, (53 * k, 97 * k), axis=(0, 1))
        t0 = time.perf_counter()
        est = oracle.estimate(pa, pc, trace=False)
        for t in TS:
            oracle.synth(pa, pc, est, t)
        if i >= a.warmup:
            step_ms.append((time.perf_counter() - t0) * 1e3)
    v = statistics.median(step_ms)
    sample = f"full 3840x2160 pairs (4 distinct, cycled), estimate + 3 synths per step; oracle, {cores} threads"
    port = {"value": round(v, 3), "unit": "ms", "cores": cores, "kind": "port", "sample": sample,
            "cpu_model": cpu_model()}
    cpu_impl = "oracle port (plain C, OpenMP) of proto/interp.py"
    numpy_ref = reference_interp_leg(a, p, c)
    if numpy_ref is not None:   # the reference's own NumPy + OpenCV code is the arm; the port stays as a second row
        v, cpu_impl = numpy_ref["value"], "proto/interp.py (NumPy + OpenCV), imported from FGR_REF"
        base = dict(numpy_ref, kind="reference")
    else:
        base = port
    line = {"metric": METRIC, "value": round(v, 3), "unit": "ms", "impl": "reference", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "V1 plain, 3840x2160 Rgba8, 4x (estimate + 3 synths), flowScale 2",
                       "cpu_impl": cpu_impl},
            "cpu_baseline": base,
            "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if numpy_ref is not None:
        line["port"] = port
    print(json.dumps(line), flush=True)


INTERP_SHA256 = "b5f5c7000221002e31a1f4c2b2883878eeab4ffd83760c4080facad527904315"


def reference_interp_leg(a, p, c):
    """The reference's own CPU implementation, proto/interp.py (NumPy + OpenCV), timed on the same full 3840x2160
    pairs as the port: estimate + 3 synths per pair, median over --interp-pairs pairs after one untimed pair, each
    pair's 3 frames compared byte for byte with the port's. Runs only where FGR_REF names a checkout of the reference
    (the directory that holds proto/interp.py, sha256-pinned) and cv2 imports; None otherwise."""
    ref = os.environ.get("FGR_REF")
    if not ref or a.interp_pairs <= 0:
        return None
    path = os.path.join(ref, "proto", "interp.py")
    if not os.path.isfile(path):
        return None
    try:
        import cv2
    except ImportError:
        return None
    import hashlib
    with open(path, "rb") as f:
        digest = hashlib.sha256(f.read()).hexdigest()
    if digest != INTERP_SHA256:
        raise SystemExit(f"{path}: sha256 {digest} is not the pinned {INTERP_SHA256}")
    sys.path.insert(0, os.path.dirname(path))
    import interp
    import oracle
    ms, equal = [], True
    for i in range(1 + a.interp_pairs):
        k = i % 4
        pa, pc = np.roll(p, (53 * k, 97 * k), axis=(0, 1)), np.roll(c, (53 * k, 97 * k), axis=(0, 1))
        ba, bc = pa[..., [2, 1, 0]].copy(), pc[..., [2, 1, 0]].copy()   # interp.py takes 8-bit BGR
        t0 = time.perf_counter()
        est = interp.estimate(ba, bc)
        got = [interp.synth(ba, bc, est, t) for t in TS]
        if i >= 1:
            ms.append((time.perf_counter() - t0) * 1e3)
        eo = oracle.estimate(pa, pc, trace=False)
        equal &= all(np.array_equal(g, oracle.synth(pa, pc, eo, t)[0][..., [2, 1, 0]]) for g, t in zip(got, TS))
    return {"value": round(statistics.median(ms), 3), "unit": "ms", "pairs": len(ms),
            "cores": cv2.getNumThreads(), "cv2_threads": cv2.getNumThreads(), "cv2": cv2.__version__,
            "numpy": np.__version__, "cpu_model": cpu_model(), "bytes_equal_to_port": bool(equal),
            "sample": f"{len(ms)} full 3840x2160 pairs (4 distinct, cycled), estimate + 3 synths each, after 1 untimed"}


def seed_net_arm(a, fg, pool, outs, stream, world, plain):
    """The CNN-seeded arm (Interpolator::setSeedNet at --seed-level, the trained weights): its graph-replayed ms per
    pair on the same pool as the plain path, and its PSNR against the plain path's on --psnr-pairs held-out 4K pairs
    of the smooth-flow generator (ground truth at t = 1/4, 1/2, 3/4)."""
    import torch
    import torch.distributed as dist
    import replicas
    import workloads_gpu
    params = np.fromfile(a.seed_net, np.float32)
    I = fg.Interpolator()
    assert I.init(W4K, H4K, fg.VK_R8G8B8A8_UNORM, device=torch.cuda.current_device()), I.init_error()
    assert I.set_seed_net(params, a.seed_level), "setSeedNet failed"
    graphs = []
    for k in range(a.pool):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            I.begin_frame()
            assert I.record_estimate(pool[k][0], pool[k][1], stream=stream)
            for o, t in zip(outs[k], TS):
                assert I.record_synth(pool[k][0], pool[k][1], o, t, stream=stream)
        graphs.append(g)
    with torch.cuda.stream(stream):
        for i in range(max(a.warmup, 3)):
            graphs[i % a.pool].replay()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for i in range(a.steps):
            graphs[i % a.pool].replay()
        ev1.record(stream)
    torch.cuda.synchronize()
    t_ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), device="cuda")
    del graphs
    gen = torch.Generator(device="cuda")
    gen.manual_seed(424242)
    o = torch.empty((H4K, W4K, 4), dtype=torch.uint8, device="cuda")
    ps = {"plain": [], "cnn": []}

    def psnr(x, y):
        mse = float(((x[..., :3].float() - y[..., :3].float()) ** 2).mean())
        return 99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)

    for i in range(a.psnr_pairs):
        d = workloads_gpu.flow_batch(1, W4K, H4K, gen, ts=TS)
        p, c = d["prev"][0], d["curr"][0]
        for name, J in (("plain", plain), ("cnn", I)):
            J.begin_frame()
            assert J.record_estimate(p, c)
            for t in TS:
                assert J.record_synth(p, c, o, t)
                ps[name].append(psnr(o, d["truth"][t][0]))
    torch.cuda.synchronize()
    I.close()
    dp = float(np.mean(ps["cnn"]) - np.mean(ps["plain"]))
    return {"level": a.seed_level, "ms_per_pair": round(t_ms / (a.steps * world), 4),
            "psnr_db": round(float(np.mean(ps["cnn"])), 3), "plain_psnr_db": round(float(np.mean(ps["plain"])), 3),
            "psnr_delta_db": round(dp, 4), "within_0_1_db": abs(dp) <= 0.1, "psnr_frames": len(ps["cnn"]),
            "data": "held-out smooth-flow pairs (workloads_gpu, seed 424242), 4K, ground truth at t = 1/4, 1/2, 3/4"}


def blur_arm(a, fg, pool, stream, world):
    """recordSynthBlur at 4K: one Gaussian-weighted output over [0.25, 0.75] from --blur-samples sub-frames, against
    the same sub-frames as separate recordSynth outputs (the unfused way, before any blend of them). Both timed as CUDA
    graphs behind the pair's estimate, cycling the pool; their cost = that graph minus the estimate-only graph."""
    import torch
    import replicas
    n = a.blur_samples
    fs = fg.Settings()
    fs.blurSamples, fs.blurWeights = n, 1
    I = fg.Interpolator()
    assert I.init(W4K, H4K, fg.VK_R8G8B8A8_UNORM, settings=fs, device=torch.cuda.current_device()), I.init_error()
    times, _ = fg.blur_plan(n, 1, 0.25, 0.75)
    o = torch.empty_like(pool[0][0])

    def graph(k, what):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            I.begin_frame()
            assert I.record_estimate(pool[k][0], pool[k][1], stream=stream)
            if what == "blur":
                assert I.record_synth_blur(pool[k][0], pool[k][1], o, 0.25, 0.75, stream=stream)
            elif what == "synths":
                for t in times.tolist():
                    assert I.record_synth(pool[k][0], pool[k][1], o, t, stream=stream)
        return g

    res = {}
    for what in ("estimate", "blur", "synths"):
        gs = [graph(k, what) for k in range(a.pool)]
        with torch.cuda.stream(stream):
            for i in range(max(a.warmup, 3)):
                gs[i % a.pool].replay()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for i in range(a.steps):
                gs[i % a.pool].replay()
            ev1.record(stream)
        torch.cuda.synchronize()
        res[what] = replicas.max_over_ranks(ev0.elapsed_time(ev1), device="cuda") / a.steps
        del gs
    I.close()
    return {"samples": n, "weights": "gaussian", "window": [0.25, 0.75],
            "blur_ms": round(res["blur"] - res["estimate"], 4),
            "separate_synths_ms": round(res["synths"] - res["estimate"], 4),
            "method": "graph replay over the pool, minus the estimate-only graph; 3840x2160 Rgba8"}


def main():
    a = args()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ and not (a.impl == "reference" and not a.dry_run):
        import replicas
        sys.exit(replicas.spawn_ranks(os.path.abspath(__file__), sys.argv[1:], a.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a)
    if world != a.gpus:
        raise SystemExit(f"bench.py: --gpus {a.gpus} but the launcher started {world} rank(s)")
    if a.dry_run:
        return dry_run(a, world, rank)
    import torch
    import torch.distributed as dist
    import datetime
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    import framegen as fg
    import replicas

    p_np, c_np = workload_pair()
    base_a = torch.from_numpy(p_np).cuda()
    base_c = torch.from_numpy(c_np).cuda()
    # pool of distinct pairs: the same content rolled (both frames alike, so the motion is unchanged)
    pool = []
    for k in range(a.pool):
        sh = (k * 97 + rank * 13) % W4K, (k * 53 + rank * 7) % H4K
        pool.append((torch.roll(base_a, shifts=(sh[1], sh[0]), dims=(0, 1)).contiguous(),
                     torch.roll(base_c, shifts=(sh[1], sh[0]), dims=(0, 1)).contiguous()))
    outs = [[torch.empty_like(base_a) for _ in TS] for _ in range(a.pool)]
    I = fg.Interpolator()
    assert I.init(W4K, H4K, fg.VK_R8G8B8A8_UNORM, device=local), I.init_error()
    stream = torch.cuda.Stream()
    if a.eager:   # for ncu: plain records, one pair, nothing else
        for i in range(a.eager):
            k = i % a.pool
            I.begin_frame()
            assert I.record_estimate(pool[k][0], pool[k][1], stream=stream)
            for o, t in zip(outs[k], TS):
                assert I.record_synth(pool[k][0], pool[k][1], o, t, stream=stream)
        torch.cuda.synchronize()
        I.close()
        return

    # correctness guard: the graph path gives the eager bytes
    with torch.cuda.stream(stream):
        I.begin_frame()
        assert I.record_estimate(pool[0][0], pool[0][1], stream=stream)
        for o, t in zip(outs[0], TS):
            assert I.record_synth(pool[0][0], pool[0][1], o, t, stream=stream)
    torch.cuda.synchronize()
    eager0 = [o.clone() for o in outs[0]]

    graphs = []
    for k in range(a.pool):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            I.begin_frame()
            assert I.record_estimate(pool[k][0], pool[k][1], stream=stream)
            for o, t in zip(outs[k], TS):
                assert I.record_synth(pool[k][0], pool[k][1], o, t, stream=stream)
        graphs.append(g)
    n_levels = I.trace_layout().nLevels
    # luma (+ deeper downsamples), search + median3 per level, subpixel, pixel field, synth + fallback per t
    launches_per_step = 1 + max(0, n_levels - 6) + 2 * n_levels + 2 + 2 * len(TS)

    with torch.cuda.stream(stream):
        for i in range(max(a.warmup, 3)):
            graphs[i % a.pool].replay()
    torch.cuda.synchronize()
    for o, e in zip(outs[0], eager0):
        assert torch.equal(o, e), "graph replay differs from the eager record"

    # ---- timed region: K steps, device time, max over ranks
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = clock_sampler(local)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for i in range(a.steps):
            graphs[i % a.pool].replay()
        ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clock_summary(clk)
    t_ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), device="cuda")
    ms_per_step = t_ms / a.steps          # the slowest rank's time per step (one pair on every rank)
    value = t_ms / (a.steps * world)      # the whole job's time per pair

    # ---- per-pass device times (the library's CUDA events on its stream; the launches queue behind a sleep so the
    # events see back-to-back execution, not host gaps)
    I.set_profiling(True)
    groups = {}
    for rep in range(5):
        k = rep % a.pool
        with torch.cuda.stream(stream):
            torch.cuda._sleep(5_000_000)
            I.begin_frame()
            I.record_estimate(pool[k][0], pool[k][1], stream=stream)
            for o, t in zip(outs[k], TS):
                I.record_synth(pool[k][0], pool[k][1], o, t, stream=stream)
        tm = I.read_timings()
        for name, ns in tm:
            groups.setdefault(name, []).append(ns / 1e3)
    I.set_profiling(False)
    synth_us = statistics.median(groups["synth"])
    breakdown = {n: round(statistics.median(v) * (3 if n in ("synth", "fallback") else 1), 2) for n, v in groups.items()}

    # ---- e2e through the public API with host buffers: every step uploads its pair from pinned host memory and
    # downloads its 3 frames; two buffer sets and separate copy streams let step i+1's upload and step i-1's download
    # run on the copy engines while step i computes
    ha = torch.from_numpy(p_np).pin_memory()
    hc = torch.from_numpy(c_np).pin_memory()
    hout = [[torch.empty(base_a.shape, dtype=torch.uint8).pin_memory() for _ in TS] for _ in range(2)]
    dA = [torch.empty_like(base_a) for _ in range(2)]
    dC = [torch.empty_like(base_c) for _ in range(2)]
    douts = [[torch.empty_like(base_a) for _ in TS] for _ in range(2)]
    nc = max(1, a.copy_streams)
    s_in = [torch.cuda.Stream() for _ in range(nc)]
    s_out = [torch.cuda.Stream() for _ in range(nc)]
    ev_in = [[torch.cuda.Event() for _ in range(nc)] for _ in range(2)]
    ev_out = [[torch.cuda.Event() for _ in range(nc)] for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    bands = [(H4K * j // nc, H4K * (j + 1) // nc) for j in range(nc)]   # row bands, one per copy stream
    step_no = [0]

    def e2e_step():
        i = step_no[0]
        step_no[0] += 1
        k = i % 2
        for j, (r0, r1) in enumerate(bands):
            with torch.cuda.stream(s_in[j]):
                if i >= 2:
                    s_in[j].wait_event(ev_done[k])   # step i-2's compute has read these inputs
                dA[k][r0:r1].copy_(ha[r0:r1], non_blocking=True)
                dC[k][r0:r1].copy_(hc[r0:r1], non_blocking=True)
                ev_in[k][j].record(s_in[j])
            stream.wait_event(ev_in[k][j])
            if i >= 2:
                stream.wait_event(ev_out[k][j])      # step i-2's outputs have left the device
        I.begin_frame()
        assert I.record_estimate(dA[k], dC[k], stream=stream)
        for o, t in zip(douts[k], TS):
            assert I.record_synth(dA[k], dC[k], o, t, stream=stream)
        ev_done[k].record(stream)
        for j, (r0, r1) in enumerate(bands):
            with torch.cuda.stream(s_out[j]):
                s_out[j].wait_event(ev_done[k])
                for o, h in zip(douts[k], hout[k]):
                    h[r0:r1].copy_(o[r0:r1], non_blocking=True)
                ev_out[k][j].record(s_out[j])

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0.record(s_in[0])
    for j in range(1, nc):
        s_in[j].wait_event(ev0)
    for _ in range(a.e2e_steps):
        e2e_step()
    last_k = (step_no[0] - 1) % 2
    for j in range(1, nc):
        s_out[0].wait_event(ev_out[last_k][j])
    ev1.record(s_out[0])
    torch.cuda.synchronize()
    e2e_ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), device="cuda")
    e2e_value = e2e_ms / (a.e2e_steps * world)
    if rank == 0:   # the downloaded frames are the pair's (pool pair 0 is the unshifted pair on rank 0)
        last = (step_no[0] - 1) % 2
        assert all(torch.equal(h, e.cpu()) for h, e in zip(hout[last], eager0)), "e2e output differs"

    # config 3, the batched path (rank 0, N = 1)
    b3 = batch = None
    if rank == 0 and world == 1 and (a.batch_reps > 0 or not a.no_cpu):
        b3 = config3_inputs(fg)
        if a.batch_reps > 0:
            batch = batch_arm(a, b3)
    # the CPU leg (rank 0, N = 1): every pool slot's plain outputs once more, then the oracle on the same pairs
    cpu = parity = None
    if rank == 0 and world == 1 and not a.no_cpu:
        with torch.cuda.stream(stream):
            for g in graphs:
                g.replay()
        torch.cuda.synchronize()
        v, n, tally = cpu_leg(pool, outs, a.cpu_seconds)
        cpu = {"value": round(v, 1), "unit": "ms", "cores": os.cpu_count(), "kind": "port", "cpu_model": cpu_model(),
               "sample": f"{n} full 3840x2160 pairs of the pool, estimate + 3 synths each, median; oracle (plain-C "
                         f"restatement of proto/interp.py, OpenMP, all host threads)"}
        parity = {"metric_workload": tally.report(workload="the bench's 4K pool: the GPU's graph outputs against the "
                                                            "oracle's")}
        parity["metric_workload"].pop("decisions_agree")
        parity.update(parity_configs(a, fg, b3))

    blur = blur_arm(a, fg, pool, stream, world) if a.blur_samples >= 2 else None
    seed = None
    if not a.no_seed_net and os.path.exists(a.seed_net):
        seed = seed_net_arm(a, fg, pool, outs, stream, world, I)


    peak, peak_kind = measured_peak()
    achieved = SYNTH_BYTES / (synth_us * 1e-6) / 1e9
    prof = ncu_synth()
    traffic = prof.get("dram_bytes_per_launch")   # None when the capture is stale
    del graphs
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 4), "unit": "ms", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": False,
                "per_rank_ms_per_pair": round(ms_per_step, 4),
                "value_is": "the whole job's device time per pair: the slowest rank's span / the pairs of all ranks",
                "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                "config": {"workload": "V1 plain, 3840x2160 Rgba8, 4x (estimate + synths at t=1/4, 1/2, 3/4), "
                                       "flowScale 2, radii 6/2, subpixel on",
                           "pairs_in_pool": a.pool, "l2": f"inputs larger than L2: {a.pool} distinct pairs "
                                                         f"({a.pool * 2 * 4 * W4K * H4K / 1e6:.0f} MB) cycled",
                           "parallelism": f"dp{world} (independent pairs per GPU)",
                           "algorithmic_bytes_per_pair": PAIR_BYTES},
                "hbm_gbs_per_pair": round(PAIR_BYTES / (value * 1e-3) / 1e9 / world, 1),
                "roofline": {"bound": "hbm", "kernel": "k_synth", "achieved": round(achieved, 1),
                             "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                             "traffic": traffic, "traffic_stale": bool(prof.get("stale")),
                             "algorithmic_bytes": SYNTH_BYTES, "duration_us": round(synth_us, 2)},
                "issue_roofline": issue_roofline(prof, synth_us, clocks),
                "breakdown_us": breakdown,
                "gpu_launches": launches_per_step * a.steps,
                "e2e": {"value": round(e2e_value, 4), "unit": "ms", "h2d_bytes_per_step": 2 * 4 * W4K * H4K,
                        "d2h_bytes_per_step": len(TS) * 4 * W4K * H4K},
                "cpu_baseline": cpu, "parity": parity, "clocks": clocks, "seed_net": seed, "motion_blur": blur,
                "batch": batch}
        print(json.dumps(line), flush=True)
    I.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
