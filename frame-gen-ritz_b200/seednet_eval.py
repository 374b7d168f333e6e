"""Evaluate the seed proposer: CNN-seeded against plain V1 on held-out smooth-flow pairs, against the ground truth.

    python frame-gen-ritz_b200/seednet_eval.py [--pairs 200] [--size 3840x2160] [--weights seednet_l1.bin] [--level 1]

Per pair (workloads_gpu.flow_batch, a seed the training never used): estimate + synths at t = 1/4, 1/2, 3/4 with
  plain   the V1 path (the full pyramid, searchRadiusTop at the coarsest level);
  cnn     the seed net at --level, the levels above it skipped, equal search radii below;
  zero    the same truncated pyramid seeded by a net whose output is all zero (the method without the net);
and the PSNR (RGB, peak 255) of each synthesized frame against the generator's ground truth at that t. Prints one
JSON line: mean PSNR per arm over all frames, the cnn - plain and cnn - zero differences, and the device time of the
estimate + 3 synths per arm (CUDA events, median over the pairs).
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import framegen as fg  # noqa: E402
import workloads_gpu  # noqa: E402

TS = (0.25, 0.5, 0.75)


def psnr(a, b):
    d = (a[..., :3].float() - b[..., :3].float()) ** 2
    mse = float(d.mean())
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)


def arm(W, H, params, level):
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM), I.init_error()
    if params is not None:
        assert I.set_seed_net(params, level)
    return I


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=200)
    ap.add_argument("--size", default="3840x2160")
    ap.add_argument("--weights", default=os.path.join(HERE, "seednet_l1.bin"))
    ap.add_argument("--level", type=int, default=1)
    ap.add_argument("--seed", type=int, default=424242)
    a = ap.parse_args()
    W, H = (int(v) for v in a.size.split("x"))
    params = np.fromfile(a.weights, np.float32)
    arms = {"plain": arm(W, H, None, 0), "cnn": arm(W, H, params, a.level),
            "zero": arm(W, H, np.zeros_like(params), a.level)}
    gen = torch.Generator(device="cuda")
    gen.manual_seed(a.seed)
    outs = [torch.empty((H, W, 4), dtype=torch.uint8, device="cuda") for _ in TS]
    ps = {k: [] for k in arms}
    ms = {k: [] for k in arms}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(a.pairs):
        d = workloads_gpu.flow_batch(1, W, H, gen, ts=TS)
        p, c = d["prev"][0], d["curr"][0]
        for name, I in arms.items():
            torch.cuda.synchronize()
            ev0.record()
            I.begin_frame()
            assert I.record_estimate(p, c), I.last_error()
            for o, t in zip(outs, TS):
                assert I.record_synth(p, c, o, t), I.last_error()
            ev1.record()
            torch.cuda.synchronize()
            ms[name].append(ev0.elapsed_time(ev1))
            for o, t in zip(outs, TS):
                ps[name].append(psnr(o, d["truth"][t][0]))
    res = {"pairs": a.pairs, "size": a.size, "level": a.level, "frames_per_arm": len(ps["plain"]),
           "psnr_db": {k: round(float(np.mean(v)), 4) for k, v in ps.items()},
           "cnn_minus_plain_db": round(float(np.mean(ps["cnn"]) - np.mean(ps["plain"])), 4),
           "cnn_minus_zero_db": round(float(np.mean(ps["cnn"]) - np.mean(ps["zero"])), 4),
           "ms_per_pair_eager": {k: round(float(np.median(v)), 4) for k, v in ms.items()}}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
