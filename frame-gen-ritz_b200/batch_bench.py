"""Time the batched path on the mixed batch: 64 frame pairs in one batch, sizes 1280x720 / 1920x1080 /
2560x1440 / 3840x2160 in ratio 8:4:2:1 (34 / 17 / 9 / 4), formats cycling Rgba8 / Rgb10 / Nv12 / P010, multipliers
cycling 2 / 3 / 4, content from the smooth-flow generator (workloads_gpu, per-pair seeds).

    python frame-gen-ritz_b200/batch_bench.py [--reps 20] [--gpus N]
    torchrun --nproc-per-node N --master-addr 127.0.0.1 frame-gen-ritz_b200/batch_bench.py --gpus N

Each launch shape is timed as a CUDA graph of one whole-batch record (device time, CUDA events, median of --reps
replays); tune() then picks its shape. Prints one JSON line. Under torchrun the 64 pairs are partitioned over the ranks
by cost (replicas.shard_by_cost: the pixels each pair moves), each rank records its share as one batch on its GPU,
and a shape's time is the slowest rank's (no collective on the data path).
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
import replicas  # noqa: E402
import workloads  # noqa: E402
import workloads_gpu  # noqa: E402

VK = {"rgba8": fg.VK_R8G8B8A8_UNORM, "rgb10": fg.VK_A2B10G10R10_UNORM, "nv12": fg.VK_R8_UNORM,
      "p010": fg.VK_R16_UNORM}
SHAPES = [(0, 0, 1, 0), (3, 1, 1, 0), (0, 0, 4, 0), (3, 1, 4, 0), (0, 0, 8, 0), (2, 1, 8, 0), (3, 0, 8, 0), (3, 1, 8, 0),
          (0, 0, 1, 1), (3, 1, 1, 1), (0, 0, 8, 1), (3, 1, 8, 1), (0, 0, 8, 4), (3, 1, 8, 4), (0, 0, 8, 8),
          (3, 1, 8, 8)]   # Batch::tune's candidates, in its order


def slots():
    sizes = [(1280, 720)] * 34 + [(1920, 1080)] * 17 + [(2560, 1440)] * 9 + [(3840, 2160)] * 4
    fmts = ["rgba8", "rgb10", "nv12", "p010"]
    return [(w, h, fmts[i % 4], 2 + i % 3) for i, (w, h) in enumerate(sizes)]


def to_dev(fmt, rgba):
    if fmt == "rgba8":
        return rgba
    a = rgba.cpu().numpy()
    if fmt == "rgb10":
        return torch.from_numpy(workloads.to_rgb10(a).view(np.int32)).cuda()
    y, c = workloads.to_yuv(a, 8 if fmt == "nv12" else 10, "bt709")
    if fmt == "p010":
        y, c = y.view(np.int16), c.view(np.int16)
    return torch.from_numpy(y).cuda(), torch.from_numpy(c).cuda()


def like(d):
    return tuple(torch.zeros_like(x) for x in d) if isinstance(d, tuple) else torch.zeros_like(d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--gpus", type=int, default=1, help="ranks, one per GPU (started here unless a launcher did)")
    a = ap.parse_args()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(replicas.spawn_ranks(os.path.abspath(__file__), sys.argv[1:], a.gpus))
    if int(os.environ.get("WORLD_SIZE", "1")) != a.gpus:
        raise SystemExit(f"batch_bench.py: --gpus {a.gpus} but the launcher started {os.environ.get('WORLD_SIZE')} "
                         "rank(s)")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    rank, n = replicas.world()
    all_slots = slots()
    mine = replicas.shard_by_cost([replicas.pair_cost(w, h, m) for w, h, _, m in all_slots], n)[rank]
    B = fg.Batch()
    prev, curr, outs = [], [], []
    px = 0
    for j, i in enumerate(mine):
        w, h, fmt, m = all_slots[i]
        assert B.add(w, h, VK[fmt], multiplier=m) == j, B.error()
        gen = torch.Generator(device="cuda")
        gen.manual_seed(3 * 10 ** 6 + i)   # the pair's content does not depend on the partition
        d = workloads_gpu.flow_batch(1, w, h, gen)
        prev.append(to_dev(fmt, d["prev"][0]))
        curr.append(to_dev(fmt, d["curr"][0]))
        outs += [like(prev[-1]) for _ in range(m - 1)]
        px += w * h * (m - 1)
    s = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {}
    for shape in SHAPES:
        B.set_shape(*shape)
        with torch.cuda.stream(s):
            assert B.record(prev, curr, outs, stream=s), B.error()
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                assert B.record(prev, curr, outs, stream=s)
            g.replay()
            torch.cuda.synchronize()
            ts = []
            for _ in range(a.reps):
                e0.record(s)
                g.replay()
                e1.record(s)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
        res["%d_%d_%d_%d" % shape] = round(replicas.max_over_ranks(float(np.median(ts)), device="cuda"), 3)
        del g
    with torch.cuda.stream(s):
        best = B.tune(prev, curr, outs, reps=3, stream=s)
    frames = len(outs)
    if n > 1:   # totals over the ranks
        import torch.distributed as dist
        t = torch.tensor([len(outs), px], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        frames, px = int(t[0]), int(t[1])
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"workload": "mixed batch: 64 pairs, 34x720p / 17x1080p / 9x1440p / 4x2160p, Rgba8 / Rgb10 / "
                                      "Nv12 / P010, 2x / 3x / 4x", "ranks": n, "generated_frames": frames,
                          "generated_megapixels": round(px / 1e6, 1), "ms_per_batch": res,
                          "shape_keys": "ctasPerSm_order_streams_mergeEstimates (ctasPerSm 0: one launch per synthesis; mergeEstimates G: the estimates merged into one launch per pass for each of G groups of slots)",
                          "tuned_shape_rank0": "%d_%d_%d_%d" % SHAPES[best] if best >= 0 else None}), flush=True)


if __name__ == "__main__":
    main()
