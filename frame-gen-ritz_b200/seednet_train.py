"""Train the seed proposer (csrc/fg_seednet.cu) on the GPU with the library's own kernels.

    python frame-gen-ritz_b200/seednet_train.py [--steps 3125] [--batch 64] [--lr 1e-3] [--out seednet_l1.bin]
    python frame-gen-ritz_b200/seednet_train.py --gpus N ...   (or torchrun --nproc-per-node N ... --gpus N)

Data-parallel under torchrun (one process per GPU, NCCL): every rank draws its own crops (--batch per rank, a global
batch of N x --batch), the ranks' gradients are summed by one all-reduce of the 39,912 float32 values per step,
in place in the net's gradient buffer, and the Adam step reads them times 1 / N (the mean gradient of the global
batch); the ranks start from the same parameters and so stay identical. Rank 0 logs and writes the parameters.

Data: 256x256 crops from the smooth-flow generator (workloads_gpu.flow_batch: smooth motion up to 24 px, 5 % scene
cuts, 5 % fresh content), 3125 steps x 64 crops = 200k crops, each crop new. Input: the crop pair's level-1 luma
(64x64 at flowScale 2, the library's own luma pyramid, read back with recordTrace). Targets per 8x8 block of level 1:
  - candidate 1: the ground-truth half-vector, the block's mean of v / 8 (content displacement prev -> curr in
    level-1 pixels, halved: a at q - h, c at q + h);
  - candidate 2: the plain search's vector at level 1 (the library's median-filtered integer search field);
  - confidence: candidate 1 within one level-1 pixel of the truth (the loss's BCE target);
  - weight 0 for scene cuts (no truth), 1 otherwise.
Adam (0.9, 0.999), lr 1e-3. Writes the float32 parameters (fg_seednet_param_count() values) to --out and a log of
the loss to --log.
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import framegen as fg  # noqa: E402
import replicas  # noqa: E402
import workloads_gpu  # noqa: E402

CROP = 256


def init_params(seed):
    """He-uniform weights, zero biases, in the flat layout of fg_seednet (per layer [cout][9][cin] then [cout])"""
    cin = [2, 32, 32, 32, 32, 32]
    cout = [32, 32, 32, 32, 32, 8]
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in zip(cin, cout):
        lim = np.sqrt(6.0 / (9 * ci))
        parts.append(rng.uniform(-lim, lim, co * 9 * ci).astype(np.float32))
        parts.append(np.zeros(co, np.float32))
    p = np.concatenate(parts)
    assert p.size == fg.lib().fg_seednet_param_count()
    return p


class Labeller:
    """the library's level-1 luma and plain search field of crop pairs, on the device (no host round trip)"""

    def __init__(self, batch):
        self.I = fg.Interpolator()
        assert self.I.init(CROP, CROP, fg.VK_R8G8B8A8_UNORM), self.I.init_error()
        self.l = self.I.trace_layout()
        assert self.l.nLevels >= 2
        self.buf = torch.zeros((batch, self.l.size), dtype=torch.uint8, device="cuda")

    def __call__(self, prev, curr):
        B = prev.shape[0]
        for b in range(B):
            self.I.begin_frame()
            assert self.I.record_estimate(prev[b], curr[b]), self.I.last_error()
            assert self.I.record_trace(self.buf[b])
        l = self.l
        w1, h1, bw1, bh1 = l.lw[1], l.lh[1], l.bw[1], l.bh[1]
        o = l.lumaOff + 8 * l.lw[0] * l.lh[0]   # level 1: a then c
        la = self.buf[:B, o:o + 4 * w1 * h1].view(torch.float32).reshape(B, h1, w1)
        lc = self.buf[:B, o + 4 * w1 * h1:o + 8 * w1 * h1].view(torch.float32).reshape(B, h1, w1)
        of = l.fieldOff + 16 * l.bw[0] * l.bh[0] + 8 * bw1 * bh1   # level 1's median3 field
        v1 = self.buf[:B, of:of + 8 * bw1 * bh1].view(torch.float32).reshape(B, bh1, bw1, 2)
        return la, lc, v1


def targets(v, kind, v1):
    """(B, 8, 8, 6) targets of a batch: truth half-vectors at level 1 (block means of v / 8), the search field, weights"""
    B = v.shape[0]
    bh, bw = v1.shape[1:3]
    truth = (v.reshape(B, bh, CROP // bh, bw, CROP // bw, 2).mean(dim=(2, 4))) / 8.0
    t = torch.zeros(B, bh, bw, 6, device="cuda")
    t[..., 0:2] = truth
    t[..., 2:4] = v1
    t[..., 4] = (kind != 1).float()[:, None, None]
    return t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=3125)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=os.path.join(HERE, "seednet_l1.bin"))
    ap.add_argument("--log", default=None)
    ap.add_argument("--gpus", type=int, default=1, help="ranks, one per GPU (started here unless a launcher did)")
    a = ap.parse_args()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(replicas.spawn_ranks(os.path.abspath(__file__), sys.argv[1:], a.gpus))
    if int(os.environ.get("WORLD_SIZE", "1")) != a.gpus:
        raise SystemExit(f"seednet_train.py: --gpus {a.gpus} but the launcher started {os.environ.get('WORLD_SIZE')} "
                         "rank(s)")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    sync = replicas.GradSync()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(sync.rank_seed(a.seed))
    net = fg.SeedNet(a.batch, CROP // 4, CROP // 4, device=local)
    net.set_params(init_params(a.seed))
    grad = net.grad_buffer()
    lab = Labeller(a.batch)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    hist, t0 = [], time.time()
    for step in range(a.steps):
        d = workloads_gpu.flow_batch(a.batch, CROP, CROP, gen)
        la, lc, v1 = lab(d["prev"], d["curr"])
        x = fg.SeedNet.pack(la.contiguous(), lc.contiguous())
        net.backward(x, targets(d["v"], d["kind"], v1), loss)
        sync(grad)
        net.adam(a.lr, grad_scale=sync.scale())
        if step % 100 == 0 or step == a.steps - 1:
            torch.cuda.synchronize()
            hist.append((step, float(loss)))
            if sync.rank == 0:
                print(f"step {step} loss {float(loss):.4f} ({time.time() - t0:.1f} s)", flush=True)
    p = net.params()
    if sync.n > 1:   # the ranks took identical steps: their parameters agree bit for bit
        import torch.distributed as dist
        lo, hi = torch.from_numpy(p).cuda(), torch.from_numpy(p).cuda()
        dist.all_reduce(lo, op=dist.ReduceOp.MIN)
        dist.all_reduce(hi, op=dist.ReduceOp.MAX)
        assert torch.equal(lo, hi), "ranks' parameters diverged"
        dist.destroy_process_group()
    if sync.rank == 0:
        p.tofile(a.out)
        if a.log:
            with open(a.log, "w") as f:
                json.dump({"steps": a.steps, "batch": a.batch * sync.n, "ranks": sync.n, "lr": a.lr,
                           "crops": a.steps * a.batch * sync.n, "seconds": round(time.time() - t0, 1),
                           "loss": hist}, f)
        print("wrote", a.out)


if __name__ == "__main__":
    main()
