"""One small instance of each kernel family of the library, for a profiler to capture (every launch once or a few
times, a few hundred MB on the device at most). Seeded synthetic content (workloads.py).

python frame-gen-ritz_b200/profile_cases.py --case pair|formats|blur|seednet|ui|train [--size 3840x2160]

  pair      estimate + syntheses at t = 1/4, 1/2, 3/4 of one Rgba8 pair (luma pyramid, search, median3, sub-pixel,
            pixel field, synthesis, fallback)
  formats   estimate + one synthesis (t = 1/2) in Rgb10, RgbaF16 linear, Nv12 and P010
  blur      one motion-blurred frame (4 Gaussian samples over [1/4, 3/4]) of an Rgba8 pair
  seednet   the estimate with the shipped seed net at level 1 (the fused tcgen05 forward)
  ui        CrosshairV2: observe, estimate with the estimate fill, synthesis with warp-tap rejection and paste-back
  train     one seed-net training step on 24 crops of 256 x 256 (fused forward, tcgen05 gradients, Adam)
"""
import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import framegen as fg  # noqa: E402
import workloads  # noqa: E402


def pair_frames(W, H):
    p, c, _ = workloads.flow_pair(W, H, seed=4 * 10 ** 6)
    return p, c


def dev(x):
    if isinstance(x, tuple):
        return tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in x)
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def like(d):
    return tuple(torch.zeros_like(q) for q in d) if isinstance(d, tuple) else torch.zeros_like(d)


def run(I, a, c, ts):
    I.begin_frame()
    assert I.record_estimate(a, c), I.last_error()
    for t in ts:
        o = like(a)
        assert I.record_synth(a, c, o, t), I.last_error()


def case_pair(W, H, settings=None):
    p, c = pair_frames(W, H)
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=settings), I.init_error()
    run(I, dev(p), dev(c), (0.25, 0.5, 0.75))
    torch.cuda.synchronize()
    I.close()


def case_formats(W, H):
    p, c = pair_frames(W, H)
    kinds = (
        (fg.VK_A2B10G10R10_UNORM, {}, lambda f: workloads.to_rgb10(f).view(np.int32)),
        (fg.VK_R16G16B16A16_SFLOAT, {"transfer": 1}, lambda f: workloads.to_f16(f).view(np.int16)),
        (fg.VK_R8_UNORM, {"yuv_matrix": 1}, lambda f: workloads.to_yuv(f, 8)),
        (fg.VK_R16_UNORM, {"yuv_matrix": 1},
         lambda f: tuple(q.view(np.int16) for q in workloads.to_yuv(f, 10))),
    )
    for vk, extra, enc in kinds:
        I = fg.Interpolator()
        assert I.init(W, H, vk, **extra), I.init_error()
        run(I, dev(enc(p)), dev(enc(c)), (0.5,))
        torch.cuda.synchronize()
        I.close()


def case_blur(W, H):
    p, c = pair_frames(W, H)
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=fg.Settings(blurSamples=4)), I.init_error()
    a, b = dev(p), dev(c)
    I.begin_frame()
    assert I.record_estimate(a, b)
    o = torch.empty_like(a)
    assert I.record_synth_blur(a, b, o, 0.25, 0.75), I.last_error()
    torch.cuda.synchronize()
    I.close()


def case_seednet(W, H):
    p, c = pair_frames(W, H)
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM), I.init_error()
    assert I.set_seed_net(np.fromfile(os.path.join(HERE, "seednet_l1.bin"), np.float32), 1)
    run(I, dev(p), dev(c), (0.5,))
    torch.cuda.synchronize()
    I.close()


def case_ui(W, H):
    p, c = pair_frames(W, H)
    for f in (p, c):   # a static crosshair in the middle
        f[H // 2 - 1:H // 2 + 1, W // 2 - 40:W // 2 + 40, :3] = (0, 255, 255)
        f[H // 2 - 40:H // 2 + 40, W // 2 - 1:W // 2 + 1, :3] = (0, 255, 255)
    s = fg.Settings(uiProtection=3, uiBoxWidth=128, uiBoxHeight=128, uiEstimateFill=True)
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=s), I.init_error()
    a, b = dev(p), dev(c)
    for f in (a, b, a, b):
        I.begin_frame()
        assert I.record_observe(f), I.last_error()
    run(I, a, b, (0.5,))
    torch.cuda.synchronize()
    I.close()


def case_train():
    import seednet_train as st
    import workloads_gpu
    batch = 24
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    net = fg.SeedNet(batch, st.CROP // 4, st.CROP // 4)
    net.set_params(st.init_params(5))
    lab = st.Labeller(batch)
    d = workloads_gpu.flow_batch(batch, st.CROP, st.CROP, gen, vmax=48.0)
    la, lc, v1 = lab(d["prev"], d["curr"])
    x = fg.SeedNet.pack(la.contiguous(), lc.contiguous())
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.backward(x, st.targets(d["v"], d["kind"], v1), loss)
    net.adam(1e-3)
    torch.cuda.synchronize()
    assert net.fused_errors() == 0
    net.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True, choices=("pair", "formats", "blur", "seednet", "ui", "train"))
    ap.add_argument("--size", default="3840x2160")
    a = ap.parse_args()
    W, H = (int(v) for v in a.size.split("x"))
    import build
    build.build()
    {"pair": lambda: case_pair(W, H), "formats": lambda: case_formats(W, H), "blur": lambda: case_blur(W, H),
     "seednet": lambda: case_seednet(W, H), "ui": lambda: case_ui(W, H), "train": case_train}[a.case]()
    print(f"{a.case}: ok")


if __name__ == "__main__":
    main()
