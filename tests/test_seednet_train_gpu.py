"""Training the seed proposer on the GPU with the library's own kernels (the fused tcgen05 forward that keeps every
layer's output, the tcgen05 weight / input gradients, the loss and Adam), and what the trained net gains.

The workload is one where the net can matter: smooth motion of up to 48 px (the generator's 24 px doubled), so the
level-1 half-vectors reach 6 and the zero seed's radius-2 search at level 1 cannot find most of them. A fresh net is
trained for 250 steps of 24 crops (256 x 256, labels as seednet_train.py makes them), then three arms synthesize 6
held-out 512 x 512 pairs at t = 1/4, 1/2, 3/4 and are scored by PSNR against the generator's ground truth:
  cnn   the trained net at level 1 (the level above skipped, equal radii below);
  zero  the same truncated pyramid with a net whose outputs are all zero (the method without the net);
  plain the full V1 pyramid.
Asserted: the training loss falls by more than a quarter in these few steps, and cnn beats zero by at least 0.5 dB
(the gain, and its sign, are printed beside plain's; measured on a B200: loss 3.65 -> 2.33, cnn 42.96 dB, zero
41.18 dB, a gain of +1.78 dB, plain 43.48 dB).
"""
import numpy as np
import pytest
import torch

import framegen as fg

pytestmark = pytest.mark.gpu

TS = (0.25, 0.5, 0.75)


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def psnr(a, b):
    mse = float(((a[..., :3].float() - b[..., :3].float()) ** 2).mean())
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)


def test_training_gains_over_the_zero_seed():
    import seednet_train as st
    import workloads_gpu
    batch, steps, vmax = 24, 250, 48.0
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    net = fg.SeedNet(batch, st.CROP // 4, st.CROP // 4)
    net.set_params(st.init_params(5))
    lab = st.Labeller(batch)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    losses = []
    for step in range(steps):
        d = workloads_gpu.flow_batch(batch, st.CROP, st.CROP, gen, vmax=vmax)
        la, lc, v1 = lab(d["prev"], d["curr"])
        x = fg.SeedNet.pack(la.contiguous(), lc.contiguous())
        net.backward(x, st.targets(d["v"], d["kind"], v1), loss)
        net.adam(1e-3)
        if step < 10 or step >= steps - 10:
            torch.cuda.synchronize()
            losses.append(float(loss))
    assert net.fused_errors() == 0
    params = net.params()
    net.close()
    first, last = float(np.mean(losses[:10])), float(np.mean(losses[-10:]))
    W = H = 512
    arms = {}
    for name, p in (("cnn", params), ("zero", np.zeros_like(params)), ("plain", None)):
        I = fg.Interpolator()
        assert I.init(W, H, fg.VK_R8G8B8A8_UNORM), I.init_error()
        if p is not None:
            assert I.set_seed_net(p, 1)
        arms[name] = I
    gen.manual_seed(987654)
    o = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    score = {k: [] for k in arms}
    for _ in range(6):
        d = workloads_gpu.flow_batch(1, W, H, gen, ts=TS, vmax=vmax, cut_frac=0.0, fresh_frac=0.0)
        a, c = d["prev"][0].contiguous(), d["curr"][0].contiguous()
        for name, I in arms.items():
            I.begin_frame()
            assert I.record_estimate(a, c), I.last_error()
            for t in TS:
                assert I.record_synth(a, c, o, t)
                torch.cuda.synchronize()
                score[name].append(psnr(o, d["truth"][t][0]))
    for I in arms.values():
        I.close()
    m = {k: float(np.mean(v)) for k, v in score.items()}
    print(f"training loss {first:.3f} -> {last:.3f}; PSNR cnn {m['cnn']:.2f} dB, zero {m['zero']:.2f} dB "
          f"(gain {m['cnn'] - m['zero']:+.2f} dB), plain {m['plain']:.2f} dB")
    assert last < 0.75 * first
    assert m["cnn"] - m["zero"] >= 0.5
