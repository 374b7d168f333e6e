"""The seed proposer's CUDA kernels (fg_seednet_*) against the float64 CPU reference (oracle/seednet_ref.py).

The net computes in bfloat16 (weights, inputs, the activations stored between layers) with float32 accumulation; the
reference is the same net in float64 with the same bf16 weights and inputs. Stated tolerances:
  - logits: max |gpu - fp64| <= 0.03 * max(1, max |fp64|) (bf16 activation rounding, 2^-9 relative per layer);
  - gradients: per layer, relative L2 error <= 0.05 and cosine >= 0.998; loss relative error <= 0.01;
  - the Adam step: float32 against float64 on the GPU's own gradient, rtol 1e-5.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import seednet_ref as ref
import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def level1_lumas(n, size=256, seed=0):
    """(n, size/4, size/4) level-1 luma pairs of smooth-flow pairs (the oracle's luma)"""
    la, lc = [], []
    for i in range(n):
        p, c, _ = workloads.flow_pair(size, size, seed=seed + i)
        est = oracle.estimate(p, c)
        la.append(est["luma"][1][0])
        lc.append(est["luma"][1][1])
    return np.stack(la), np.stack(lc)


def params(seed):
    p = ref.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    for (wo, bo), co in zip(ref.offsets()[0], ref.COUT):
        p[bo:bo + co] = rng.uniform(-0.1, 0.1, co).astype(np.float32)
    return p


def targets(B, bh, bw, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros((B, bh, bw, 6), np.float32)
    t[..., :4] = rng.uniform(-3, 3, (B, bh, bw, 4))
    t[..., 4] = 1.0
    return t


def test_param_count():
    assert fg.lib().fg_seednet_param_count() == ref.N_PARAMS == 39912


def test_forward_matches_fp64():
    la, lc = level1_lumas(2)
    p = params(1)
    net = fg.SeedNet(4, 64, 64)
    net.set_params(p)
    x = fg.SeedNet.pack(torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda())
    xr = ref.pack(la, lc)
    assert np.array_equal(x.float().cpu().numpy(), xr.permute(0, 2, 3, 1).numpy().astype(np.float32)), "packed input"
    out = net.forward(x)
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    want = ref.forward(ref.unflatten(p), xr).detach().numpy()
    assert got.shape == want.shape == (2, 8, 8, 8)
    err, scale = np.abs(got - want).max(), np.abs(want).max()
    assert err <= 0.03 * max(1.0, scale), f"logit error {err:.4g} at scale {scale:.3g}"
    net.close()


@pytest.mark.parametrize("shape", [(2, 64, 64), (3, 37, 51)])
def test_gradients_match_fp64(shape):
    B, h, w = shape
    rng = np.random.default_rng(5)
    if (h, w) == (64, 64):
        la, lc = level1_lumas(B, seed=10)
    else:   # odd sizes: the ceil grids and the zero padding at every edge
        la = (rng.random((B, h, w)) * 255).astype(np.float32)
        lc = np.roll(la, 2, axis=2)
    p = params(2)
    bh, bw = (h + 7) // 8, (w + 7) // 8
    tgt = targets(B, bh, bw, 3)
    net = fg.SeedNet(4, 64, 64)
    net.set_params(p)
    x = fg.SeedNet.pack(torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda())
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.backward(x, torch.from_numpy(tgt).cuda(), loss)
    torch.cuda.synchronize()
    g = net.grads().astype(np.float64)
    gr, lr_ = ref.grads(p, ref.pack(la, lc), tgt)
    assert abs(float(loss) - lr_) <= 0.01 * abs(lr_), (float(loss), lr_)
    for l, ((wo, bo), co) in enumerate(zip(ref.offsets()[0], ref.COUT)):
        for name, sl in (("weights", slice(wo, bo)), ("biases", slice(bo, bo + co))):
            a, b = g[sl], gr[sl]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
            cos = float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
            assert rel <= 0.05 and cos >= 0.998, f"layer {l + 1} {name}: rel {rel:.3g} cos {cos:.5f}"
    net.close()


def test_adam_step():
    la, lc = level1_lumas(2, seed=20)
    p = params(4)
    tgt = targets(2, 8, 8, 5)
    net = fg.SeedNet(2, 64, 64)
    net.set_params(p)
    x = fg.SeedNet.pack(torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda())
    net.backward(x, torch.from_numpy(tgt).cuda())
    g = net.grads().astype(np.float64)
    net.adam(1e-3)
    torch.cuda.synchronize()
    got = net.params()
    want, _, _ = ref.adam(p.astype(np.float64), 0.0, 0.0, g, 1, 1e-3)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-7), np.abs(got - want).max()
    assert not net.grads().any(), "the step zeroes the gradient"
    net.close()


def test_grad_buffer_and_scaled_step():
    """the data-parallel hooks: grad_buffer() is the accumulator itself (a write through it is what the step reads),
    and adam(grad_scale=s) on a summed gradient equals adam() on the gradient times s, bit for bit when s is a power
    of two (two ranks: sum / 2 is the mean)"""
    la, lc = level1_lumas(2, seed=21)
    p = params(8)
    tgt = targets(2, 8, 8, 9)
    x = fg.SeedNet.pack(torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda())
    a, b = fg.SeedNet(2, 64, 64), fg.SeedNet(2, 64, 64)
    for net in (a, b):
        net.set_params(p)
        net.backward(x, torch.from_numpy(tgt).cuda())
    torch.cuda.synchronize()
    ga, gb = a.grad_buffer(), b.grad_buffer()
    assert ga.dtype == torch.float32 and ga.numel() == ref.N_PARAMS
    assert np.array_equal(ga.cpu().numpy(), a.grads())
    ga.mul_(2.0)                        # what an all-reduce sum of two equal ranks leaves
    a.adam(1e-3, grad_scale=0.5)
    b.adam(1e-3)
    torch.cuda.synchronize()
    assert np.array_equal(a.params(), b.params())
    assert not ga.any() and not gb.any(), "the step zeroes the buffer"
    a.close()
    b.close()


def test_training_lowers_the_loss():
    """200 Adam steps on one fixed batch: the loss falls well below its start (the kernels train the net)"""
    la, lc = level1_lumas(8, seed=30)
    tgt = targets(8, 8, 8, 6)
    tgt[..., :4] *= 0.5
    net = fg.SeedNet(8, 64, 64)
    net.set_params(ref.init_params(7))
    x = fg.SeedNet.pack(torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda())
    t = torch.from_numpy(tgt).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    hist = []
    for i in range(200):
        net.backward(x, t, loss)
        net.adam(1e-3)
        if i % 50 == 0 or i == 199:
            torch.cuda.synchronize()
            hist.append(float(loss))
    assert hist[-1] < 0.5 * hist[0], hist
    net.close()


def test_forward_from_luma_equals_packed_forward():
    """fg_seednet_forward_luma (the first layer packing the float luma planes as it reads them) gives the bits of
    fg_seednet_pack + fg_seednet_forward"""
    la, lc = level1_lumas(2, seed=40)
    net = fg.SeedNet(2, 64, 64)
    net.set_params(params(6))
    dla, dlc = torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda()
    a = net.forward(fg.SeedNet.pack(dla, dlc))
    b = net.forward_luma(dla, dlc)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    net.close()


@pytest.mark.parametrize("B,h,w,seed", [(2, 64, 64, 1), (1, 135, 240, 2), (3, 37, 51, 3), (1, 8, 8, 4),
                                        (1, 540, 960, 5)])
def test_fused_forward_matches_layers_and_fp64(B, h, w, seed):
    """The Interpolator's fused forward (two launches, tcgen05 implicit GEMMs with accumulators in tensor memory)
    against the per-layer forward (mma.sync) and the float64 reference. Same bf16 weights, inputs and activation
    rounding; only the f32 accumulation order differs, so an activation can round to the other neighbouring bf16
    now and then. Tolerances: against the per-layer forward max |diff| <= 0.02 * max(1, max |logit|) with the mean
    |diff| below 1e-3 of that scale; against float64 the per-layer forward's own bound (0.03 * scale). The measured
    errors are printed. Sizes: a 256x256 crop's level 1, a 1080p frame's level 1, odd sizes, one block, and a 4K
    frame's level 1 (960x540, 144 encoder tiles)."""
    rng = np.random.default_rng(seed)
    la = (rng.random((B, h, w)) * 255).round(2).astype(np.float32)
    lc = np.roll(la, (1, 2), axis=(1, 2)) + rng.normal(0, 2, (B, h, w)).astype(np.float32)
    p = params(seed)
    net = fg.SeedNet(B, h, w)
    net.set_params(p)
    ta, tc = torch.from_numpy(la).cuda(), torch.from_numpy(lc).cuda()
    fused = net.forward_fused(ta, tc)
    layers = net.forward_luma(ta, tc)
    torch.cuda.synchronize()
    assert net.fused_errors() == 0
    f, l = fused.cpu().numpy().astype(np.float64), layers.cpu().numpy().astype(np.float64)
    scale = max(1.0, np.abs(l).max())
    d = np.abs(f - l)
    print(f"fused vs per-layer: max {d.max():.4g} mean {d.mean():.3g} (scale {scale:.3g})")
    assert d.max() <= 0.02 * scale and d.mean() <= 1e-3 * scale
    if h * w <= 64 * 64 * 4:
        want = ref.forward(ref.unflatten(p), ref.pack(la, lc)).detach().numpy()
        err = np.abs(f - want).max()
        print(f"fused vs float64: max {err:.4g}")
        assert err <= 0.03 * max(1.0, np.abs(want).max())
    net.close()
