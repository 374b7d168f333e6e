"""CPU float64 reference of the seed proposer (frame-gen-ritz_b200/csrc/fg_seednet.cu), for its tests.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA net's forward pass (logits), gradients and Adam step. The product
never imports it.

The net: 6 3x3 convolutions, zero padding 1, strides 2, 2, 2, 1, 1, 1, channels 2 -> 32 -> 32 -> 32 -> 32 -> 32 -> 8,
ReLU after the first five; input (luma - 128) / 64 of (prev, curr); output per block (c1x, c1y, c2x, c2y, confidence
logit, 3 unused). Flat parameters: per layer weights [cout][3 ky + kx][cin] then biases [cout]. The loss per block
(weight w): w [huber(c1 - truth) + huber(c2 - search) + BCE(logit, |c1 - truth|_inf < 1)], averaged over the blocks.
This module computes all of it in float64 with torch on the CPU (autograd for the gradients).
"""
import numpy as np
import torch

CIN = [2, 32, 32, 32, 32, 32]
COUT = [32, 32, 32, 32, 32, 8]
STRIDE = [2, 2, 2, 1, 1, 1]


def offsets():
    """(weight offset, bias offset) per layer in the flat parameter array, and the total count"""
    o, res = 0, []
    for ci, co in zip(CIN, COUT):
        res.append((o, o + co * 9 * ci))
        o += co * (9 * ci + 1)
    return res, o


N_PARAMS = offsets()[1]


def bf16_round(a):
    """float32 -> the nearest bfloat16 (ties to even), returned as float32"""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


def init_params(seed=0):
    """He-uniform weights, zero biases (float32)"""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for (wo, bo), ci, co in zip(offsets()[0], CIN, COUT):
        lim = np.sqrt(6.0 / (9 * ci))
        p[wo:bo] = rng.uniform(-lim, lim, co * 9 * ci).astype(np.float32)
    return p


def unflatten(p, dtype=torch.float64, bf16_weights=True):
    """flat parameters -> [(weight (cout, cin, 3, 3), bias (cout,))] as torch tensors; weights rounded to bf16 as the
    forward kernel reads them"""
    res = []
    for (wo, bo), ci, co in zip(offsets()[0], CIN, COUT):
        w = p[wo:bo].reshape(co, 3, 3, ci)
        if bf16_weights:
            w = bf16_round(w)
        w = torch.tensor(np.ascontiguousarray(w.transpose(0, 3, 1, 2)), dtype=dtype, requires_grad=True)
        b = torch.tensor(p[bo:bo + co], dtype=dtype, requires_grad=True)
        res.append((w, b))
    return res


def pack(luma_prev, luma_curr):
    """the net input of a luma pair (B, h, w) float32: ((v - 128) / 64 in bf16) as (B, 2, h, w) float64"""
    a = bf16_round((np.asarray(luma_prev, np.float32) - np.float32(128.0)) * np.float32(1.0 / 64.0))
    c = bf16_round((np.asarray(luma_curr, np.float32) - np.float32(128.0)) * np.float32(1.0 / 64.0))
    return torch.tensor(np.stack([a, c], axis=1), dtype=torch.float64)


def forward(params, x):
    """x (B, 2, h, w) -> output (B, bh, bw, 8), float64"""
    h = x
    for l, (w, b) in enumerate(params):
        h = torch.nn.functional.conv2d(h, w, b, stride=STRIDE[l], padding=1)
        if l < 5:
            h = torch.relu(h)
    return h.permute(0, 2, 3, 1)


def loss(out, tgt):
    """the training loss of an output (B, bh, bw, 8) against targets (B, bh, bw, 6), both float64 tensors"""
    wgt = tgt[..., 4]
    e = out[..., :4] - tgt[..., :4]
    ae = e.abs()
    hub = torch.where(ae < 1, 0.5 * e * e, ae - 0.5).sum(-1)
    y = (ae[..., :2].amax(-1) < 1).to(out.dtype)
    z = out[..., 4]
    bce = torch.clamp(z, min=0) - z * y + torch.log1p(torch.exp(-z.abs()))
    return (wgt * (hub + bce)).sum() / wgt.numel()


def grads(p, x, tgt):
    """flat float64 gradient of the loss with respect to the flat parameters (through the bf16-rounded weights)"""
    params = unflatten(p)
    lo = loss(forward(params, x), torch.tensor(tgt, dtype=torch.float64))
    lo.backward()
    g = np.zeros(N_PARAMS, np.float64)
    for (wo, bo), (w, b), co in zip(offsets()[0], params, COUT):
        g[wo:bo] = w.grad.numpy().transpose(0, 2, 3, 1).reshape(-1)
        g[bo:bo + co] = b.grad.numpy()
    return g, float(lo.detach())


def adam(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """one Adam step in float64 (the returned parameters, moments)"""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh, vh = m / (1 - b1 ** step), v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
