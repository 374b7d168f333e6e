"""The smooth-flow pair generator of workloads.py (flow_pair), batched on the GPU with torch (data generation only: training
and evaluating the seed proposer needs hundreds of thousands of pairs, which the numpy generator makes too slowly).

Same construction as workloads.flow_pair: a 5-octave value-noise texture T, a smooth motion field v from 2-octave
low-frequency noise scaled to max |v| = 24 px, prev = T, curr(p) = T(p - v(p)) by bilinear backward warp (edge
replicate), the ground truth at t = T(p - t v(p)); 5 % of pairs are scene cuts (curr an independent texture) and 5 %
have 20 % of curr's area replaced by fresh noise. Random streams are torch's (seeded per batch), not numpy's, so the
pairs are statistically like workloads.flow_pair's, not bit-identical to them.

hdr_pair makes the 4K HDR workload's RgbaF16 linear-light pairs (log-uniform channels, a pan and rigid sprites) at 4K, which the
numpy generators would take minutes for.
"""
import math

import torch


def _bilinear(img, x, y):
    """img (B, H, W, C) float sampled at (x, y) (B, h, w) with clamped taps"""
    B, H, W, C = img.shape
    x0 = torch.floor(x)
    y0 = torch.floor(y)
    fx = (x - x0)[..., None]
    fy = (y - y0)[..., None]
    x0 = x0.long()
    y0 = y0.long()
    x1, y1 = (x0 + 1).clamp(0, W - 1), (y0 + 1).clamp(0, H - 1)
    x0, y0 = x0.clamp(0, W - 1), y0.clamp(0, H - 1)
    flat = img.reshape(B, H * W, C)

    def g(yy, xx):
        idx = (yy * W + xx).reshape(B, -1, 1).expand(-1, -1, C)
        return torch.gather(flat, 1, idx).reshape(B, *x.shape[1:], C)

    top = g(y0, x0) * (1 - fx) + g(y0, x1) * fx
    bot = g(y1, x0) * (1 - fx) + g(y1, x1) * fx
    return top * (1 - fy) + bot * fy


def value_noise(B, h, w, gen, octaves=5, base=96.0, channels=3, device="cuda"):
    """(B, h, w, channels) in [0, 1]: sum of bilinear value-noise octaves (periods base / 2^k, amplitudes 1 / 2^k),
    normalised per image"""
    ys, xs = torch.meshgrid(torch.arange(h, device=device, dtype=torch.float32),
                            torch.arange(w, device=device, dtype=torch.float32), indexing="ij")
    ys, xs = ys.expand(B, h, w), xs.expand(B, h, w)
    acc = torch.zeros(B, h, w, channels, device=device)
    tot = 0.0
    for k in range(octaves):
        p = base / 2 ** k
        gh, gw = int(math.ceil(h / p)) + 2, int(math.ceil(w / p)) + 2
        grid = torch.rand(B, gh, gw, channels, generator=gen, device=device)
        amp = 0.5 ** k
        acc += amp * _bilinear(grid, xs / p, ys / p)
        tot += amp
    acc /= tot
    lo = acc.amin(dim=(1, 2, 3), keepdim=True)
    hi = acc.amax(dim=(1, 2, 3), keepdim=True)
    return (acc - lo) / (hi - lo).clamp_min(1e-9)


def to_rgba(f):
    rgb = torch.clamp(torch.round(f * 255.0), 0, 255).to(torch.uint8)
    return torch.cat([rgb, torch.full(rgb.shape[:3] + (1,), 255, dtype=torch.uint8, device=rgb.device)], dim=3)


def flow_batch(B, W, H, gen, ts=(), vmax=24.0, cut_frac=0.05, fresh_frac=0.05, device="cuda"):
    """B pairs: returns dict prev, curr (B, H, W, 4) uint8, v (B, H, W, 2) float (content displacement prev -> curr,
    px), kind (B,) 0 normal / 1 cut / 2 fresh, truth {t: (B, H, W, 4) uint8}"""
    tex = value_noise(B, H, W, gen, device=device)
    n = value_noise(B, H, W, gen, octaves=2, base=max(H, W) / 3.0, channels=2, device=device) * 2.0 - 1.0
    mag = torch.sqrt((n ** 2).sum(-1)).amax(dim=(1, 2)).clamp_min(1e-9)
    v = n * (vmax / mag)[:, None, None, None]
    ys, xs = torch.meshgrid(torch.arange(H, device=device, dtype=torch.float32),
                            torch.arange(W, device=device, dtype=torch.float32), indexing="ij")
    ys, xs = ys.expand(B, H, W), xs.expand(B, H, W)
    curr = _bilinear(tex, xs - v[..., 0], ys - v[..., 1])
    truth = {t: to_rgba(_bilinear(tex, xs - t * v[..., 0], ys - t * v[..., 1])) for t in ts}
    r = torch.rand(B, generator=gen, device=device)
    kind = torch.where(r < cut_frac, 1, torch.where(r < cut_frac + fresh_frac, 2, 0))
    if bool((kind == 1).any()):
        other = value_noise(B, H, W, gen, device=device)
        curr = torch.where((kind == 1)[:, None, None, None], other, curr)
    if bool((kind == 2).any()):
        fh, fw = int(H * math.sqrt(0.2)), int(W * math.sqrt(0.2))
        for b in torch.nonzero(kind == 2).flatten().tolist():
            y0 = int(torch.randint(0, H - fh + 1, (1,), generator=gen, device=device))
            x0 = int(torch.randint(0, W - fw + 1, (1,), generator=gen, device=device))
            curr[b, y0:y0 + fh, x0:x0 + fw] = torch.rand(fh, fw, 3, generator=gen, device=device)
    return {"prev": to_rgba(tex), "curr": to_rgba(curr), "v": v, "kind": kind, "truth": truth}


def hdr_pair(W, H, gen, pan=16.0, sprites=3, smin=128, smax=384, smove=32.0, device="cuda"):
    """A 4K HDR pair: RgbaF16 linear light (scRGB), prev / curr (H, W, 4) float16 on the device, alpha 1. Each
    channel is log-uniform in 1e-3..10 with 4-octave spatial correlation, 10^(-3 + 4 u) with u 4-octave value noise
    normalised to [0, 1]; the background pans by a uniform (+-pan, +-pan) px and `sprites` rigid squares of side
    smin..smax px (their own textures) move by up to +-smove px, composited over the background in both frames."""
    def rnd(lo, hi):
        return float(lo + (hi - lo) * torch.rand(1, generator=gen, device=device))

    bg = value_noise(1, H + 2 * int(pan) + 2, W + 2 * int(pan) + 2, gen, octaves=4, base=128.0, device=device)[0]
    dx, dy = rnd(-pan, pan), rnd(-pan, pan)
    ys, xs = torch.meshgrid(torch.arange(H, device=device, dtype=torch.float32),
                            torch.arange(W, device=device, dtype=torch.float32), indexing="ij")
    o = float(int(pan) + 1)
    prev = _bilinear(bg[None], (xs + o)[None], (ys + o)[None])[0]
    curr = _bilinear(bg[None], (xs + o - dx)[None], (ys + o - dy)[None])[0]
    for _ in range(sprites):
        s = int(rnd(smin, smax))
        tex = value_noise(1, s, s, gen, octaves=4, base=s / 4.0, device=device)
        x0, y0 = rnd(0, W - s), rnd(0, H - s)
        mx, my = rnd(-smove, smove), rnd(-smove, smove)
        for img, (ox, oy) in ((prev, (x0, y0)), (curr, (x0 + mx, y0 + my))):
            u, v = xs - ox, ys - oy
            inside = (u >= 0) & (u <= s - 1) & (v >= 0) & (v <= s - 1)
            val = _bilinear(tex, u.clamp(0, s - 1)[None], v.clamp(0, s - 1)[None])[0]
            img[inside] = val[inside]

    def lin(u):
        rgb = torch.pow(10.0, -3.0 + 4.0 * u)
        return torch.cat([rgb, torch.ones_like(rgb[..., :1])], dim=-1).to(torch.float16)

    return lin(prev), lin(curr)
