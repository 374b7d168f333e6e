"""Seeded synthetic frame pairs for the V1 path (numpy only, deterministic across machines for a numpy version).

The reference measures on real footage that it does not ship; these generators stand in for it with the shapes, sizes
and motion statistics of the workloads the path is measured on:

  pan_pair        640x360 Rgba8: 5-octave value-noise texture, curr = bilinear shift (+5.25, -2.50) px, a 64x64
                  noise sprite moving (-12, +7) px, a constant 80x20 flat HUD at the top-left.
  flow_pair       1920x1080 (any size) Rgba8: the same texture, a smooth per-pixel motion field from 2-octave
                  low-frequency noise with |v| <= 24 px applied by bilinear backward warp; kind "cut" (two independent
                  textures) and "fresh" (20 % of the area replaced by fresh noise) exercise the fallbacks. Returns the
                  ground-truth frame at t as well (rendered from the same field).
  flow_pair_seq   the 500-pair sequence of flow_pair with 5 % cuts and 5 % fresh pairs, seed = stream * 10**6 + pair.

Frames are (H, W, 4) uint8 in R,G,B,A order, alpha 255.
"""
import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _bilinear(img, x, y):
    """Sample img (H, W, C) float at float coords (x, y) with clamped taps (edge replicate)."""
    H, W = img.shape[:2]
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    fx = (x - x0)[..., None]
    fy = (y - y0)[..., None]
    x1, y1 = np.clip(x0 + 1, 0, W - 1), np.clip(y0 + 1, 0, H - 1)
    x0, y0 = np.clip(x0, 0, W - 1), np.clip(y0, 0, H - 1)
    top = img[y0, x0] * (1 - fx) + img[y0, x1] * fx
    bot = img[y1, x0] * (1 - fx) + img[y1, x1] * fx
    return top * (1 - fy) + bot * fy


def value_noise(h, w, rng, octaves=5, base=96.0, channels=3):
    """Sum of `octaves` bilinear value-noise layers, periods base / 2^k, amplitudes 1 / 2^k; float in [0, 1]."""
    acc = np.zeros((h, w, channels), np.float64)
    tot = 0.0
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    for k in range(octaves):
        p = base / (2 ** k)
        gh, gw = int(np.ceil(h / p)) + 2, int(np.ceil(w / p)) + 2
        grid = rng.random((gh, gw, channels))
        amp = 0.5 ** k
        acc += amp * _bilinear(grid, xs / p, ys / p)
        tot += amp
    acc /= tot
    lo, hi = acc.min(), acc.max()
    return (acc - lo) / max(hi - lo, 1e-9)


def _to_rgba(f):
    rgb = np.clip(np.rint(f * 255.0), 0, 255).astype(np.uint8)
    return np.concatenate([rgb, np.full(rgb.shape[:2] + (1,), 255, np.uint8)], axis=2)


def _shift(img, dx, dy):
    """Content moved by (dx, dy): out(p) = img(p - d), bilinear, edge replicate."""
    H, W = img.shape[:2]
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    return _bilinear(img, xs - dx, ys - dy)


def pan_pair(W=640, H=360, seed=0):
    """The 640x360 2x workload (one pair): returns (prev, curr) RGBA8."""
    rng = _rng(seed)
    tex = value_noise(H, W, rng)
    prev = tex.copy()
    curr = _shift(tex, 5.25, -2.50)
    n = min(64, W // 4, H // 4)   # 64 at the workload's size; smaller frames get a smaller sprite
    sprite = value_noise(n, n, rng, octaves=3, base=16.0)
    sx, sy = max(W // 2 - n // 2, 12), max(H // 2 - n // 2, 0)
    prev[sy:sy + n, sx:sx + n] = sprite
    curr[sy + 7:sy + 7 + n, sx - 12:sx - 12 + n] = sprite[:max(0, min(n, H - sy - 7))]
    hud = rng.random(3)
    prev[8:28, 8:88] = hud
    curr[8:28, 8:88] = hud
    return _to_rgba(prev), _to_rgba(curr)


def motion_field(H, W, rng, vmax=24.0):
    """Smooth per-pixel motion (H, W, 2) from 2-octave low-frequency noise, |v| <= vmax."""
    n = value_noise(H, W, rng, octaves=2, base=max(H, W) / 3.0, channels=2) * 2.0 - 1.0
    mag = np.sqrt((n ** 2).sum(-1, keepdims=True))
    scale = vmax / max(float(mag.max()), 1e-9)
    return n * scale


def flow_pair(W=1920, H=1080, seed=0, kind="normal", t=0.5):
    """A pair whose content moves along a smooth field v: prev(p) = T(p), curr(p) = T(p - v(p)), the ground truth at
    time t is T(p - t v(p)). kind: "normal", "cut" (curr is an independent texture), "fresh" (20 % of curr's area is
    fresh noise). Returns (prev, curr, truth_at_t) RGBA8."""
    rng = _rng(seed)
    tex = value_noise(H, W, rng)
    v = motion_field(H, W, rng)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    prev = tex
    curr = _bilinear(tex, xs - v[..., 0], ys - v[..., 1])
    truth = _bilinear(tex, xs - t * v[..., 0], ys - t * v[..., 1])
    if kind == "cut":
        curr = value_noise(H, W, rng)
    elif kind == "fresh":
        fh, fw = int(H * np.sqrt(0.2)), int(W * np.sqrt(0.2))
        y0, x0 = int(rng.integers(0, H - fh + 1)), int(rng.integers(0, W - fw + 1))
        curr = curr.copy()
        curr[y0:y0 + fh, x0:x0 + fw] = rng.random((fh, fw, 3))
    return _to_rgba(prev), _to_rgba(curr), _to_rgba(truth)


def pair_kind(stream, pair):
    """The kind of pair `pair` of a sequence: 5 % cuts, 5 % fresh, the rest normal (seeded per pair)."""
    r = _rng(stream * 10 ** 6 + pair).random()
    return "cut" if r < 0.05 else ("fresh" if r < 0.10 else "normal")


def flow_pair_seq(stream, pair, W=1920, H=1080, t=0.5):
    return flow_pair(W, H, seed=stream * 10 ** 6 + pair, kind=pair_kind(stream, pair), t=t)


def contrast_texture(H, W, rng, cell=6):
    """High-contrast texture: random 0 / 255 cells of `cell` px, per channel (scene cuts between two of them exceed
    the default scene-cut SAD)."""
    gh, gw = -(-H // cell), -(-W // cell)
    g = (rng.random((gh, gw, 3)) < 0.5).astype(np.float64)
    return np.repeat(np.repeat(g, cell, 0), cell, 1)[:H, :W]


def contrast_pair(W=160, H=96, seed=0, kind="cut"):
    """kind "cut": two independent high-contrast textures (a scene cut); "noisy": a (3, -2) px pan of one with
    strong per-pixel noise on curr (mismatch high everywhere: the untrusted-share fallback)."""
    rng = _rng(seed)
    a = contrast_texture(H, W, rng)
    if kind == "cut":
        c = contrast_texture(H, W, rng)
    else:
        c = np.clip(_shift(a, 3, -2) * 0.6 + 0.2 + rng.normal(0, 0.12, a.shape), 0, 1)
    return _to_rgba(a), _to_rgba(c)


# ---------------------------------------------------------------------------------------------- other frame formats
# Conversions of the 8-bit RGBA pairs above into the library's other formats (framegen::Format), deterministic per
# pixel value so a pair keeps its motion: Rgb10 words, RgbaF16 (linear light log-uniform in 1e-3..10, or display
# encoded), Nv12 / P010 planes (BT.601 / 709 / 2020, limited or full range, 4:2:0 chroma from 2x2 means).
_KR_KB = {"bt601": (0.299, 0.114), "bt709": (0.2126, 0.0722), "bt2020": (0.2627, 0.0593)}


def to_rgb10(rgba, r_high=False):
    """(H, W) uint32 A2B10G10R10 words (A2R10G10B10 with r_high): code = 4 v + (v >> 6), alpha 3."""
    v = rgba[..., :3].astype(np.uint32)
    c = 4 * v + (v >> 6)
    r, g, b = c[..., 0], c[..., 1], c[..., 2]
    lo, hi = (b, r) if r_high else (r, b)
    return (np.uint32(3) << 30) | (hi << 20) | (g << 10) | lo


def to_f16(rgba, linear=True):
    """(H, W, 4) float16: linear light 10^(-3 + 4 v / 255) (log-uniform in 1e-3..10), or encoded v / 255; alpha 1."""
    v = rgba[..., :3].astype(np.float64) / 255.0
    rgb = 10.0 ** (-3.0 + 4.0 * v) if linear else v
    out = np.empty(rgba.shape[:2] + (4,), np.float16)
    out[..., :3] = rgb.astype(np.float16)
    out[..., 3] = 1.0
    return out


def to_yuv(rgba, bits=8, matrix="bt709", full_range=False):
    """(Y, CbCr) planes: Nv12 (bits 8: uint8) or P010 (bits 10: uint16 words, the code in the high 10 bits).
    Y' = kr R' + kg G' + kb B', Cb = (B' - Y') / (2 (1 - kb)), Cr = (R' - Y') / (2 (1 - kr)); chroma = the mean of
    each 2x2 block (edge pixels repeated for odd sizes)."""
    kr, kb = _KR_KB[matrix]
    kg = 1.0 - kr - kb
    e = rgba[..., :3].astype(np.float64) / 255.0
    y = kr * e[..., 0] + kg * e[..., 1] + kb * e[..., 2]
    cb = (e[..., 2] - y) / (2.0 * (1.0 - kb))
    cr = (e[..., 0] - y) / (2.0 * (1.0 - kr))
    H, W = y.shape
    ph, pw = H + (H & 1), W + (W & 1)
    cbp = np.pad(cb, ((0, ph - H), (0, pw - W)), mode="edge")
    crp = np.pad(cr, ((0, ph - H), (0, pw - W)), mode="edge")
    cbm = cbp.reshape(ph // 2, 2, pw // 2, 2).mean(axis=(1, 3))
    crm = crp.reshape(ph // 2, 2, pw // 2, 2).mean(axis=(1, 3))
    q = 1 << (bits - 8)
    top = (1 << bits) - 1
    if full_range:
        yc, cbc, crc = y * top, 128 * q + cbm * top, 128 * q + crm * top
    else:
        yc, cbc, crc = 16 * q + 219 * q * y, 128 * q + 224 * q * cbm, 128 * q + 224 * q * crm
    Y = np.clip(np.rint(yc), 0, top).astype(np.uint32)
    C = np.stack([np.clip(np.rint(cbc), 0, top), np.clip(np.rint(crc), 0, top)], axis=2).astype(np.uint32)
    if bits == 8:
        return Y.astype(np.uint8), C.astype(np.uint8)
    return (Y << 6).astype(np.uint16), (C << 6).astype(np.uint16)
