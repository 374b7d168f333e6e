"""CPU oracle for the MotionVersion::V1 path: Python face of oracle/fg_oracle.c (a plain-C restatement of
frame-gen-ritz's proto/interp.py and the OpenCV 4.13 / numpy primitives it calls).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the checker.
The product path never imports it.

Frames are numpy uint8 arrays (H, W, 4) in R,G,B,A order ("rgba"), (H, W, 4) B,G,R,A ("bgra"), or (H, W, 3) in
interp.py's own B,G,R order ("bgr"). Outputs keep the input's layout; alpha is the nearer real frame's.
"""
import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libfg_oracle.so")
ORDERS = {"rgba": 0, "bgra": 1, "bgr": 2}
REASONS = {0: None, 1: "cut", 2: "untrusted"}


@dataclass
class Settings:
    """The V1 fields of framegen::Settings (gpu/framegen.h:167-409) with their defaults, which are the tuned
    constants of proto/interp.py:43-61."""
    trustLow: float = 12.0
    trustHigh: float = 40.0
    globalFallback: float = 0.15
    sceneCutSad: float = 30.0
    hudBonus: float = 1.0
    smoothBonus: float = 0.5
    searchPenalty: float = 0.5
    searchRadius: int = 2
    searchRadiusTop: int = 6
    subpixel: bool = True
    flowScale: int = 2
    pyramidMinSide: int = 48


class _CSettings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("trustLow", "trustHigh", "globalFallback", "sceneCutSad", "hudBonus",
                                              "smoothBonus", "searchPenalty")] + \
               [(n, ctypes.c_int) for n in ("searchRadius", "searchRadiusTop", "subpixel", "flowScale", "pyramidMinSide")]


def _cs(s):
    s = s or Settings()
    return _CSettings(*[getattr(s, n) for n, _ in _CSettings._fields_])


def build():
    """Compile the oracle library (gcc + OpenMP) in place."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.fgo_layout.argtypes = [ctypes.c_int] * 4 + [P] * 4 + [ctypes.c_int]
        L.fgo_layout.restype = ctypes.c_int
        L.fgo_estimate.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_CSettings),
                                   P, P, P, P, P, P, P, P, ctypes.c_int]
        L.fgo_estimate.restype = ctypes.c_int
        L.fgo_estimate_cnn.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_CSettings), ctypes.c_int, P, P, P, P, P, P, P, P, P, ctypes.c_int]
        L.fgo_estimate_cnn.restype = ctypes.c_int
        L.fgo_synth.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_CSettings),
                                P, ctypes.c_int, ctypes.c_float, P, ctypes.c_int, P, P, P, P, ctypes.c_int]
        L.fgo_synth.restype = ctypes.c_int
        L.fgo_synth_ui.argtypes = L.fgo_synth.argtypes + [ctypes.POINTER(_CUiMask), ctypes.POINTER(_CUiMask)]
        L.fgo_synth_ui.restype = ctypes.c_int
        L.fgo_estimate_ui.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(_CSettings), P, P, P, P, P, P, P, P, ctypes.c_int,
                                      ctypes.POINTER(_CUiMask), ctypes.POINTER(_CUiMask)]
        L.fgo_estimate_ui.restype = ctypes.c_int
        L.fgo_mean_f32.argtypes = [P, ctypes.c_long]
        L.fgo_mean_f32.restype = ctypes.c_float
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Layout:
    W: int
    H: int
    fw: int
    fh: int
    levels: list = field(default_factory=list)   # (w, h, bw, bh) per level, finest first


def layout(W, H, flow_scale=2, min_side=48):
    fw, fh = ctypes.c_int(), ctypes.c_int()
    lw, lh = (ctypes.c_int * 16)(), (ctypes.c_int * 16)()
    n = lib().fgo_layout(W, H, flow_scale, min_side, ctypes.byref(fw), ctypes.byref(fh), lw, lh, 16)
    if n < 1:
        raise ValueError("bad size")
    return Layout(W, H, fw.value, fh.value, [(lw[i], lh[i], (lw[i] + 7) // 8, (lh[i] + 7) // 8) for i in range(n)])


def _frame_args(a, order):
    if a.dtype != np.uint8 or a.ndim != 3 or a.shape[2] != (3 if order == "bgr" else 4):
        raise ValueError("frame must be uint8 (H, W, %d)" % (3 if order == "bgr" else 4))
    a = np.ascontiguousarray(a)
    return a, a.shape[1], a.shape[0], a.strides[0]


def estimate(a, c, settings=None, order="rgba", trace=True, threads=0, seed_net=None, ui_fill=None):
    """interp.estimate(a, c) plus every intermediate: returns a dict with sad (the float32 mean as a Python float),
    cut (bool), pf (fh, fw, 2) and, with trace, luma/fields/seeds/meds/sads per level. seed_net = (level, output):
    the CNN-seeded estimate from the seed net's output (bh, bw, 8) at that level (no counterpart in interp.py).
    ui_fill = (prev's mask, curr's mask), each (bytes, rect): CrosshairV2's estimate fill of the level-0 luma."""
    s = settings or Settings()
    a, W, H, pitch = _frame_args(a, order)
    c, _, _, _ = _frame_args(c, order)
    L = layout(W, H, s.flowScale, s.pyramidMinSide)
    nl = sum(2 * w * h for w, h, _, _ in L.levels)
    nf = sum(4 * bw * bh for _, _, bw, bh in L.levels) + 4 * L.levels[0][2] * L.levels[0][3]
    ns = sum(2 * bw * bh for _, _, bw, bh in L.levels)
    luma = np.zeros(nl, np.float32) if trace else None
    fields = np.zeros(nf, np.float32) if trace else None
    seeds = np.zeros(ns, np.float32) if trace else None
    meds = np.zeros(2 * len(L.levels), np.float32) if trace else None
    nb0 = L.levels[0][2] * L.levels[0][3]
    sads = np.zeros(nb0, np.float32)
    pf = np.zeros((L.fh, L.fw, 2), np.float32)
    mean, cut = ctypes.c_float(), ctypes.c_int()
    lvl, cnn = (-1, None) if seed_net is None else (int(seed_net[0]), np.ascontiguousarray(seed_net[1], np.float32))
    if ui_fill is not None:
        (ma, ka), (mc, kc) = _uimask(ui_fill[0]), _uimask(ui_fill[1])
        n = lib().fgo_estimate_ui(_p(a), _p(c), W, H, pitch, ORDERS[order], ctypes.byref(_cs(s)), _p(luma), _p(fields),
                                  _p(seeds), _p(meds), _p(sads), _p(pf), ctypes.byref(mean), ctypes.byref(cut), threads,
                                  ctypes.byref(ma) if ma else None, ctypes.byref(mc) if mc else None)
    else:
        n = lib().fgo_estimate_cnn(_p(a), _p(c), W, H, pitch, ORDERS[order], ctypes.byref(_cs(s)), lvl, _p(cnn),
                                   _p(luma), _p(fields), _p(seeds), _p(meds), _p(sads), _p(pf), ctypes.byref(mean),
                                   ctypes.byref(cut), threads)
    if n != len(L.levels):
        raise RuntimeError("fgo_estimate failed")
    est = {"sad": float(mean.value), "cut": bool(cut.value), "pf": pf, "layout": L,
           "sads": sads.reshape(L.levels[0][3], L.levels[0][2])}
    if trace:
        lum, fl, sd = [], [], []
        o = of = os_ = 0
        for w, h, bw, bh in L.levels:
            lum.append((luma[o:o + w * h].reshape(h, w), luma[o + w * h:o + 2 * w * h].reshape(h, w)))
            o += 2 * w * h
            fl.append((fields[of:of + 2 * bw * bh].reshape(bh, bw, 2), fields[of + 2 * bw * bh:of + 4 * bw * bh].reshape(bh, bw, 2)))
            of += 4 * bw * bh
            sd.append(seeds[os_:os_ + 2 * bw * bh].reshape(bh, bw, 2))
            os_ += 2 * bw * bh
        bw0, bh0 = L.levels[0][2], L.levels[0][3]
        est["luma"] = lum
        est["fields"] = fl
        est["seeds"] = sd
        est["meds"] = meds.reshape(-1, 2)
        est["sub"] = [fields[of:of + 2 * bw0 * bh0].reshape(bh0, bw0, 2), fields[of + 2 * bw0 * bh0:].reshape(bh0, bw0, 2)]
        est["v"] = est["sub"][1] if s.subpixel else fl[0][1]
    return est


class _CUiMask(ctypes.Structure):   # fgo_uimask: a UI mask over its rectangle
    _fields_ = [("m", ctypes.c_void_p), ("x", ctypes.c_int), ("y", ctypes.c_int), ("w", ctypes.c_int),
                ("h", ctypes.c_int), ("stride", ctypes.c_int)]


def _uimask(m):
    """(mask bytes (h, w), (x, y, w, h)) -> (fgo_uimask, the array it points into), or (None, None)"""
    if m is None:
        return None, None
    mask, (x, y, w, h) = m
    mask = np.ascontiguousarray(mask, np.uint8)
    return _CUiMask(mask.ctypes.data, x, y, w, h, mask.strides[0]), mask


def synth(a, c, est, t, settings=None, order="rgba", trace=False, threads=0, ui=None):
    """interp.synth(a, c, est, t, why=True): returns (frame, reason) or, with trace, a dict that adds field_t,
    e (the per-pixel mismatch before the 7x7 box) and untrusted (pixels whose trust is past 0.5).
    ui = (prev's mask, curr's mask), each (bytes, rect) or None: CrosshairV2's warp-tap rejection (no paste-back here;
    ui_v2.patch does that)."""
    s = settings or Settings()
    a, W, H, pitch = _frame_args(a, order)
    c, _, _, _ = _frame_args(c, order)
    out = np.zeros_like(a)
    L = est["layout"]
    pf = np.ascontiguousarray(est["pf"], np.float32)
    ft = np.zeros((L.fh, L.fw, 2), np.float32) if trace else None
    e = np.zeros((H, W), np.uint8) if trace else None
    unt, reason = ctypes.c_longlong(), ctypes.c_int()
    args = (_p(a), _p(c), W, H, pitch, ORDERS[order], ctypes.byref(_cs(s)), _p(pf), int(est["cut"]), float(t), _p(out),
            out.strides[0], _p(ft), _p(e), ctypes.byref(unt), ctypes.byref(reason), threads)
    if ui is not None:
        (ma, ka), (mc, kc) = _uimask(ui[0]), _uimask(ui[1])
        r = lib().fgo_synth_ui(*args, ctypes.byref(ma) if ma else None, ctypes.byref(mc) if mc else None)
    else:
        r = lib().fgo_synth(*args)
    if r != 0:
        raise ValueError("fgo_synth failed (t outside (0, 1)?)")
    if trace:
        return {"out": out, "reason": REASONS[reason.value], "field_t": ft, "e": e, "untrusted": int(unt.value)}
    return out, REASONS[reason.value]


# ---------------------------------------------------------------------------------------------- motion blur
# recordSynthBlur (gpu/framegen.h:553-573, gpu/framegen.cpp:3534-3630): the weighted average of N sub-frames, each
# exactly the frame recordSynth(t_k) gives. The reference's own check of it (gpu/blurtest.cpp:602-620, 757-806) takes
# the sub-frames, weights them in double precision and rounds half up, allowing 1 level. This restatement fixes the
# rounding: the normalised weights in units of 2^-16 (largest remainders), out = (sum q_k v_k + 2^15) >> 16.

def blur_plan(samples, gaussian, t0, t1):
    """(times as float32, weights q_k in units of 2^-16) of a blur over [t0, t1], or None if refused. Times: the
    midpoints t0 + (t1 - t0)(k + 0.5) / N in double, rounded to float32 and clamped to [t0, t1]
    (gpu/framegen.cpp:3552-3557); N < 2 or t0 == t1: the single instant t1. Weights: 1 (even) or exp(-2 x_k^2),
    x_k = (2k + 1 - N) / N (gpu/blurtest.cpp:610-620, gpu/shaders/blur_resolve.comp:135-140)."""
    t0, t1 = np.float32(t0), np.float32(t1)
    if not (t0 >= 0 and t1 <= 1 and t0 <= t1):
        return None
    on = samples >= 2 and t0 < t1
    n = min(int(samples), 16) if on else 1
    d0, d1 = float(t0), float(t1)
    times, w, tot_w = [], [], 0.0
    for k in range(n):
        t = d0 + (d1 - d0) * (k + 0.5) / n if on else d1
        times.append(min(max(np.float32(t), t0), t1))
        x = (2.0 * k + 1.0 - n) / n
        w.append(math.exp(-2.0 * x * x) if gaussian else 1.0)
        tot_w += w[-1]
    q, frac = [], []
    for v in w:
        r = v / tot_w * 65536.0
        q.append(math.floor(r))
        frac.append(r - q[-1])
    tot = sum(q)
    while tot != 65536:   # the remaining units to the largest remainders, ties to the lower sample
        best = 0
        for k in range(1, n):
            if (frac[k] > frac[best]) if tot < 65536 else (frac[k] < frac[best]):
                best = k
        if tot < 65536:
            q[best] += 1
            frac[best] -= 1.0
            tot += 1
        else:
            q[best] -= 1
            frac[best] += 1.0
            tot -= 1
    return np.array(times, np.float32), q


def blur_subframes(a, c, est, t0, t1, samples, gaussian, settings=None, order="rgba"):
    """the sub-frames of a blur: [(t_k, q_k, frame_k)], frame_k = synth(t_k)'s frame, a / c at t_k <= 0 / >= 1"""
    plan = blur_plan(samples, gaussian, t0, t1)
    if plan is None:
        return None
    out = []
    for tk, qk in zip(*plan):
        if tk <= 0:
            f = a
        elif tk >= 1:
            f = c
        else:
            f, _ = synth(a, c, est, float(tk), settings, order)
        out.append((float(tk), qk, f))
    return out


def synth_blur(a, c, est, t0, t1, samples, gaussian, settings=None, order="rgba"):
    """recordSynthBlur's frame (None if refused): with blur off (N < 2) or t0 == t1 and t1 inside (0, 1), synth(t1);
    otherwise (sum q_k frame_k + 2^15) >> 16 per byte"""
    t0f, t1f = np.float32(t0), np.float32(t1)
    if not (t0f >= 0 and t1f <= 1 and t0f <= t1f):
        return None
    if not (samples >= 2 and t0f < t1f) and 0 < t1f < 1:
        return synth(a, c, est, float(t1f), settings, order)[0]
    acc = np.zeros(np.shape(a), np.int64)
    for _, qk, f in blur_subframes(a, c, est, t0, t1, samples, gaussian, settings, order):
        acc += qk * f.astype(np.int64)
    return ((acc + 32768) >> 16).astype(np.uint8)


def mean_f32(a):
    """numpy's float32 mean (pairwise) as restated in the oracle."""
    a = np.ascontiguousarray(a, np.float32).reshape(-1)
    return float(lib().fgo_mean_f32(_p(a), a.size))


# ---------------------------------------------------------------------------------------------- other frame formats
# Restated from the reference's shader math (fg_oracle_fmt.c): Rgb10, RgbaF16, Nv12, P010. Frames:
#   rgb10: uint32 (H, W) pixel words;  f16: float16 (H, W, 4);  nv12: (Y uint8 (H, W), CbCr uint8 (ch, cw, 2));
#   p010: (Y uint16 (H, W), CbCr uint16 (ch, cw, 2)), ch, cw = ceil(H / 2), ceil(W / 2).
FORMATS = {"rgb10": 1, "f16": 2, "nv12": 3, "p010": 4}
MATRICES = {"bt601": 0, "bt709": 1, "bt2020": 2}


@dataclass
class FormatSpec:
    """A frame format and what InitInfo says about it (gpu/framegen.h:411-441)."""
    format: str
    r_high: bool = False        # rgb10: A2R10G10B10 (R in bits 20..29) rather than A2B10G10R10
    linear: bool = False        # f16: Transfer::Linear (mismatch measured as PQ codes)
    white: float = 80.0         # f16 linear: nits of 1.0
    matrix: str = "bt709"       # yuv
    full_range: bool = False    # yuv


class _CFmt(ctypes.Structure):
    _fields_ = [("format", ctypes.c_int), ("rHigh", ctypes.c_int), ("linear", ctypes.c_int)] + \
               [(n, ctypes.c_float) for n in ("kWhite", "k10", "k10i", "black", "ys", "rcr", "bcb", "gcb", "gcr")]


class _CFrame(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("pitch", ctypes.c_long), ("c", ctypes.c_void_p), ("cpitch", ctypes.c_long)]


def _fmt_lib():
    L = lib()
    if not hasattr(L, "_fmt_ready"):
        P = ctypes.c_void_p
        L.fgo_fmt_init.argtypes = [ctypes.POINTER(_CFmt), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                   ctypes.c_int, ctypes.c_int]
        L.fgo_estimate_fmt.argtypes = [ctypes.POINTER(_CFrame), ctypes.POINTER(_CFrame), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_CFmt), ctypes.POINTER(_CSettings)] + [P] * 8 + [ctypes.c_int]
        L.fgo_estimate_fmt.restype = ctypes.c_int
        L.fgo_synth_fmt.argtypes = [ctypes.POINTER(_CFrame), ctypes.POINTER(_CFrame), ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(_CFmt), ctypes.POINTER(_CSettings), P, ctypes.c_int, ctypes.c_float,
                                    ctypes.POINTER(_CFrame), P, P, P, P, ctypes.c_int]
        L.fgo_synth_fmt.restype = ctypes.c_int
        L.fgo_estimate_fmt_ui.argtypes = L.fgo_estimate_fmt.argtypes + [ctypes.POINTER(_CUiMask), ctypes.POINTER(_CUiMask)]
        L.fgo_estimate_fmt_ui.restype = ctypes.c_int
        L.fgo_synth_fmt_ui.argtypes = L.fgo_synth_fmt.argtypes + [ctypes.POINTER(_CUiMask), ctypes.POINTER(_CUiMask)]
        L.fgo_synth_fmt_ui.restype = ctypes.c_int
        for n in ("fgo_log2", "fgo_exp2"):
            getattr(L, n).argtypes = [ctypes.c_float]
            getattr(L, n).restype = ctypes.c_float
        L.fgo_pq255.argtypes = [ctypes.c_float, ctypes.c_float]
        L.fgo_pq255.restype = ctypes.c_float
        L.fgo_f2h.argtypes = [ctypes.c_float]
        L.fgo_f2h.restype = ctypes.c_uint16
        L.fgo_h2f.argtypes = [ctypes.c_uint16]
        L.fgo_h2f.restype = ctypes.c_float
        L._fmt_ready = True
    return L


def fmt_struct(spec):
    f = _CFmt()
    _fmt_lib().fgo_fmt_init(ctypes.byref(f), FORMATS[spec.format], int(spec.r_high), int(spec.linear),
                            float(spec.white), MATRICES[spec.matrix], int(spec.full_range))
    return f


def frame_size(frame, spec):
    y = frame[0] if spec.format in ("nv12", "p010") else frame
    return y.shape[1], y.shape[0]


def _cframe(frame, spec):
    if spec.format in ("nv12", "p010"):
        y, uv = frame
        return _CFrame(y.ctypes.data, y.strides[0], uv.ctypes.data, uv.strides[0])
    return _CFrame(frame.ctypes.data, frame.strides[0], None, 0)


def empty_like_frame(frame, spec):
    if spec.format in ("nv12", "p010"):
        return (np.zeros_like(frame[0]), np.zeros_like(frame[1]))
    return np.zeros_like(frame)


def estimate_fmt(a, c, spec, settings=None, trace=True, threads=0, ui_fill=None):
    """estimate() for the other formats (same dict). ui_fill = (prev's mask, curr's mask), each (bytes, rect):
    CrosshairV2's estimate fill of both frames' level 0 (Rgb10 / RgbaF16)."""
    s = settings or Settings()
    W, H = frame_size(a, spec)
    L = layout(W, H, s.flowScale, s.pyramidMinSide)
    nl = sum(2 * w * h for w, h, _, _ in L.levels)
    nf = sum(4 * bw * bh for _, _, bw, bh in L.levels) + 4 * L.levels[0][2] * L.levels[0][3]
    ns = sum(2 * bw * bh for _, _, bw, bh in L.levels)
    luma = np.zeros(nl, np.float32) if trace else None
    fields = np.zeros(nf, np.float32) if trace else None
    seeds = np.zeros(ns, np.float32) if trace else None
    meds = np.zeros(2 * len(L.levels), np.float32) if trace else None
    nb0 = L.levels[0][2] * L.levels[0][3]
    sads = np.zeros(nb0, np.float32)
    pf = np.zeros((L.fh, L.fw, 2), np.float32)
    mean, cut = ctypes.c_float(), ctypes.c_int()
    fa, fc = _cframe(a, spec), _cframe(c, spec)
    (ma, ka), (mc, kc) = (_uimask(ui_fill[0]), _uimask(ui_fill[1])) if ui_fill else ((None, None), (None, None))
    n = _fmt_lib().fgo_estimate_fmt_ui(ctypes.byref(fa), ctypes.byref(fc), W, H, ctypes.byref(fmt_struct(spec)),
                                       ctypes.byref(_cs(s)), _p(luma), _p(fields), _p(seeds), _p(meds), _p(sads), _p(pf),
                                       ctypes.byref(mean), ctypes.byref(cut), threads,
                                       ctypes.byref(ma) if ma is not None else None,
                                       ctypes.byref(mc) if mc is not None else None)
    if n != len(L.levels):
        raise RuntimeError("fgo_estimate_fmt failed")
    est = {"sad": float(mean.value), "cut": bool(cut.value), "pf": pf, "layout": L,
           "sads": sads.reshape(L.levels[0][3], L.levels[0][2])}
    if trace:
        lum, fl = [], []
        o = of = 0
        for w, h, bw, bh in L.levels:
            lum.append((luma[o:o + w * h].reshape(h, w), luma[o + w * h:o + 2 * w * h].reshape(h, w)))
            o += 2 * w * h
            fl.append((fields[of:of + 2 * bw * bh].reshape(bh, bw, 2), fields[of + 2 * bw * bh:of + 4 * bw * bh].reshape(bh, bw, 2)))
            of += 4 * bw * bh
        bw0, bh0 = L.levels[0][2], L.levels[0][3]
        est["luma"] = lum
        est["fields"] = fl
        est["meds"] = meds.reshape(-1, 2)
        est["sub"] = [fields[of:of + 2 * bw0 * bh0].reshape(bh0, bw0, 2), fields[of + 2 * bw0 * bh0:].reshape(bh0, bw0, 2)]
    return est


def synth_fmt(a, c, est, t, spec, settings=None, trace=False, threads=0, ui=None):
    """synth() for the other formats: returns (frame, reason) or, with trace, a dict with out, reason, field_t, e,
    untrusted. The frame has the input's layout (a tuple of planes for YUV). ui = (prev's mask, curr's mask), each
    (bytes, rect) or None: CrosshairV2's warp-tap rejection (Rgb10 / RgbaF16; no paste-back here: ui_v2.patch_fmt)."""
    s = settings or Settings()
    W, H = frame_size(a, spec)
    out = empty_like_frame(a, spec)
    L = est["layout"]
    pf = np.ascontiguousarray(est["pf"], np.float32)
    ft = np.zeros((L.fh, L.fw, 2), np.float32) if trace else None
    e = np.zeros((H, W), np.uint8) if trace else None
    unt, reason = ctypes.c_longlong(), ctypes.c_int()
    fa, fc, fo = _cframe(a, spec), _cframe(c, spec), _cframe(out, spec)
    (ma, ka), (mc, kc) = (_uimask(ui[0]), _uimask(ui[1])) if ui else ((None, None), (None, None))
    r = _fmt_lib().fgo_synth_fmt_ui(ctypes.byref(fa), ctypes.byref(fc), W, H, ctypes.byref(fmt_struct(spec)),
                                    ctypes.byref(_cs(s)), _p(pf), int(est["cut"]), float(t), ctypes.byref(fo), _p(ft),
                                    _p(e), ctypes.byref(unt), ctypes.byref(reason), threads,
                                    ctypes.byref(ma) if ma is not None else None,
                                    ctypes.byref(mc) if mc is not None else None)
    if r != 0:
        raise ValueError("fgo_synth_fmt failed (t outside (0, 1)?)")
    if trace:
        return {"out": out, "reason": REASONS[reason.value], "field_t": ft, "e": e, "untrusted": int(unt.value)}
    return out, REASONS[reason.value]


def synth_blur_fmt(a, c, est, t0, t1, samples, gaussian, spec, settings=None, ui=None):
    """recordSynthBlur's frame in the other formats (None if refused), from synth_fmt's sub-frames: Rgb10 codes (by bit
    position, alpha's 2 bits included) and Nv12 / P010 luma and chroma codes averaged as (sum q_k v_k + 2^15) >> 16;
    RgbaF16 summed in sample order as float32 sums of fl32(q_k 2^-16 h_k) per channel (alpha included), then rounded
    to half. With blur off (N < 2) or t0 == t1 and t1 inside (0, 1): synth_fmt(t1). ui: as synth_fmt's, for every
    synthesized sub-frame."""
    t0f, t1f = np.float32(t0), np.float32(t1)
    if not (t0f >= 0 and t1f <= 1 and t0f <= t1f):
        return None
    if not (samples >= 2 and t0f < t1f) and 0 < t1f < 1:
        return synth_fmt(a, c, est, float(t1f), spec, settings, ui=ui)[0]
    times, q = blur_plan(samples, gaussian, t0, t1)
    subs = [a if tk <= 0 else c if tk >= 1 else synth_fmt(a, c, est, float(tk), spec, settings, ui=ui)[0]
            for tk in times.tolist()]

    def avg_codes(planes, shift):   # integer codes (after >> shift), then back
        acc = sum(qk * (f.astype(np.int64) >> shift) for qk, f in zip(q, planes))
        return ((acc + 32768) >> 16) << shift

    if spec.format == "rgb10":
        out = np.zeros_like(subs[0], dtype=np.uint32)
        for pos, mask in ((0, 1023), (10, 1023), (20, 1023), (30, 3)):
            acc = sum(qk * ((f.astype(np.int64) >> pos) & mask) for qk, f in zip(q, subs))
            out |= (((acc + 32768) >> 16) << pos).astype(np.uint32)
        return out
    if spec.format == "f16":
        acc = np.zeros(subs[0].shape, np.float32)
        for qk, f in zip(q, subs):
            acc = (acc + np.float32(qk / 65536.0) * f.astype(np.float32)).astype(np.float32)
        return acc.astype(np.float16)
    shift = 6 if spec.format == "p010" else 0
    dt = subs[0][0].dtype
    return (avg_codes([f[0] for f in subs], shift).astype(dt), avg_codes([f[1] for f in subs], shift).astype(dt))


def pq255(v, white=80.0):
    """the oracle's PQ level of a linear value (format.glsl fgPq * 255)"""
    L = _fmt_lib()
    return float(L.fgo_pq255(float(v), float(np.float32(white) / np.float32(10000.0))))


def f2h(v):
    return int(_fmt_lib().fgo_f2h(float(v)))


def h2f(h):
    return float(_fmt_lib().fgo_h2f(int(h)))


def log2(v):
    return float(_fmt_lib().fgo_log2(float(v)))


def exp2(v):
    return float(_fmt_lib().fgo_exp2(float(v)))
