"""Test infrastructure (the oracle): a CPU restatement of frame-gen-ritz's static-UI protection in its CrosshairV2 mode
for 8-bit RGBA frames and the Rgb10 / RgbaF16 formats. Only the tests use it, as the checker of the library's kernels;
the library never runs it.

The reference implements this mode only as Vulkan compute shaders (no CPU version exists), so this file restates the
shader math step by step; each function cites the shader it follows. Levels are the shaders' 8-bit-equivalent FG_STILL
levels (gpu/shaders/format.glsl:35-53): the 8-bit values themselves, floor(code x 255 / 1023 + 0.5) for Rgb10,
clamp(floor(level + 0.5), 0, 255) for RgbaF16 (level: the PQ code x 255 of a linear value, value x 255 encoded).

  box_size / box_rect / work_rect    gpu/framegen.cpp:1041-1075 (Interpolator::boxSize, boxRect, boxMargin, workRect)
  State.update                       gpu/shaders/ui_v2_update.comp (observe and recordTrack: the per-pixel state machine)
  State.mask                         gpu/shaders/ui_v2_mask.comp (the mask bytes 255 / 64 / 0 with the 1 px grow)
  footprint / hit                    gpu/shaders/ui_reject.glsl:22-58 (which pixels a warp tap reads; is one of them UI)
  patch / patch_fmt                  gpu/shaders/ui_patch.comp with binary = 1 (paste the real curr pixel where 255)
  levels_fmt                         gpu/shaders/ui_v2_update.comp pixAt with format.glsl FG_STILL (Rgb10, RgbaF16)
The warp-tap rejection itself sits inside the oracle's synthesis (fg_oracle.c, fgo_synth_ui).
"""
import math

import numpy as np

SIDE_MIN = 8


def lround(v):
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))


def box_size(s, W, H):
    """(boxW, boxH): the explicit size, else the square of side round(H * uiBoxHeightFrac) (legacy: the area)"""
    if s.uiBoxHeightFrac > 0.0:
        side = min(max(lround(H * float(np.float32(s.uiBoxHeightFrac))), SIDE_MIN), min(W, H))
    else:
        side = min(max(lround(math.sqrt(float(np.float32(s.uiCrosshairArea)) * W * H)), 32), min(W, H))
    bw = min(max(int(s.uiBoxWidth), 4), W) if s.uiBoxWidth else side
    bh = min(max(int(s.uiBoxHeight), 4), H) if s.uiBoxHeight else side
    return bw, bh


def box_rect(s, W, H):
    bw, bh = box_size(s, W, H)
    x = min(max((W - bw) // 2 + int(s.uiBoxOffsetX), 0), W - bw)
    y = min(max((H - bh) // 2 + int(s.uiBoxOffsetY), 0), H - bh)
    return x, y, bw, bh


def work_rect(s, W, H, margin=1):
    x, y, w, h = box_rect(s, W, H)
    x0, y0 = max(x - margin, 0), max(y - margin, 0)
    x1, y1 = min(x + w + margin, W), min(y + h + margin, H)
    return x0, y0, x1 - x0, y1 - y0


def _levels(frame, order):
    """(H, W, 3) int32 levels in R, G, B order"""
    idx = [0, 1, 2] if order == "rgba" else [2, 1, 0]
    return frame[..., idx].astype(np.int32)


_PQ_TABLES = {}


def _pq_table(white):
    """the oracle's PQ level (x 255) of every half value, by its bits"""
    if white not in _PQ_TABLES:
        import oracle
        L = oracle._fmt_lib()
        kw = float(np.float32(white) / np.float32(10000.0))
        _PQ_TABLES[white] = np.array([L.fgo_pq255(L.fgo_h2f(i), kw) for i in range(65536)], np.float32)
    return _PQ_TABLES[white]


def levels_fmt(frame, spec):
    """(H, W, 3) int32 8-bit-equivalent levels in R, G, B order of an Rgb10 frame ((H, W) uint32 words) or an
    RgbaF16 frame ((H, W, 4) halves): FG_STILL of gpu/shaders/format.glsl, in float32 steps"""
    if spec.format == "rgb10":
        w = frame.view(np.uint32)
        shifts = (20, 10, 0) if spec.r_high else (0, 10, 20)
        codes = np.stack([(w >> sh) & 1023 for sh in shifts], axis=-1).astype(np.float32)
        k10 = np.float32(255.0 / 1023.0)
        return np.floor((codes * k10).astype(np.float32) + np.float32(0.5)).astype(np.int32)
    if spec.format == "f16":
        bits = frame.view(np.uint16)[..., :3]
        if spec.linear:
            lv = _pq_table(spec.white)[bits]
        else:
            lv = (bits.view(np.float16).astype(np.float32) * np.float32(255.0)).astype(np.float32)
        v = np.floor((lv + np.float32(0.5)).astype(np.float32))
        v = np.nan_to_num(v, nan=0.0, posinf=255.0, neginf=0.0)
        return np.clip(v, 0, 255).astype(np.int32)
    if spec.format in ("nv12", "p010"):   # fgStillYuv: (Y, Cb, Cr) levels of the pixel and its chroma texel
        y, uv = frame
        yc = y.view(np.uint16 if spec.format == "p010" else np.uint8).astype(np.float32)
        cc = uv.view(np.uint16 if spec.format == "p010" else np.uint8).astype(np.float32)
        if spec.format == "p010":
            yc, cc = yc * np.float32(2 ** -8), cc * np.float32(2 ** -8)
        H, W = yc.shape
        c = cc[np.arange(H)[:, None] // 2, np.arange(W)[None, :] // 2]   # (H, W, 2)
        lv = np.concatenate([yc[..., None], c], axis=-1).astype(np.float32)
        return np.clip(np.floor((lv + np.float32(0.5)).astype(np.float32)), 0, 255).astype(np.int32)
    raise ValueError("CrosshairV2 levels: not this format")


def yuv_diff_max(d, spec):
    """format.glsl fgYuvDiff + max |.|: the R'G'B' difference a (Y, Cb, Cr) level difference stands for, in the
    library's float32 order (y = ys dY; r = y + rcr dCr; g = (y + gcb dCb) + gcr dCr; b = y + bcb dCb)"""
    import oracle
    f = oracle.fmt_struct(spec)
    f32 = np.float32
    dy, db, dr = (f32(v) for v in d)
    y = f32(f32(f.ys) * dy)
    r = f32(y + f32(f32(f.rcr) * dr))
    g = f32(f32(y + f32(f32(f.gcb) * db)) + f32(f32(f.gcr) * dr))
    b = f32(y + f32(f32(f.bcb) * db))
    return max(abs(r), abs(g), abs(b))


def _median7(lv, y, x):
    """per channel, the median of the 7x7 window around (y, x), taps clamped to the frame (the 25th of 49 values)"""
    H, W = lv.shape[:2]
    ys = np.clip(np.arange(y - 3, y + 4), 0, H - 1)
    xs = np.clip(np.arange(x - 3, x + 4), 0, W - 1)
    win = lv[ys][:, xs].reshape(49, 3)
    return np.sort(win, axis=0)[24]


class State:
    """The state of the work rectangle's pixels, unpacked: prev (3) the previous original, cnt the still-and-contrasty
    count, stored (3) the last confirmed colour, flags (bit 0 in the mask, bit 1 has a stored colour, bit 2 still in
    this pair), leave, match."""

    def __init__(self, s, W, H):
        self.s, self.W, self.H = s, W, H
        self.box = box_rect(s, W, H)
        self.work = work_rect(s, W, H)
        wx, wy, ww, wh = self.work
        self.prev = np.zeros((wh, ww, 3), np.int32)
        self.cnt = np.zeros((wh, ww), np.int32)
        self.stored = np.zeros((wh, ww, 3), np.int32)
        self.flags = np.zeros((wh, ww), np.int32)
        self.leave = np.zeros((wh, ww), np.int32)
        self.match = np.zeros((wh, ww), np.int32)
        self.reset = True

    def update(self, frame, order="rgba", spec=None):
        """one observed (or tracked) frame: gpu/shaders/ui_v2_update.comp; spec: the frame's format (oracle.FormatSpec)
        when it is not 8-bit RGBA / BGRA"""
        s = self.s
        lv = _levels(frame, order) if spec is None else levels_fmt(frame, spec)
        yuv = spec is not None and spec.format in ("nv12", "p010")
        wx, wy, ww, wh = self.work
        bx, by, bw, bh = self.box
        thr = float(np.float32(s.uiStillThreshold))
        cthr = float(np.float32(s.uiContrastThreshold))
        reset = self.reset
        for y in range(wh):
            for x in range(ww):
                sy, sx = wy + y, wx + x
                now = lv[sy, sx]
                if not (bx <= sx < bx + bw and by <= sy < by + bh):   # the margin ring: the pair gate only
                    still = (not reset) and np.abs(now - self.prev[y, x]).max() <= thr
                    self.prev[y, x] = now
                    self.cnt[y, x] = 0
                    self.stored[y, x] = 0
                    self.flags[y, x] = 4 if still else 0
                    self.leave[y, x] = self.match[y, x] = 0
                    continue
                cnt = flags = leave = match = 0
                stored = np.zeros(3, np.int32)
                if not reset:
                    flags, stored = int(self.flags[y, x]), self.stored[y, x].copy()
                    leave, match = int(self.leave[y, x]), int(self.match[y, x])
                    still = np.abs(now - self.prev[y, x]).max() <= thr
                    in_mask, has_stored = bool(flags & 1), bool(flags & 2)
                    match_s = (not in_mask) and has_stored and s.uiReentryFrames > 0 and np.abs(now - stored).max() <= thr
                    contrasty = cthr <= 0.0
                    if not in_mask and not contrasty and (still or match_s):
                        d = now - _median7(lv, sy, sx)
                        contrasty = (yuv_diff_max(d, spec) if yuv else np.abs(d).max()) >= cthr
                    if in_mask:
                        leave = 0 if still else min(leave + 1, 255)
                        if still:
                            stored = now.copy()
                        if leave >= s.uiLeaveFrames:
                            in_mask, leave, match = False, 0, 0
                        cnt = 0
                    else:
                        cnt = min(int(self.cnt[y, x]) + 1, 255) if (still and contrasty) else 0
                        match = min(match + 1, 255) if (match_s and contrasty) else 0
                        if cnt >= s.uiStillFrames or (s.uiReentryFrames > 0 and has_stored and match >= s.uiReentryFrames):
                            in_mask, has_stored, stored, leave, match = True, True, now.copy(), 0, 0
                    flags = (1 if in_mask else 0) | (2 if has_stored else 0) | (4 if still else 0)
                self.prev[y, x] = now
                self.cnt[y, x] = cnt
                self.stored[y, x] = stored
                self.flags[y, x] = flags
                self.leave[y, x] = leave
                self.match[y, x] = match
        self.reset = False

    def mask(self):
        """(wh, ww) uint8: 255 in the mask or its 1 px grow and still in this pair, 64 in it but changed, else 0
        (gpu/shaders/ui_v2_mask.comp)"""
        inm = (self.flags & 1) != 0
        wh, ww = inm.shape
        pad = np.pad(inm, 1)
        near = np.zeros_like(inm)
        for dy in range(3):
            for dx in range(3):
                near |= pad[dy:dy + wh, dx:dx + ww]
        return np.where(near, np.where((self.flags & 4) != 0, 255, 64), 0).astype(np.uint8)


def footprint(px, py):
    """the pixels a bilinear tap at (px, py) (pixel-centre coordinates, float32) reads with a non-zero weight: X =
    roundEven(32 p), lo = X >> 5, hi = lo + (X & 31 != 0), per axis (gpu/shaders/ui_reject.glsl:44-57)"""
    X = int(np.rint(np.float32(px) * np.float32(32.0)))
    Y = int(np.rint(np.float32(py) * np.float32(32.0)))
    lo = (X >> 5, Y >> 5)
    return lo, (lo[0] + (X & 31 != 0), lo[1] + (Y & 31 != 0))


def hit(mask, rect, lo, hi):
    """is any pixel of lo..hi (frame coordinates, inclusive) non-zero in the mask over rect?"""
    if mask is None:
        return False
    ox, oy, w, h = rect
    x0, y0 = max(lo[0] - ox, 0), max(lo[1] - oy, 0)
    x1, y1 = min(hi[0] - ox, w - 1), min(hi[1] - oy, h - 1)
    if x0 > x1 or y0 > y1:
        return False
    return bool((mask[y0:y1 + 1, x0:x1 + 1] != 0).any())


def patch(out, curr, mask, rect):
    """out = the real curr pixel (its colour channels; alpha kept) where the mask byte is 255
    (gpu/shaders/ui_patch.comp, binary)"""
    ox, oy, w, h = rect
    sel = mask == 255
    reg = out[oy:oy + h, ox:ox + w]
    src = curr[oy:oy + h, ox:ox + w]
    for c in range(3):
        reg[..., c][sel] = src[..., c][sel]
    return out


def patch_fmt(out, curr, mask, rect, spec):
    """patch() for Rgb10 (the colour codes from curr, the 2 alpha bits kept), RgbaF16 (R, G, B halves from curr,
    alpha kept) and YUV (the luma plane where 255; a chroma texel takes the strongest mask byte of its 2x2 pixels
    inside the rectangle and is copied where that is 255: gpu/shaders/ui_patch_chroma.comp, binary)"""
    ox, oy, w, h = rect
    sel = mask == 255
    if spec.format in ("nv12", "p010"):
        oy_, ouv = out
        cy_, cuv = curr
        oy_[oy:oy + h, ox:ox + w][sel] = cy_[oy:oy + h, ox:ox + w][sel]
        for ty in range(oy >> 1, ((oy + h - 1) >> 1) + 1):
            for tx in range(ox >> 1, ((ox + w - 1) >> 1) + 1):
                a = 0
                for j in range(2):
                    for i in range(2):
                        ry, rx = 2 * ty + j - oy, 2 * tx + i - ox
                        if 0 <= ry < h and 0 <= rx < w:
                            a = max(a, int(mask[ry, rx]))
                if a == 255:
                    ouv[ty, tx] = cuv[ty, tx]
        return out
    if spec.format == "rgb10":
        reg = out.view(np.uint32)[oy:oy + h, ox:ox + w]
        src = curr.view(np.uint32)[oy:oy + h, ox:ox + w]
        reg[sel] = (src[sel] & np.uint32(0x3FFFFFFF)) | (reg[sel] & np.uint32(0xC0000000))
        return out
    reg = out.view(np.uint16)[oy:oy + h, ox:ox + w]
    src = curr.view(np.uint16)[oy:oy + h, ox:ox + w]
    for c in range(3):
        reg[..., c][sel] = src[..., c][sel]
    return out
