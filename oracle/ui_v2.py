"""Test infrastructure (the oracle): a CPU restatement of frame-gen-ritz's static-UI protection in its CrosshairV2 mode
for 8-bit RGBA frames. Only the tests use it, as the checker of the library's kernels; the library never runs it.

The reference implements this mode only as Vulkan compute shaders (no CPU version exists), so this file restates the
shader math step by step; each function cites the shader it follows. Levels are the 8-bit values themselves (the
shaders' FG_STILL of an 8-bit UNORM texel, gpu/shaders/format.glsl:35).

  box_size / box_rect / work_rect    gpu/framegen.cpp:1041-1075 (Interpolator::boxSize, boxRect, boxMargin, workRect)
  State.update                       gpu/shaders/ui_v2_update.comp (observe and recordTrack: the per-pixel state machine)
  State.mask                         gpu/shaders/ui_v2_mask.comp (the mask bytes 255 / 64 / 0 with the 1 px grow)
  footprint / hit                    gpu/shaders/ui_reject.glsl:22-58 (which pixels a warp tap reads; is one of them UI)
  patch                              gpu/shaders/ui_patch.comp with binary = 1 (paste the real curr pixel where 255)
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

    def update(self, frame, order="rgba"):
        """one observed (or tracked) frame: gpu/shaders/ui_v2_update.comp"""
        s = self.s
        lv = _levels(frame, order)
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
                        contrasty = np.abs(now - _median7(lv, sy, sx)).max() >= cthr
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
