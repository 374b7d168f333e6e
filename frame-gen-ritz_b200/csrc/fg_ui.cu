// Static-UI protection, CrosshairV2 mode, for 8-bit RGBA / BGRA, Rgb10 and RgbaF16 frames: the passes of recordObserve
// / recordTrack and the paste-back after a synthesis. Pixels enter the state machine as the shaders' 8-bit-equivalent
// levels (format.glsl FG_STILL): the bytes of 8-bit RGBA, floor(code x fl32(255 / 1023) + 0.5) for Rgb10,
// clamp(floor(level + 0.5), 0, 255) for RgbaF16 (level: the PQ code x 255 of a linear value, the value x 255 encoded). The warp-tap rejection between them lives in the synthesis kernels (uiHitMask in
// fg_device.h). Restates the reference's Vulkan shaders gpu/shaders/ui_v2_update.comp, ui_v2_mask.comp and
// ui_patch.comp (binary paste); layouts in fg_params.h (UiV2Params).
//
//   k_ui_v2_update  one thread per pixel of the work rectangle: the per-pixel state machine (still / contrasty / in the
//                   mask / leave and re-entry counters). The local contrast, max channel |I - median7x7(I)|, is found
//                   only where it can matter (out of the mask and still or matching its stored colour): per channel a
//                   binary search on the value for the smallest m with at least 25 of the 49 levels <= m, the window's
//                   49 pixels packed one word each in registers.
//   k_ui_v2_mask    one thread per mask word (4 pixels): in the mask or within 1 px of it -> 255 if still in this pair,
//                   else 64; writes the rectangle into the header.
//   k_ui_patch      one thread per work-rectangle pixel: out = the real curr pixel (colour channels) where the byte is
//                   255.
// The work rectangle of a 4K frame's default box is 56 x 56 pixels: these passes are latency-sized, not bandwidth-sized.
#include <cstdint>

#include <cuda_fp16.h>

#include "fg_device.h"
#include "fg_params.h"

namespace fgk {
namespace {

constexpr int kUiTX = 16, kUiTY = 8;   // threads per CTA of the update and patch passes

// an RgbaF16 half's 8-bit-equivalent level
__device__ __forceinline__ uint32_t uiLevelF16(const UiV2Params& p, uint32_t bits) {
    const float lv = p.f.linear ? __ldg(p.pq + bits)
                                : __fmul_rn(__half2float(__ushort_as_half((unsigned short)bits)), 255.0f);
    return (uint32_t)fminf(fmaxf(floorf(__fadd_rn(lv, 0.5f)), 0.0f), 255.0f);   // NaN -> 0
}

__device__ __forceinline__ uint32_t uiPixel(const UiV2Params& p, int x, int y) {   // r | g << 8 | b << 16, clamped
    x = min(max(x, 0), p.W - 1);
    y = min(max(y, 0), p.H - 1);
    const uint8_t* row = p.frame + (size_t)y * p.pitch;
    if (p.f.format == kFmtRgb10) {
        const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(row) + x);
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t code = (w >> (p.f.rHigh ? 20 - 10 * k : 10 * k)) & 1023u;
            o |= (uint32_t)floorf(__fadd_rn(__fmul_rn((float)code, p.f.k10), 0.5f)) << (8 * k);
        }
        return o;
    }
    if (p.f.format == kFmtF16) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(row) + x);
        return uiLevelF16(p, q.x & 0xFFFFu) | (uiLevelF16(p, q.x >> 16) << 8) | (uiLevelF16(p, q.y & 0xFFFFu) << 16);
    }
    const uint8_t* crow = p.frameC + (size_t)(y >> 1) * p.cpitch;
    if (p.f.format == kFmtNv12)   // (Y, Cb, Cr): the bytes themselves
        return (uint32_t)__ldg(row + x) | ((uint32_t)__ldg(reinterpret_cast<const unsigned short*>(crow) + (x >> 1)) << 8);
    if (p.f.format == kFmtP010) {   // floor(s 2^-8 + 0.5) of each 16-bit sample, at most 255
        auto lv = [](uint32_t s16) { return min((s16 + 128u) >> 8, 255u); };
        const uint32_t c = __ldg(reinterpret_cast<const uint32_t*>(crow) + (x >> 1));
        return lv(__ldg(reinterpret_cast<const unsigned short*>(row) + x)) | (lv(c & 0xFFFFu) << 8) | (lv(c >> 16) << 16);
    }
    const uint32_t v = __ldg(reinterpret_cast<const uint32_t*>(row) + x);
    return ((v >> (8 * p.ri)) & 255u) | (((v >> (8 * p.gi)) & 255u) << 8) | (((v >> (8 * p.bi)) & 255u) << 16);
}

__device__ __forceinline__ int maxAbsDiff(uint32_t a, uint32_t b) {
    int m = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) m = max(m, abs((int)((a >> (8 * c)) & 255u) - (int)((b >> (8 * c)) & 255u)));
    return m;
}

// max channel |v - median7x7| at (x, y); YUV: of the R'G'B' difference the (Y, Cb, Cr) difference stands for
// (format.glsl fgYuvDiff, in the order of the synthesis' mismatch)
__device__ float contrastAt(const UiV2Params& p, int x, int y, uint32_t v) {
    uint32_t w[49];
#pragma unroll
    for (int j = 0; j < 7; j++)
#pragma unroll
        for (int i = 0; i < 7; i++) w[j * 7 + i] = uiPixel(p, x + i - 3, y + j - 3);
    int d = 0, dc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        int lo = 0, hi = 255;
        for (int it = 0; it < 8; it++) {
            const int mid = (lo + hi) >> 1;
            int cnt = 0;
#pragma unroll
            for (int j = 0; j < 49; j++) cnt += (int)((w[j] >> (8 * c)) & 255u) <= mid;
            if (cnt >= 25) hi = mid;
            else lo = mid + 1;
        }
        dc[c] = (int)((v >> (8 * c)) & 255u) - lo;
        d = max(d, abs(dc[c]));
    }
    if (p.f.format == kFmtNv12 || p.f.format == kFmtP010) {
        const float dy = (float)dc[0], db = (float)dc[1], dr = (float)dc[2];
        const float yv = __fmul_rn(p.f.ys, dy);
        const float r = __fadd_rn(yv, __fmul_rn(p.f.rcr, dr));
        const float g = __fadd_rn(__fadd_rn(yv, __fmul_rn(p.f.gcb, db)), __fmul_rn(p.f.gcr, dr));
        const float b = __fadd_rn(yv, __fmul_rn(p.f.bcb, db));
        return fmaxf(fabsf(r), fmaxf(fabsf(g), fabsf(b)));
    }
    return (float)d;
}

__global__ void __launch_bounds__(kUiTX * kUiTY) k_ui_v2_update(const UiV2Params p) {
    pdlEnter();
    const int x = blockIdx.x * kUiTX + threadIdx.x, y = blockIdx.y * kUiTY + threadIdx.y;
    if (x >= p.ww || y >= p.wh) return;
    const int sx = p.wx + x, sy = p.wy + y;
    const uint32_t now = uiPixel(p, sx, sy);
    uint32_t* s = p.st + ((size_t)y * p.ww + x) * 4;
    const int ix = sx - p.bx, iy = sy - p.by;
    if (ix < 0 || iy < 0 || ix >= p.bw || iy >= p.bh) {   // the margin ring: only the pair gate
        uint32_t ring = 0;
        if (!p.reset && (float)maxAbsDiff(now, s[0] & 0xFFFFFFu) <= p.thr) ring = 4u;
        s[0] = now;
        s[1] = ring << 24;
        s[2] = 0u;
        return;
    }
    uint32_t cnt = 0, flags = 0, leave = 0, match = 0, stored = 0;
    if (!p.reset) {
        const uint32_t w0 = s[0], w1 = s[1], w2 = s[2];
        flags = w1 >> 24;
        stored = w1 & 0xFFFFFFu;
        leave = w2 & 255u;
        match = (w2 >> 8) & 255u;
        const bool still = (float)maxAbsDiff(now, w0 & 0xFFFFFFu) <= p.thr;
        bool inMask = (flags & 1u) != 0u, hasStored = (flags & 2u) != 0u;
        const bool matchS = !inMask && hasStored && p.reentry > 0 && (float)maxAbsDiff(now, stored) <= p.thr;
        bool contrasty = p.cthr <= 0.0f;
        if (!inMask && !contrasty && (still || matchS)) contrasty = contrastAt(p, sx, sy, now) >= p.cthr;
        if (inMask) {
            leave = still ? 0u : min(leave + 1u, 255u);
            if (still) stored = now;
            if ((int)leave >= p.leave) {
                inMask = false;
                leave = 0u;
                match = 0u;
            }
            cnt = 0u;
        } else {
            cnt = (still && contrasty) ? min((w0 >> 24) + 1u, 255u) : 0u;
            match = (matchS && contrasty) ? min(match + 1u, 255u) : 0u;
            if ((int)cnt >= p.still || (p.reentry > 0 && hasStored && (int)match >= p.reentry)) {
                inMask = true;
                hasStored = true;
                stored = now;
                leave = 0u;
                match = 0u;
            }
        }
        flags = (inMask ? 1u : 0u) | (hasStored ? 2u : 0u) | (still ? 4u : 0u);
    }
    s[0] = now | (cnt << 24);
    s[1] = stored | (flags << 24);
    s[2] = leave | (match << 8);
}

__device__ __forceinline__ uint32_t uiFlagsAt(const UiV2Params& p, int x, int y) {
    if (x < 0 || y < 0 || x >= p.ww || y >= p.wh) return 0u;
    return p.st[((size_t)y * p.ww + x) * 4 + 1] >> 24;
}

__global__ void __launch_bounds__(128) k_ui_v2_mask(const UiV2Params p) {
    pdlEnter();
    const int g = blockIdx.x * 128 + threadIdx.x;
    if (g >= p.maskStride * p.wh) return;
    const int gx = g % p.maskStride, gy = g / p.maskStride;
    uint32_t word = 0;
    for (int k = 0; k < 4; k++) {
        const int x = gx * 4 + k;
        if (x >= p.ww) break;
        bool near = false;
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) near = near || (uiFlagsAt(p, x + dx, gy + dy) & 1u) != 0u;
        uint32_t a = 0;
        if (near) a = (uiFlagsAt(p, x, gy) & 4u) != 0u ? 255u : 64u;
        word |= a << (8 * k);
    }
    p.mask[kUiMaskHeader + g] = word;
    if (g == 0) {
        p.mask[0] = 0u;
        p.mask[1] = (uint32_t)p.wx | ((uint32_t)p.wy << 16);
        p.mask[2] = (uint32_t)p.ww | ((uint32_t)p.wh << 16);
        p.mask[3] = (uint32_t)p.maskStride;
    }
}

__global__ void __launch_bounds__(kUiTX * kUiTY) k_ui_patch(const UiPatchParams p, int wx, int wy, int ww, int wh) {
    pdlEnter();
    const int x = blockIdx.x * kUiTX + threadIdx.x, y = blockIdx.y * kUiTY + threadIdx.y;
    if (x >= ww || y >= wh) return;
    const int stride = (int)p.mask[3];
    const uint32_t a = (p.mask[kUiMaskHeader + y * stride + (x >> 2)] >> (8 * (x & 3))) & 255u;
    if (a != 255u) return;
    if (p.format == kFmtNv12 || p.format == kFmtP010) {   // the luma sample (the chroma: k_ui_patch_chroma)
        const size_t o = (size_t)(wy + y), i = (size_t)(wx + x);
        if (p.format == kFmtNv12) p.out[o * p.outPitch + i] = __ldg(p.curr + o * p.pitch + i);
        else reinterpret_cast<unsigned short*>(p.out + o * p.outPitch)[i] =
                 __ldg(reinterpret_cast<const unsigned short*>(p.curr + o * p.pitch) + i);
        return;
    }
    if (p.format == kFmtF16) {   // R, G, B halves from the real frame, alpha kept
        uint2* o = reinterpret_cast<uint2*>(p.out + (size_t)(wy + y) * p.outPitch) + wx + x;
        const uint2 real = __ldg(reinterpret_cast<const uint2*>(p.curr + (size_t)(wy + y) * p.pitch) + wx + x);
        *o = make_uint2(real.x, (real.y & 0xFFFFu) | (o->y & 0xFFFF0000u));
        return;
    }
    // colour channels from the real frame, alpha kept (8-bit RGBA: byte 3; Rgb10: the top 2 bits)
    const uint32_t keep = p.format == kFmtRgb10 ? 0xC0000000u : 0xFF000000u;
    uint32_t* o = reinterpret_cast<uint32_t*>(p.out + (size_t)(wy + y) * p.outPitch) + wx + x;
    const uint32_t real = __ldg(reinterpret_cast<const uint32_t*>(p.curr + (size_t)(wy + y) * p.pitch) + wx + x);
    *o = (real & ~keep) | (*o & keep);
}

// YUV: gpu/shaders/ui_patch_chroma.comp (binary): one thread per CbCr texel of the work rectangle; a texel takes the
// strongest mask byte of its 2x2 pixels inside the rectangle and is copied from the real frame where that is 255
__global__ void __launch_bounds__(kUiTX * kUiTY) k_ui_patch_chroma(const UiPatchParams p, int wx, int wy, int ww, int wh) {
    pdlEnter();
    const int tx = (wx >> 1) + (int)(blockIdx.x * kUiTX + threadIdx.x), ty = (wy >> 1) + (int)(blockIdx.y * kUiTY + threadIdx.y);
    if (tx > (wx + ww - 1) >> 1 || ty > (wy + wh - 1) >> 1) return;
    const int stride = (int)p.mask[3];
    uint32_t a = 0;
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) {
            const int rx = 2 * tx + i - wx, ry = 2 * ty + j - wy;
            if (rx < 0 || ry < 0 || rx >= ww || ry >= wh) continue;
            a = max(a, (p.mask[kUiMaskHeader + ry * stride + (rx >> 2)] >> (8 * (rx & 3))) & 255u);
        }
    if (a != 255u) return;
    if (p.format == kFmtNv12)
        reinterpret_cast<unsigned short*>(p.outC + (size_t)ty * p.outCPitch)[tx] =
            __ldg(reinterpret_cast<const unsigned short*>(p.currC + (size_t)ty * p.cpitch) + tx);
    else
        reinterpret_cast<uint32_t*>(p.outC + (size_t)ty * p.outCPitch)[tx] =
            __ldg(reinterpret_cast<const uint32_t*>(p.currC + (size_t)ty * p.cpitch) + tx);
}

// The estimate fill (gpu/shaders/ui_v2_lumafill.comp), one thread per level-0 cell of the mask rectangle, z = 0 prev,
// 1 curr: a cell holding a UI pixel takes the mean gray level (cv2's weights, the library's level-0 source) of its
// not-UI pixels, the window widened by fs px per side per step up to 8 px while there are none, rounded half up to the
// level-0 grid (multiples of 1 / fs^2) so the estimate's sums stay exact.
__global__ void __launch_bounds__(64) k_ui_v2_fill(const UiFillParams p) {
    pdlEnter();
    const int cx = p.cx0 + (int)(blockIdx.x * 8 + (threadIdx.x & 7)), cy = p.cy0 + (int)(blockIdx.y * 8 + (threadIdx.x >> 3));
    if (cx >= p.cx0 + p.ncx || cy >= p.cy0 + p.ncy || cx >= p.fw || cy >= p.fh) return;
    const bool isC = blockIdx.z != 0;
    const uint32_t* __restrict__ m = isC ? p.mc : p.ma;
    const uint8_t* f = isC ? p.c : p.a;
    const int fs = p.fs, px = cx * fs, py = cy * fs;
    bool has = false;
    for (int j = 0; j < fs && !has; j++)
        for (int i = 0; i < fs; i++)
            if (px + i < p.W && py + j < p.H && uiPx(m, px + i, py + j)) {
                has = true;
                break;
            }
    if (!has) return;
    for (int k = 0; k <= 8; k += fs) {
        int sum = 0, n = 0;
        for (int y = py - k; y < py + fs + k; y++)
            for (int x = px - k; x < px + fs + k; x++) {
                if (x < 0 || y < 0 || x >= p.W || y >= p.H || uiPx(m, x, y)) continue;
                sum += gray8(__ldg(reinterpret_cast<const uint32_t*>(f + (size_t)y * p.pitch) + x), p.ri, p.gi, p.bi);
                n++;
            }
        if (n > 0) {
            const int s2 = fs * fs;
            (isC ? p.lc : p.la)[(size_t)cy * p.fw + cx] = (float)((2 * sum * s2 + n) / (2 * n)) / (float)s2;
            return;
        }
    }
}

}  // namespace

cudaError_t launchUiFill(const UiFillParams& p, cudaStream_t s) {
    return launchPdl(k_ui_v2_fill, dim3(divUp(p.ncx, 8), divUp(p.ncy, 8), 2), dim3(64), 0, s, p);
}

cudaError_t launchUiV2Update(const UiV2Params& p, cudaStream_t s) {
    return launchPdl(k_ui_v2_update, dim3(divUp(p.ww, kUiTX), divUp(p.wh, kUiTY)), dim3(kUiTX, kUiTY), 0, s, p);
}
cudaError_t launchUiV2Mask(const UiV2Params& p, cudaStream_t s) {
    return launchPdl(k_ui_v2_mask, dim3(divUp(p.maskStride * p.wh, 128)), dim3(128), 0, s, p);
}
cudaError_t launchUiPatch(const UiPatchParams& p, int wx, int wy, int ww, int wh, cudaStream_t s) {
    cudaError_t e = launchPdl(k_ui_patch, dim3(divUp(ww, kUiTX), divUp(wh, kUiTY)), dim3(kUiTX, kUiTY), 0, s, p, wx, wy, ww, wh);
    if (e == cudaSuccess && (p.format == kFmtNv12 || p.format == kFmtP010)) {
        const int tw = ((wx + ww - 1) >> 1) - (wx >> 1) + 1, th = ((wy + wh - 1) >> 1) - (wy >> 1) + 1;
        e = launchPdl(k_ui_patch_chroma, dim3(divUp(tw, kUiTX), divUp(th, kUiTY)), dim3(kUiTX, kUiTY), 0, s, p, wx, wy,
                      ww, wh);
    }
    return e;
}

}  // namespace fgk
