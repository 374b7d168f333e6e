// CUDA kernels of the V1 path for the frame formats other than 8-bit RGBA: Rgb10 (A2B10G10R10 / A2R10G10B10),
// RgbaF16 (display-encoded, or linear light measured as PQ codes), Nv12 and P010 (two planes, 4:2:0).
//
// The reference defines these formats in its shaders (gpu/shaders/format.glsl:29-106, luma.comp:9-27,
// motion_v1.glsl:86-144, resolve.comp:48-83, the constants of gpu/framegen.cpp:1508-1539); proto/interp.py has no
// counterpart. The kernels compute exactly this arithmetic:
//   - motion-estimate luma in quarter levels (the 10-bit code grid): Q = rint(4 clamp(y, 0, 255)) of the format's
//     luma y; level 0 = rint(4 sum(Q) / n) / 16 over each flowScale cell; pyramid levels rounded to a multiple of
//     2^-10. Every SAD, tap and box sum of the estimate is then exact in float32 whatever the order, so the search,
//     median, sub-pixel and pixel-field kernels are the 8-bit RGBA path's own;
//   - warp taps at the sample point rounded to 1/32 px (chroma: the same normalised point, 1/64 chroma texel), the
//     bilinear tap ((p00 w00 + p01 w01) + p10 w10) + p11 w11 in float, clamped to the edge; the mismatch, blend and
//     stores of format.glsl / resolve.comp with a fixed operation order (round-to-nearest intrinsics, no fusion);
//   - PQ (SMPTE ST 2084) via the log2 / exp2 series below, built from IEEE float operations only.
// Synthesis tiles are the 8-bit path's (kSyE x kSyEH mismatch region, 3-pixel halo); the warps of the output
// pixels are taken again after the 7x7 box instead of being held in registers (up to 3 floats per channel).
#include <cuda_fp16.h>

#include "fg_device.h"

namespace fgk {

// ============================================================================================== float helpers
// log2 of a positive normal float: x = 2^e m, m in [sqrt(1/2), sqrt(2)); log2 m = 2/ln2 atanh(s),
// s = (m - 1) / (m + 1), by its odd series to s^9
__device__ __forceinline__ float fmtLog2(float x) {
    const uint32_t b = __float_as_uint(x);
    int e = (int)((b >> 23) & 255u) - 127;
    float m = __uint_as_float((b & 0x7FFFFFu) | 0x3F800000u);
    if (m > 0x1.6a09e6p+0f) { m = __fmul_rn(m, 0.5f); e += 1; }
    const float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float z = __fmul_rn(s, s);
    float p = 0x1.484b14p-2f;
    p = __fadd_rn(__fmul_rn(p, z), 0x1.a61762p-2f);
    p = __fadd_rn(__fmul_rn(p, z), 0x1.2776c6p-1f);
    p = __fadd_rn(__fmul_rn(p, z), 0x1.ec709ep-1f);
    p = __fadd_rn(__fmul_rn(p, z), 0x1.715476p+1f);
    return __fadd_rn((float)e, __fmul_rn(s, p));
}

// 2^x for -126 <= x < 128 (0 below): x = n + g + 1/2, n = floor(x); 2^(g + 1/2) = sqrt2 e^(g ln2), series to g^7
__device__ __forceinline__ float fmtExp2(float x) {
    if (!(x >= -126.0f)) return 0.0f;
    const float n = floorf(x);
    const float g = __fsub_rn(__fsub_rn(x, n), 0.5f);
    float p = 0x1.ffcbfcp-17f;
    p = __fadd_rn(__fmul_rn(p, g), 0x1.430912p-13f);
    p = __fadd_rn(__fmul_rn(p, g), 0x1.5d87fep-10f);
    p = __fadd_rn(__fmul_rn(p, g), 0x1.3b2ab6p-7f);
    p = __fadd_rn(__fmul_rn(p, g), 0x1.c6b08ep-5f);
    p = __fadd_rn(__fmul_rn(p, g), 0x1.ebfbe0p-3f);
    p = __fadd_rn(__fmul_rn(p, g), 0x1.62e430p-1f);
    p = __fadd_rn(__fmul_rn(p, g), 1.0f);
    p = __fmul_rn(p, 0x1.6a09e6p+0f);
    return __fmul_rn(p, __uint_as_float((uint32_t)((int)n + 127) << 23));
}

__device__ __forceinline__ float clampF(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// format.glsl fgPq * 255: the level of a linear-light value as an 8-bit PQ code
__device__ __noinline__ float fmtPq255(float v, float kWhite) {
    const float y = clampF(__fmul_rn(v, kWhite), 0.0f, 1.0f);
    float p = 0.0f;
    if (y >= 0x1p-126f) p = fmtExp2(__fmul_rn(0.1593017578125f, fmtLog2(y)));
    const float num = __fadd_rn(0.8359375f, __fmul_rn(18.8515625f, p));
    const float den = __fadd_rn(1.0f, __fmul_rn(18.6875f, p));
    const float r = __fdiv_rn(num, den);
    return __fmul_rn(fmtExp2(__fmul_rn(78.84375f, fmtLog2(r))), 255.0f);
}

__device__ __forceinline__ float h2f(uint32_t h16) { return __half2float(__ushort_as_half((unsigned short)h16)); }

// ============================================================================================== pixel access
__device__ __forceinline__ uint32_t ldw(const uint8_t* base, size_t pitch, int x, int y) {
    return __ldg(reinterpret_cast<const uint32_t*>(base + (size_t)y * pitch) + x);
}
__device__ __forceinline__ uint32_t ldh(const uint8_t* base, size_t pitch, int x, int y) {   // a 16-bit sample
    return __ldg(reinterpret_cast<const unsigned short*>(base + (size_t)y * pitch) + x);
}

// a raw channel of an Rgb10 word (k: 0 R, 1 G, 2 B)
__device__ __forceinline__ int rgb10(const FmtConst& f, uint32_t w, int k) {
    return (int)((w >> (f.rHigh ? 20 - 10 * k : 10 * k)) & 1023u);
}

// the three raw channels of texel (x, y): Rgb10 codes, F16 values; YUV: the Y level only (r[0])
template <int F>
__device__ __forceinline__ void texel(const FmtConst& f, const uint8_t* base, size_t pitch, int x, int y, float r[3]) {
    if (F == kFmtRgb10) {
        const uint32_t w = ldw(base, pitch, x, y);
#pragma unroll
        for (int k = 0; k < 3; k++) r[k] = i2f(rgb10(f, w, k));
    } else if (F == kFmtF16) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(base + (size_t)y * pitch) + x);
        r[0] = h2f(q.x & 0xFFFFu);
        r[1] = h2f(q.x >> 16);
        r[2] = h2f(q.y & 0xFFFFu);
    } else if (F == kFmtNv12) {
        r[0] = i2f(__ldg(base + (size_t)y * pitch + x));
    } else {
        r[0] = __fmul_rn(i2f((int)ldh(base, pitch, x, y)), 0x1p-8f);
    }
}

// the (Cb, Cr) levels of chroma texel (x, y)
template <int F>
__device__ __forceinline__ float2 ctexel(const uint8_t* cbase, size_t cpitch, int x, int y) {
    if (F == kFmtNv12) {
        const unsigned short v = __ldg(reinterpret_cast<const unsigned short*>(cbase + (size_t)y * cpitch) + x);
        return make_float2(i2f(v & 255), i2f(v >> 8));
    }
    const uint32_t v = ldw(cbase, cpitch, x, y);
    return make_float2(__fmul_rn(i2f((int)(v & 0xFFFFu)), 0x1p-8f), __fmul_rn(i2f((int)(v >> 16)), 0x1p-8f));
}

// a raw channel -> its level (RGB formats)
template <int F>
__device__ __forceinline__ float levelOf(const FmtConst& f, float r) {
    if (F == kFmtRgb10) return __fmul_rn(r, f.k10);
    if (F == kFmtF16) return f.linear ? fmtPq255(r, f.kWhite) : __fmul_rn(r, 255.0f);
    return r;
}

// ============================================================================================== luma
// the motion estimate's luma of pixel (x, y) in quarter levels (luma.comp:9-27, format.glsl fgLuma)
// pq: linear RgbaF16's table of fmtPq255 by half bits (the same function, evaluated once per value), or null
template <int F>
__device__ __forceinline__ int lumaQ(const FmtConst& f, const uint8_t* base, size_t pitch, int x, int y, const float* pq) {
    float r[3];
    float yl;
    if (F == kFmtF16 && pq) {   // the three channels' PQ levels looked up by their bits
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(base + (size_t)y * pitch) + x);
        const float lr = __ldg(pq + (q.x & 0xFFFFu)), lg = __ldg(pq + (q.x >> 16)), lb = __ldg(pq + (q.y & 0xFFFFu));
        float d = __fmul_rn(4899.0f, lr);
        d = __fadd_rn(d, __fmul_rn(9617.0f, lg));
        d = __fadd_rn(d, __fmul_rn(1868.0f, lb));
        yl = __fmul_rn(d, 1.0f / 16384.0f);
        return __float2int_rn(__fmul_rn(clampF(yl, 0.0f, 255.0f), 4.0f));
    }
    texel<F>(f, base, pitch, x, y, r);
    if (F == kFmtNv12 || F == kFmtP010) {
        yl = __fmul_rn(__fsub_rn(r[0], f.black), f.ys);
    } else {
        const float lr = levelOf<F>(f, r[0]), lg = levelOf<F>(f, r[1]), lb = levelOf<F>(f, r[2]);
        float d = __fmul_rn(4899.0f, lr);
        d = __fadd_rn(d, __fmul_rn(9617.0f, lg));
        d = __fadd_rn(d, __fmul_rn(1868.0f, lb));
        yl = __fmul_rn(d, 1.0f / 16384.0f);
    }
    return __float2int_rn(__fmul_rn(clampF(yl, 0.0f, 255.0f), 4.0f));
}

// integer num / n rounded half to even (num >= 0, n > 0)
__device__ __forceinline__ int rneDiv(int num, int n) {
    int q = num / n;
    const int r = num - q * n;
    if (2 * r > n || (2 * r == n && (q & 1))) q++;
    return q;
}

// interp.flow + pyramid for the other formats: one CTA = a 32x32 level-0 tile and its tower (as k_luma_pyr)
template <int F>
__device__ __forceinline__ void lumaFmtCta(const LumaPyrParams& p, int bx, int by) {
    __shared__ float sl[2][kTowerFloats];
    const int tx0 = bx * 32, ty0 = by * 32;
    const int fw = p.lw[0], fh = p.lh[0], fs = p.fs;
    for (int i = threadIdx.x; i < 1024; i += 256) {
        const int x = tx0 + (i & 31), y = ty0 + (i >> 5);
        float va = 0.0f, vc = 0.0f;
        if (x < fw && y < fh) {
            int sa = 0, sc = 0, n = 0;
            for (int j = 0; j < fs; j++) {
                const int yy = y * fs + j;
                if (yy >= p.H) break;
                for (int k = 0; k < fs; k++) {
                    const int xx = x * fs + k;
                    if (xx >= p.W) break;
                    sa += lumaQ<F>(p.f, p.a, p.pitch, xx, yy, p.pq);
                    sc += lumaQ<F>(p.f, p.c, p.pitch, xx, yy, p.pq);
                    n++;
                }
            }
            va = __fmul_rn(i2f(rneDiv(4 * sa, n)), 1.0f / 16.0f);
            vc = __fmul_rn(i2f(rneDiv(4 * sc, n)), 1.0f / 16.0f);
            p.la[0][(size_t)y * fw + x] = va;
            p.lc[0][(size_t)y * fw + x] = vc;
        }
        sl[0][i] = va;
        sl[1][i] = vc;
    }
    __syncthreads();
    lumaTower<true>(p, sl, tx0, ty0);
}
template <int F>
__global__ void __launch_bounds__(256) k_luma_fmt(const LumaPyrParams p) {
    pdlEnter();
    lumaFmtCta<F>(p, blockIdx.x, blockIdx.y);
}
template <int F>
__global__ void __launch_bounds__(256) k_luma_fmt_m(const __grid_constant__ Merged<LumaPyrParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    lumaFmtCta<F>(m.item[i], bx, by);
}

// ============================================================================================== warps
struct Taps {
    int x0, x1, y0, y1;
    float w00, w01, w10, w11;
};

// the texels and cv2's float weights of the sample point (X, Y) in 1/2^BITS texel units, clamped to w x h
template <int BITS>
__device__ __forceinline__ Taps mkTaps(int X, int Y, int w, int h) {
    Taps t;
    constexpr int mask = (1 << BITS) - 1;
    constexpr float sc = 1.0f / (float)(1 << BITS);
    const int ix = X >> BITS, iy = Y >> BITS;
    const float fx = __fmul_rn(i2f(X & mask), sc), fy = __fmul_rn(i2f(Y & mask), sc);
    const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy);
    t.w00 = __fmul_rn(gy, gx);
    t.w01 = __fmul_rn(gy, fx);
    t.w10 = __fmul_rn(fy, gx);
    t.w11 = __fmul_rn(fy, fx);
    t.x0 = clampi(ix, 0, w - 1); t.x1 = clampi(ix + 1, 0, w - 1);
    t.y0 = clampi(iy, 0, h - 1); t.y1 = clampi(iy + 1, 0, h - 1);
    return t;
}

__device__ __forceinline__ float bil(const Taps& t, float p00, float p01, float p10, float p11) {
    float r = __fmul_rn(p00, t.w00);
    r = __fadd_rn(r, __fmul_rn(p01, t.w01));
    r = __fadd_rn(r, __fmul_rn(p10, t.w10));
    return __fadd_rn(r, __fmul_rn(p11, t.w11));
}

// Integer taps for samples of at most 10 bits (Rgb10 codes, Nv12 bytes). With 1/2^B fractions every product of a
// sample and a weight and every partial sum of mkTaps / bil is an exact multiple of 2^-2B below 2^(10 + 2B - 2B), so
// the float bilinear equals S 2^-2B for the integer S = sum p_ij wx_j wy_i (wx, wy in 0..2^B), in any order. The
// position is clamped to [0, 2^B (n - 1)] and the left tap is min(X >> B, n - 2) with the right weight X - 2^B ix: at
// the right edge the taps (n - 2, n - 1) with weights (0, 2^B) give mkTaps' clamped (n - 1, n - 1) value, below zero
// the taps (0, 1) with weights (2^B, 0) its (0, 0) value (frames are at least 16 x 16, so n >= 2).
struct ITaps {
    int x, y;                 // the top-left tap
    uint32_t w0, w1;          // 16-bit lanes: (w00, w01) and (w10, w11)
};
template <int B>
__device__ __forceinline__ ITaps mkITaps(int X, int Y, int w, int h) {
    constexpr int one = 1 << B;
    X = clampi(X, 0, one * (w - 1));
    Y = clampi(Y, 0, one * (h - 1));
    ITaps t;
    t.x = min(X >> B, w - 2);
    t.y = min(Y >> B, h - 2);
    const uint32_t fx = (uint32_t)(X - one * t.x), fy = (uint32_t)(Y - one * t.y);
    const uint32_t wx = ((uint32_t)one - fx) | (fx << 16);   // lanes <= 2^B: the products below stay under 2^16
    t.w0 = wx * ((uint32_t)one - fy);
    t.w1 = wx * fy;
    return t;
}

// the float taps of warpChroma (formats other than Nv12, and P010 samples off the 10-bit grid)
template <int F>
__device__ __forceinline__ float2 warpChromaF(const uint8_t* cbase, size_t cpitch, int W, int H, int X, int Y) {
    const Taps t = mkTaps<6>(X - 16, Y - 16, (W + 1) >> 1, (H + 1) >> 1);
    const float2 c00 = ctexel<F>(cbase, cpitch, t.x0, t.y0), c01 = ctexel<F>(cbase, cpitch, t.x1, t.y0);
    const float2 c10 = ctexel<F>(cbase, cpitch, t.x0, t.y1), c11 = ctexel<F>(cbase, cpitch, t.x1, t.y1);
    return make_float2(bil(t, c00.x, c01.x, c10.x, c11.x), bil(t, c00.y, c01.y, c10.y, c11.y));
}
// out of line: the rare off-grid P010 case keeps its registers out of the synthesis kernels' hot path
__device__ __noinline__ float2 warpChromaP010Off(const uint8_t* cbase, size_t cpitch, int W, int H, int X, int Y) {
    return warpChromaF<kFmtP010>(cbase, cpitch, W, H, X, Y);
}

// the chroma (Cb, Cr) levels warped to the point whose 1/32-px coordinates are (X, Y)
template <int F>
__device__ __forceinline__ float2 warpChroma(const uint8_t* cbase, size_t cpitch, int W, int H, int X, int Y) {
    if (F == kFmtNv12) {   // byte pairs (Cb, Cr): gathered as (Cb00, Cb01, Cr00, Cr01), two dp2a per channel, exact
        const ITaps t = mkITaps<6>(X - 16, Y - 16, (W + 1) >> 1, (H + 1) >> 1);
        const unsigned short* q0 = reinterpret_cast<const unsigned short*>(cbase + (size_t)t.y * cpitch) + t.x;
        const unsigned short* q1 = reinterpret_cast<const unsigned short*>(cbase + (size_t)(t.y + 1) * cpitch) + t.x;
        const uint32_t c0 = __byte_perm((uint32_t)__ldg(q0), (uint32_t)__ldg(q0 + 1), 0x5140);
        const uint32_t c1 = __byte_perm((uint32_t)__ldg(q1), (uint32_t)__ldg(q1 + 1), 0x5140);
        const uint32_t cb = __dp2a_lo(t.w1, c1, __dp2a_lo(t.w0, c0, 0u)), cr = __dp2a_hi(t.w1, c1, __dp2a_hi(t.w0, c0, 0u));
        return make_float2(__fmul_rn(i2f((int)cb), 0x1p-12f), __fmul_rn(i2f((int)cr), 0x1p-12f));
    }
    if (F == kFmtP010) {   // 10-bit codes in the high bits of 16-bit samples: integer taps when the low 6 bits are zero
        const ITaps t = mkITaps<6>(X - 16, Y - 16, (W + 1) >> 1, (H + 1) >> 1);
        const uint32_t* q0 = reinterpret_cast<const uint32_t*>(cbase + (size_t)t.y * cpitch) + t.x;
        const uint32_t* q1 = reinterpret_cast<const uint32_t*>(cbase + (size_t)(t.y + 1) * cpitch) + t.x;
        const uint32_t p00 = __ldg(q0), p01 = __ldg(q0 + 1), p10 = __ldg(q1), p11 = __ldg(q1 + 1);
        if (((p00 | p01 | p10 | p11) & 0x003F003Fu) == 0u) {   // codes x 64: every float step exact (ITaps)
            const uint32_t w00 = t.w0 & 0xFFFFu, w01 = t.w0 >> 16, w10 = t.w1 & 0xFFFFu, w11 = t.w1 >> 16;
            const uint32_t cb = ((p00 >> 6) & 1023u) * w00 + ((p01 >> 6) & 1023u) * w01 + ((p10 >> 6) & 1023u) * w10 +
                                ((p11 >> 6) & 1023u) * w11;
            const uint32_t cr = (p00 >> 22) * w00 + (p01 >> 22) * w01 + (p10 >> 22) * w10 + (p11 >> 22) * w11;
            return make_float2(__fmul_rn(i2f((int)cb), 0x1p-14f), __fmul_rn(i2f((int)cr), 0x1p-14f));
        }
        return warpChromaP010Off(cbase, cpitch, W, H, X, Y);
    }
    return warpChromaF<F>(cbase, cpitch, W, H, X, Y);
}

// the float taps of a P010 luma sample off the 10-bit grid (out of line, as warpChromaP010Off)
__device__ __noinline__ float warpYP010Off(const uint8_t* base, size_t pitch, int W, int H, int X, int Y) {
    const Taps t = mkTaps<5>(X, Y, W, H);
    auto v = [&](int x, int y) { return __fmul_rn(i2f((int)ldh(base, pitch, x, y)), 0x1p-8f); };
    return bil(t, v(t.x0, t.y0), v(t.x1, t.y0), v(t.x0, t.y1), v(t.x1, t.y1));
}

// the warped sample at (px, py): Rgb10 RGB levels, F16 values, YUV (Y, Cb, Cr) levels
template <int F>
__device__ __forceinline__ void warp(const SynthParams& p, const uint8_t* base, const uint8_t* cbase, float px, float py,
                                     float out[3]) {
    const int X = rne32(px), Y = rne32(py);
    if (F == kFmtRgb10) {   // 10-bit codes: integer taps, exact (ITaps)
        const ITaps t = mkITaps<5>(X, Y, p.W, p.H);
        const uint32_t* q0 = reinterpret_cast<const uint32_t*>(base + (size_t)t.y * p.pitch) + t.x;
        const uint32_t* q1 = reinterpret_cast<const uint32_t*>(base + (size_t)(t.y + 1) * p.pitch) + t.x;
        const uint32_t p00 = __ldg(q0), p01 = __ldg(q0 + 1), p10 = __ldg(q1), p11 = __ldg(q1 + 1);
        const uint32_t w00 = t.w0 & 0xFFFFu, w01 = t.w0 >> 16, w10 = t.w1 & 0xFFFFu, w11 = t.w1 >> 16;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int sh = p.f.rHigh ? 20 - 10 * k : 10 * k;
            const uint32_t S = ((p00 >> sh) & 1023u) * w00 + ((p01 >> sh) & 1023u) * w01 + ((p10 >> sh) & 1023u) * w10 +
                               ((p11 >> sh) & 1023u) * w11;
            out[k] = __fmul_rn(__fmul_rn(i2f((int)S), 0x1p-10f), p.f.k10);
        }
        return;
    }
    if (F == kFmtNv12) {    // 8-bit luma: integer taps, two dp2a (as the 8-bit RGBA sampler), exact
        const ITaps t = mkITaps<5>(X, Y, p.W, p.H);
        const uint8_t* q0 = base + (size_t)t.y * p.pitch + t.x;
        const uint8_t* q1 = q0 + p.pitch;
        const uint32_t r0 = (uint32_t)__ldg(q0) | ((uint32_t)__ldg(q0 + 1) << 8);
        const uint32_t r1 = (uint32_t)__ldg(q1) | ((uint32_t)__ldg(q1 + 1) << 8);
        out[0] = __fmul_rn(i2f((int)__dp2a_lo(t.w1, r1, __dp2a_lo(t.w0, r0, 0u))), 0x1p-10f);
        const float2 c = warpChroma<F>(cbase, p.cpitch, p.W, p.H, X, Y);
        out[1] = c.x;
        out[2] = c.y;
        return;
    }
    if (F == kFmtP010) {    // integer taps when the four samples' low 6 bits are zero (then every float step is exact)
        const ITaps t = mkITaps<5>(X, Y, p.W, p.H);
        const unsigned short* q0 = reinterpret_cast<const unsigned short*>(base + (size_t)t.y * p.pitch) + t.x;
        const unsigned short* q1 = reinterpret_cast<const unsigned short*>(base + (size_t)(t.y + 1) * p.pitch) + t.x;
        const uint32_t s00 = __ldg(q0), s01 = __ldg(q0 + 1), s10 = __ldg(q1), s11 = __ldg(q1 + 1);
        if (((s00 | s01 | s10 | s11) & 63u) == 0u) {
            const uint32_t S = (s00 >> 6) * (t.w0 & 0xFFFFu) + (s01 >> 6) * (t.w0 >> 16) + (s10 >> 6) * (t.w1 & 0xFFFFu) +
                               (s11 >> 6) * (t.w1 >> 16);
            out[0] = __fmul_rn(i2f((int)S), 0x1p-12f);   // codes / 4 = the levels
        } else {
            out[0] = warpYP010Off(base, p.pitch, p.W, p.H, X, Y);
        }
        const float2 c = warpChroma<F>(cbase, p.cpitch, p.W, p.H, X, Y);
        out[1] = c.x;
        out[2] = c.y;
        return;
    }
    const Taps t = mkTaps<5>(X, Y, p.W, p.H);
    float r00[3], r01[3], r10[3], r11[3];
    texel<F>(p.f, base, p.pitch, t.x0, t.y0, r00);
    texel<F>(p.f, base, p.pitch, t.x1, t.y0, r01);
    texel<F>(p.f, base, p.pitch, t.x0, t.y1, r10);
    texel<F>(p.f, base, p.pitch, t.x1, t.y1, r11);
    if (F == kFmtNv12 || F == kFmtP010) {
        out[0] = bil(t, r00[0], r01[0], r10[0], r11[0]);
        const float2 c = warpChroma<F>(cbase, p.cpitch, p.W, p.H, X, Y);
        out[1] = c.x;
        out[2] = c.y;
    } else {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float r = bil(t, r00[k], r01[k], r10[k], r11[k]);
            out[k] = F == kFmtRgb10 ? __fmul_rn(r, p.f.k10) : r;
        }
    }
}

// format.glsl FG_DIFF + FG_PACKE: the max-channel difference in levels, truncated, at most 255
template <int F>
__device__ __forceinline__ int mismatch(const FmtConst& f, const float wa[3], const float wc[3]) {
    float m;
    if (F == kFmtNv12 || F == kFmtP010) {
        const float dy = __fsub_rn(wa[0], wc[0]), db = __fsub_rn(wa[1], wc[1]), dr = __fsub_rn(wa[2], wc[2]);
        const float y = __fmul_rn(f.ys, dy);
        const float r = __fadd_rn(y, __fmul_rn(f.rcr, dr));
        const float g = __fadd_rn(__fadd_rn(y, __fmul_rn(f.gcb, db)), __fmul_rn(f.gcr, dr));
        const float b = __fadd_rn(y, __fmul_rn(f.bcb, db));
        m = fmaxf(fabsf(r), fmaxf(fabsf(g), fabsf(b)));
    } else {
        m = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float d;
            if (F == kFmtF16 && f.linear) d = fabsf(__fsub_rn(fmtPq255(wa[k], f.kWhite), fmtPq255(wc[k], f.kWhite)));
            else if (F == kFmtF16) d = fabsf(__fsub_rn(__fmul_rn(wa[k], 255.0f), __fmul_rn(wc[k], 255.0f)));
            else d = fabsf(__fsub_rn(wa[k], wc[k]));
            m = fmaxf(m, d);
        }
    }
    return (int)fminf(m, 255.0f);
}

// resolve.comp: m = 0.5 (a + c) at t = 0.5, else (1 - t) a + t c; out = m (1 - u) + n u
__device__ __forceinline__ float mixF(float a, float c, const SynthParams& p) {
    return p.mid ? __fmul_rn(0.5f, __fadd_rn(a, c)) : __fadd_rn(__fmul_rn(p.wA, a), __fmul_rn(p.wC, c));
}
__device__ __forceinline__ float blendM(float m, float n, float u, float iu) {
    return __fadd_rn(__fmul_rn(m, iu), __fmul_rn(n, u));
}

// the nearer frame over one output pixel (and, for YUV, the chroma texel of an even-even pixel)
template <int F>
__device__ __forceinline__ void copyNear(const SynthParams& p, int x, int y) {
    const uint8_t* n = p.nearC ? p.c : p.a;
    uint8_t* o = p.out + (size_t)y * p.outPitch;
    if (F == kFmtRgb10) {
        reinterpret_cast<uint32_t*>(o)[x] = ldw(n, p.pitch, x, y);
    } else if (F == kFmtF16) {
        reinterpret_cast<uint2*>(o)[x] = __ldg(reinterpret_cast<const uint2*>(n + (size_t)y * p.pitch) + x);
    } else {
        if (F == kFmtNv12) o[x] = __ldg(n + (size_t)y * p.pitch + x);
        else reinterpret_cast<unsigned short*>(o)[x] = (unsigned short)ldh(n, p.pitch, x, y);
        if (((x | y) & 1) == 0) {
            const uint8_t* nc = p.nearC ? p.cc : p.ac;
            uint8_t* oc = p.outc + (size_t)(y >> 1) * p.outCPitch;
            if (F == kFmtNv12)
                reinterpret_cast<unsigned short*>(oc)[x >> 1] =
                    __ldg(reinterpret_cast<const unsigned short*>(nc + (size_t)(y >> 1) * p.cpitch) + (x >> 1));
            else
                reinterpret_cast<uint32_t*>(oc)[x >> 1] = ldw(nc, p.cpitch, x >> 1, y >> 1);
        }
    }
}

// ============================================================================================== synthesis
// interp.synth for one t in the other formats: the 8-bit path's tile (k_synth) with each format's warp, mismatch,
// blend and store (resolve.comp:48-83). YUV: the chroma of each 2x2 block is written with its even-even pixel, warped
// from the block centre with that pixel's half-vector and blended with that pixel's trust.
//
// synthFmtTile computes one output tile and hands every output value to a sink: word(k, x, y, w) for Rgb10 (the
// packed pixel), half4(k, x, y, v) for RgbaF16 (four halves), luma(k, x, y, code) and chroma(k, x, y, cb, cr) for
// YUV (codes; chroma for even-even pixels only); k is the thread's region-row slot. kCut: under a scene cut the tile is
// a copy of the nearer frame (and the core returns); without kCut the caller has taken the cut into account. The
// untrusted count goes to *p.untrusted unless that is null.
// kUi: CrosshairV2's warp-tap rejection (gpu/shaders/ui_reject.glsl): a tap whose footprint (YUV: the 2x2 chroma
// texels around it) touches its own frame's UI mask (p.uiA / p.uiC) takes the other frame's tap (both or neither:
// kept); the block-centre chroma of the even-even pixels is rejected on its own positions (uiRejectC)
template <int F, bool kCut, bool kUi = false, class Sink>
__device__ __forceinline__ void synthFmtTile(const SynthParams& p, int bx, int by, Sink& sink) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ SyCoef rowc[kSyEH];
    __shared__ unsigned int cnt;
    __shared__ int gReg[4];
    const int X0 = bx * kSyT, Y0 = by * kSyTH;
    const int tid = threadIdx.x, ex = tid & (kSyE - 1), ey0 = tid / kSyE;
    if (kCut && p.st->cut) {   // scene cut (interp.py:225-226): the nearer real frame
        for (int i = tid; i < kSyT * kSyTH; i += kSyThreads) {
            const int x = X0 + (i % kSyT), y = Y0 + (i / kSyT);
            if (x < p.W && y < p.H) copyNear<F>(p, x, y);
        }
        return;
    }
    if (tid == 0) cnt = 0;
    float2* hrow;
    uint8_t* e;
    unsigned short* hsum;
    const SyCoef cx = syFieldStage(p, X0, Y0, tid, ex, ey0, rowc, gReg, sm, hrow, e, hsum);
    const float kA = p.mid ? 1.0f : p.ka, kC = p.mid ? 1.0f : p.kc;
    constexpr bool kYuv = F == kFmtNv12 || F == kFmtP010;
    // the blend inputs m of the output pixels, kept from stage 2 for stage 4 (the warps are computed once): per channel
    // planes of kSyTH x kSyE floats (YUV: the luma plane, then the block-centre chroma (Cb, Cr) of the even-even
    // pixels, (kSyTH / 2) x (kSyE / 2))
    float* mix = reinterpret_cast<float*>(hsum + kSyEH * kSyHS);
    float2* mixc = reinterpret_cast<float2*>(mix + kSyTH * kSyE);
    const int lx = ex - kSyAp, x = X0 + lx;
    // 2. the mismatch over the region, and the blend inputs of the output pixels
    for (int k = 0; k < kSyK; k++) {
        const int ey = ey0 + (kSyThreads / kSyE) * k;
        const SyCoef cy = rowc[ey];
        const float2 h = syHalfVec(cy, hrow, ex);
        float wa[3], wc[3];
        const float pax = __fsub_rn(cx.pos, __fmul_rn(kA, h.x)), pay = __fsub_rn(cy.pos, __fmul_rn(kA, h.y));
        const float pcx = __fadd_rn(cx.pos, __fmul_rn(kC, h.x)), pcy = __fadd_rn(cy.pos, __fmul_rn(kC, h.y));
        warp<F>(p, p.a, p.ac, pax, pay, wa);
        warp<F>(p, p.c, p.cc, pcx, pcy, wc);
        if (kUi) {
            const bool ha = p.uiA && (kYuv ? uiHitMaskYuv(p.uiA, rne32(pax), rne32(pay)) : uiHitMask(p.uiA, rne32(pax), rne32(pay)));
            const bool hc = p.uiC && (kYuv ? uiHitMaskYuv(p.uiC, rne32(pcx), rne32(pcy)) : uiHitMask(p.uiC, rne32(pcx), rne32(pcy)));
            if (ha != hc) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if (ha) wa[c] = wc[c];
                    else wc[c] = wa[c];
                }
            }
        }
        e[ey * kSyES + ex] = (uint8_t)mismatch<F>(p.f, wa, wc);
        const int ly = ey - kSyAp;
        if ((unsigned)ly < (unsigned)kSyTH) {   // warp-uniform
            if (kYuv) {
                mix[ly * kSyE + ex] = mixF(wa[0], wc[0], p);
                if ((((lx | ly) & 1) == 0) && (unsigned)lx < (unsigned)kSyT && x < p.W && Y0 + ly < p.H) {
                    // the chroma of this 2x2 block, warped from its centre with this pixel's half-vector
                    const float bx = __fadd_rn(cx.pos, 0.5f), by = __fadd_rn(cy.pos, 0.5f);
                    const float qax = __fsub_rn(bx, __fmul_rn(kA, h.x)), qay = __fsub_rn(by, __fmul_rn(kA, h.y));
                    const float qcx = __fadd_rn(bx, __fmul_rn(kC, h.x)), qcy = __fadd_rn(by, __fmul_rn(kC, h.y));
                    float2 ca = warpChroma<F>(p.ac, p.cpitch, p.W, p.H, rne32(qax), rne32(qay));
                    float2 cc = warpChroma<F>(p.cc, p.cpitch, p.W, p.H, rne32(qcx), rne32(qcy));
                    if (kUi) {   // uiRejectC: the block-centre taps, with their own footprints
                        const bool ha = p.uiA && uiHitMaskYuv(p.uiA, rne32(qax), rne32(qay));
                        const bool hc = p.uiC && uiHitMaskYuv(p.uiC, rne32(qcx), rne32(qcy));
                        if (ha != hc) {
                            if (ha) ca = cc;
                            else cc = ca;
                        }
                    }
                    mixc[(ly >> 1) * (kSyE / 2) + (lx >> 1)] = make_float2(mixF(ca.x, cc.x, p), mixF(ca.y, cc.y, p));
                }
            } else {
#pragma unroll
                for (int c = 0; c < 3; c++) mix[(c * kSyTH + ly) * kSyE + ex] = mixF(wa[c], wc[c], p);
            }
        }
    }
    __syncthreads();
    // 3. horizontal 7-sums (as k_synth)
    syRowSums(e, hsum, tid);
    __syncthreads();
    // 4. output pixels: vertical 7-sum, trust, blend, store
    unsigned int myCnt = 0;
    if ((unsigned)lx < (unsigned)kSyT && x < p.W) {
        const uint8_t* nearF = p.nearC ? p.c : p.a;
#pragma unroll
        for (int k = 0; k < kSyK; k++) {
            const int ey = ey0 + (kSyThreads / kSyE) * k, ly = ey - kSyAp, y = Y0 + ly;
            if ((unsigned)ly >= (unsigned)kSyTH || y >= p.H) continue;
            const unsigned short* q = hsum + ly * kSyHS + lx;
            const int S = q[0] + q[kSyHS] + q[2 * kSyHS] + q[3 * kSyHS] + q[4 * kSyHS] + q[5 * kSyHS] + q[6 * kSyHS];
            float u, iu;
            if (S <= p.sZero) {          // the ramp is exactly 0 (host-derived threshold)
                u = 0.0f;
                iu = 1.0f;
            } else if (S >= p.sOne) {    // exactly 1
                u = 1.0f;
                iu = 0.0f;
            } else {
                const float eb = (float)((double)S * (1.0 / 49.0));   // cv2.blur: double sum * (1/49), to float
                u = clampF(__fdiv_rn(__fsub_rn(eb, p.trust0), p.trustSpan), 0.0f, 1.0f);
                iu = __fsub_rn(1.0f, u);
            }
            myCnt += u > 0.5f;
            if (F == kFmtRgb10) {
                const uint32_t nw = ldw(nearF, p.pitch, x, y);
                uint32_t ow = nw & 0xC0000000u;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float nl = __fmul_rn(i2f(rgb10(p.f, nw, c)), p.f.k10);
                    const float v = clampF(blendM(mix[(c * kSyTH + ly) * kSyE + ex], nl, u, iu), 0.0f, 255.0f);
                    const int code = clampi((int)floorf(__fadd_rn(__fmul_rn(v, p.f.k10i), 0.5f)), 0, 1023);
                    ow |= (uint32_t)code << (p.f.rHigh ? 20 - 10 * c : 10 * c);
                }
                sink.word(k, x, y, ow);
            } else if (F == kFmtF16) {
                const uint2 nq = __ldg(reinterpret_cast<const uint2*>(nearF + (size_t)y * p.pitch) + x);
                const float n0 = h2f(nq.x & 0xFFFFu), n1 = h2f(nq.x >> 16), n2 = h2f(nq.y & 0xFFFFu);
                const uint32_t o0 = __half_as_ushort(__float2half_rn(blendM(mix[(0 * kSyTH + ly) * kSyE + ex], n0, u, iu)));
                const uint32_t o1 = __half_as_ushort(__float2half_rn(blendM(mix[(1 * kSyTH + ly) * kSyE + ex], n1, u, iu)));
                const uint32_t o2 = __half_as_ushort(__float2half_rn(blendM(mix[(2 * kSyTH + ly) * kSyE + ex], n2, u, iu)));
                sink.half4(k, x, y, make_uint2(o0 | (o1 << 16), o2 | (nq.y & 0xFFFF0000u)));
            } else {
                constexpr float ql = F == kFmtP010 ? 4.0f : 1.0f;   // 1 / YU_QL
                constexpr int codes = F == kFmtP010 ? 1023 : 255;
                float ny[3];
                texel<F>(p.f, nearF, p.pitch, x, y, ny);
                const float v = blendM(mix[ly * kSyE + ex], ny[0], u, iu);
                sink.luma(k, x, y, clampi((int)floorf(__fadd_rn(__fmul_rn(v, ql), 0.5f)), 0, codes));
                if (((x | y) & 1) == 0) {   // the chroma of this 2x2 block (warped in stage 2)
                    const float2 m = mixc[(ly >> 1) * (kSyE / 2) + (lx >> 1)];
                    const float2 nc = ctexel<F>(p.nearC ? p.cc : p.ac, p.cpitch, x >> 1, y >> 1);
                    const int cb = clampi((int)floorf(__fadd_rn(__fmul_rn(blendM(m.x, nc.x, u, iu), ql), 0.5f)), 0, codes);
                    const int cr = clampi((int)floorf(__fadd_rn(__fmul_rn(blendM(m.y, nc.y, u, iu), ql), 0.5f)), 0, codes);
                    sink.chroma(k, x, y, cb, cr);
                }
            }
            if (p.emap) p.emap[(size_t)y * ((p.W + 3) & ~3) + x] = e[ey * kSyES + ex];
        }
    }
    if (myCnt) atomicAdd(&cnt, myCnt);
    __syncthreads();
    if (tid == 0 && cnt && p.untrusted) atomicAdd(p.untrusted, cnt);
}

// the store of a synthesis: the values go to p.out (and p.outc) in the format's layout
template <int F>
struct FmtStore {
    const SynthParams& p;
    __device__ __forceinline__ void word(int, int x, int y, uint32_t w) const {
        reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] = w;
    }
    __device__ __forceinline__ void half4(int, int x, int y, uint2 v) const {
        reinterpret_cast<uint2*>(p.out + (size_t)y * p.outPitch)[x] = v;
    }
    __device__ __forceinline__ void luma(int, int x, int y, int code) const {
        uint8_t* orow = p.out + (size_t)y * p.outPitch;
        if (F == kFmtP010) reinterpret_cast<unsigned short*>(orow)[x] = (unsigned short)(code << 6);
        else orow[x] = (uint8_t)code;
    }
    __device__ __forceinline__ void chroma(int, int x, int y, int cb, int cr) const {
        uint8_t* oc = p.outc + (size_t)(y >> 1) * p.outCPitch;
        if (F == kFmtP010) reinterpret_cast<uint32_t*>(oc)[x >> 1] = ((uint32_t)cb << 6) | ((uint32_t)cr << 22);
        else reinterpret_cast<unsigned short*>(oc)[x >> 1] = (unsigned short)(cb | (cr << 8));
    }
};

template <int F>
__global__ void __launch_bounds__(kSyThreads, 3) k_synth_fmt(const SynthParams p) {
    pdlEnter();
    FmtStore<F> store{p};
    synthFmtTile<F, true>(p, blockIdx.x, blockIdx.y, store);
}
// the same with CrosshairV2's tap rejection (Rgb10 / RgbaF16); a separate kernel so the plain one is unchanged
template <int F>
__global__ void __launch_bounds__(kSyThreads, 3) k_synth_fmt_ui(const SynthParams p) {
    pdlEnter();
    FmtStore<F> store{p};
    synthFmtTile<F, true, true>(p, blockIdx.x, blockIdx.y, store);
}

// Many syntheses of one format in one persistent launch (as k_synth_batch for 8-bit RGBA): every CTA takes the next
// tile of the work list from an atomic counter until the list is exhausted; an item's parameters are staged in shared
// memory per tile.
template <int F>
__global__ void __launch_bounds__(kSyThreads, 3) k_synth_fmt_batch(const SynthBatchArgs b) {
    pdlEnter();
    __shared__ int work, item;
    __shared__ __align__(16) SynthParams sp;
    for (;;) {
        if (threadIdx.x == 0) {
            work = (int)atomicAdd(b.counter, 1u);
            int lo = 0, hi = b.nItems - 1;   // the item whose tile range holds `work`
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (b.tileStart[mid] <= work) lo = mid; else hi = mid - 1;
            }
            item = lo;
        }
        __syncthreads();
        const int w = work, it = item;
        if (w >= b.total) break;
        for (int i = threadIdx.x; i < (int)(sizeof(SynthParams) / 4); i += kSyThreads)
            reinterpret_cast<uint32_t*>(&sp)[i] = __ldg(reinterpret_cast<const uint32_t*>(b.items + it) + i);
        __syncthreads();
        const int t = w - b.tileStart[it], tx = b.tilesX[it];
        FmtStore<F> store{sp};
        synthFmtTile<F, true>(sp, t % tx, t / tx, store);
        __syncthreads();   // the tile's shared memory is free again
    }
}

// ============================================================================================== motion blur
// recordSynthBlur in the other formats (gpu/framegen.h:553-573): the weighted average of n sub-frames, each the
// values recordSynth(t_k) stores, rounded once. Integer formats (Rgb10 codes, Nv12 / P010 luma and chroma codes):
// sum q_k v_k with integer weights summing to 2^16, (acc + 2^15) >> 16, in any order (exact). RgbaF16: float32 sums of
// fl32(w_k h_k), w_k = q_k 2^-16 (exact), in sample order, then rounded to half. A sample replaced by a real frame
// (scene cut, flick, t <= 0 / >= 1) adds that frame's values at its place in the order. Alpha (Rgb10's 2 bits,
// RgbaF16's half) is every sub-frame's nearer frame's, averaged the same way.
template <int F>
struct FmtAcc {
    uint32_t (&ai)[kSyK][3];   // integer formats: codes (Rgb10 by bit position; YUV: Y, Cb, Cr)
    float (&af)[kSyK][3];      // RgbaF16: the colour halves
    uint32_t q;
    float w;
    __device__ __forceinline__ void word(int k, int, int, uint32_t v) const {
#pragma unroll
        for (int c = 0; c < 3; c++) ai[k][c] += q * ((v >> (10 * c)) & 1023u);
    }
    __device__ __forceinline__ void half4(int k, int, int, uint2 v) const {
        af[k][0] = __fadd_rn(af[k][0], __fmul_rn(w, h2f(v.x & 0xFFFFu)));
        af[k][1] = __fadd_rn(af[k][1], __fmul_rn(w, h2f(v.x >> 16)));
        af[k][2] = __fadd_rn(af[k][2], __fmul_rn(w, h2f(v.y & 0xFFFFu)));
    }
    __device__ __forceinline__ void luma(int k, int, int, int code) const { ai[k][0] += q * (uint32_t)code; }
    __device__ __forceinline__ void chroma(int k, int, int, int cb, int cr) const {
        ai[k][1] += q * (uint32_t)cb;
        ai[k][2] += q * (uint32_t)cr;
    }
};

// the values a real frame (base pointers a: plane 0, ac: CbCr) holds at (x, y), handed to the sink as a synthesis
// would hand them
template <int F, class Sink>
__device__ __forceinline__ void frameValues(const SynthParams& p, const uint8_t* a, const uint8_t* ac, int k, int x,
                                            int y, Sink& sink) {
    if (F == kFmtRgb10) {
        sink.word(k, x, y, ldw(a, p.pitch, x, y));
    } else if (F == kFmtF16) {
        sink.half4(k, x, y, __ldg(reinterpret_cast<const uint2*>(a + (size_t)y * p.pitch) + x));
    } else if (F == kFmtP010) {
        sink.luma(k, x, y, __ldg(reinterpret_cast<const unsigned short*>(a + (size_t)y * p.pitch) + x) >> 6);
        if (((x | y) & 1) == 0) {
            const uint32_t cw = __ldg(reinterpret_cast<const uint32_t*>(ac + (size_t)(y >> 1) * p.cpitch) + (x >> 1));
            sink.chroma(k, x, y, (int)((cw >> 6) & 1023u), (int)(cw >> 22));
        }
    } else {
        sink.luma(k, x, y, __ldg(a + (size_t)y * p.pitch + x));
        if (((x | y) & 1) == 0) {
            const uint32_t cw = __ldg(reinterpret_cast<const unsigned short*>(ac + (size_t)(y >> 1) * p.cpitch) + (x >> 1));
            sink.chroma(k, x, y, (int)(cw & 255u), (int)(cw >> 8));
        }
    }
}

template <int F, bool kUi = false>
__global__ void __launch_bounds__(kSyThreads, 1) k_synth_blur_fmt(const BlurParams bp) {
    pdlEnter();
    __shared__ __align__(16) SynthParams sp;
    __shared__ unsigned int sRepl, sRedo, sNearC;   // replaced samples; whether this pass has work; nearer = curr
    __shared__ uint32_t sWap;                        // the weight of the samples whose nearer frame is prev
    const int tid = threadIdx.x, ex = tid & (kSyE - 1), ey0 = tid / kSyE;
    const SynthParams& b = bp.base;
    if (tid == 0) {
        const bool cut = b.st->cut != 0;
        unsigned int repl = 0, flick = 0, nearc = 0;
        uint32_t wap = 0;
        for (int k = 0; k < bp.n; k++) {
            const BlurSample& m = bp.smp[k];
            const bool nc = m.mode == 2 || (m.mode == 0 && m.nearC);
            bool r = m.mode != 0 || cut;
            if (!r && bp.fix && (double)bp.cnt[k] / ((double)b.W * (double)b.H) > bp.frac) {
                r = true;
                flick |= 1u << k;
            }
            if (r) repl |= 1u << k;
            if (nc) nearc |= 1u << k; else wap += m.q;
        }
        sRepl = repl;
        sRedo = !bp.fix || flick != 0;
        sNearC = nearc;
        sWap = wap;
    }
    __syncthreads();
    if (!sRedo) return;
    const unsigned int repl = sRepl, nearc = sNearC;
    uint32_t ai[kSyK][3];
    float af[kSyK][3];
#pragma unroll
    for (int k = 0; k < kSyK; k++) {
        ai[k][0] = ai[k][1] = ai[k][2] = 0u;
        af[k][0] = af[k][1] = af[k][2] = 0.0f;
    }
    FmtAcc<F> acc{ai, af, 0u, 0.0f};
    const int lx = ex - kSyAp, x = blockIdx.x * kSyT + lx;
    const bool colOk = (unsigned)lx < (unsigned)kSyT && x < b.W;
    for (int j = 0; j < bp.n; j++) {
        acc.q = bp.smp[j].q;
        acc.w = __fmul_rn((float)bp.smp[j].q, 1.0f / 65536.0f);
        if ((repl >> j) & 1u) {   // a real frame in the sample's place (uniform over the CTA)
            const bool nc = (nearc >> j) & 1u;
            if (colOk) {
#pragma unroll
                for (int k = 0; k < kSyK; k++) {
                    const int ly = ey0 + (kSyThreads / kSyE) * k - kSyAp, y = blockIdx.y * kSyTH + ly;
                    if ((unsigned)ly < (unsigned)kSyTH && y < b.H) frameValues<F>(b, nc ? b.c : b.a, nc ? b.cc : b.ac, k, x, y, acc);
                }
            }
            continue;
        }
        static_assert(sizeof(SynthParams) % 4 == 0, "SynthParams copies as words");
        for (int i = tid; i < (int)(sizeof(SynthParams) / 4); i += kSyThreads)
            reinterpret_cast<uint32_t*>(&sp)[i] = reinterpret_cast<const uint32_t*>(&b)[i];
        __syncthreads();
        if (tid == 0) {
            const BlurSample& m = bp.smp[j];
            sp.lookup = m.lookup; sp.mid = m.mid; sp.nearC = m.nearC;
            sp.s = m.s; sp.ka = m.ka; sp.kc = m.kc; sp.wA = m.wA; sp.wC = m.wC;
            sp.untrusted = bp.fix ? nullptr : bp.cnt + j;
            sp.emap = nullptr;
        }
        __syncthreads();
        synthFmtTile<F, false, kUi>(sp, blockIdx.x, blockIdx.y, acc);
        __syncthreads();   // the tile's shared memory and sp are free again
    }
    if (!colOk) return;
    const uint32_t wap = sWap, wac = 65536u - wap;
#pragma unroll
    for (int k = 0; k < kSyK; k++) {
        const int ly = ey0 + (kSyThreads / kSyE) * k - kSyAp, y = blockIdx.y * kSyTH + ly;
        if ((unsigned)ly >= (unsigned)kSyTH || y >= b.H) continue;
        uint8_t* orow = b.out + (size_t)y * b.outPitch;
        if (F == kFmtRgb10) {
            const uint32_t pa = ldw(b.a, b.pitch, x, y) >> 30, pc = ldw(b.c, b.pitch, x, y) >> 30;
            uint32_t w = ((wap * pa + wac * pc + 32768u) >> 16) << 30;
#pragma unroll
            for (int c = 0; c < 3; c++) w |= ((ai[k][c] + 32768u) >> 16) << (10 * c);
            reinterpret_cast<uint32_t*>(orow)[x] = w;
        } else if (F == kFmtF16) {
            const float aa = h2f(__ldg(reinterpret_cast<const uint2*>(b.a + (size_t)y * b.pitch) + x).y >> 16);
            const float ac = h2f(__ldg(reinterpret_cast<const uint2*>(b.c + (size_t)y * b.pitch) + x).y >> 16);
            float al = 0.0f;   // alpha: the nearer frames' in sample order
            for (int j = 0; j < bp.n; j++)
                al = __fadd_rn(al, __fmul_rn(__fmul_rn((float)bp.smp[j].q, 1.0f / 65536.0f), ((nearc >> j) & 1u) ? ac : aa));
            const uint32_t o0 = __half_as_ushort(__float2half_rn(af[k][0])), o1 = __half_as_ushort(__float2half_rn(af[k][1]));
            const uint32_t o2 = __half_as_ushort(__float2half_rn(af[k][2])), o3 = __half_as_ushort(__float2half_rn(al));
            reinterpret_cast<uint2*>(orow)[x] = make_uint2(o0 | (o1 << 16), o2 | (o3 << 16));
        } else {
            const uint32_t yc = (ai[k][0] + 32768u) >> 16;
            if (F == kFmtP010) reinterpret_cast<unsigned short*>(orow)[x] = (unsigned short)(yc << 6);
            else orow[x] = (uint8_t)yc;
            if (((x | y) & 1) == 0) {
                const uint32_t cb = (ai[k][1] + 32768u) >> 16, cr = (ai[k][2] + 32768u) >> 16;
                uint8_t* oc = b.outc + (size_t)(y >> 1) * b.outCPitch;
                if (F == kFmtP010) reinterpret_cast<uint32_t*>(oc)[x >> 1] = (cb << 6) | (cr << 22);
                else reinterpret_cast<unsigned short*>(oc)[x >> 1] = (unsigned short)(cb | (cr << 8));
            }
        }
    }
}

// interp.py:238-239 for the other formats: more than globalFallback of the pixels untrusted -> the nearer real frame
// (both planes of YUV) over the output. Every CTA exits at once in the normal case; clears the next synth's counter.
__device__ __forceinline__ void fallbackFmtCta(const FallbackParams& p) {
    const unsigned int cnt = *p.untrusted;
    if (!((double)cnt / ((double)p.W * (double)p.H) > p.frac)) return;
    const uint8_t* n = p.nearC ? p.c : p.a;
    const size_t stride = (size_t)gridDim.x * 256;
    const size_t n0 = p.rowBytes * (size_t)p.H;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n0; i += stride) {
        const size_t y = i / p.rowBytes, b = i % p.rowBytes;
        p.out[y * p.outPitch + b] = __ldg(n + y * p.pitch + b);
    }
    if (p.outc) {
        const uint8_t* nc = p.nearC ? p.cc : p.ac;
        const size_t n1 = p.cbytes * (size_t)p.ch;
        for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n1; i += stride) {
            const size_t y = i / p.cbytes, b = i % p.cbytes;
            p.outc[y * p.outCPitch + b] = __ldg(nc + y * p.cpitch + b);
        }
    }
}

__global__ void __launch_bounds__(256) k_fallback_fmt(const FallbackParams p) {
    pdlEnter();
    if (blockIdx.x == 0 && threadIdx.x == 0) *p.untrustedNext = 0;
    fallbackFmtCta(p);
}
// the untrusted-share decision of many syntheses of the other formats (grid.y = item; the item counters are zeroed by
// the host before the batch's synthesis launch)
__global__ void __launch_bounds__(256) k_fallback_fmt_batch(const FallbackParams* __restrict__ items) {
    pdlEnter();
    fallbackFmtCta(items[blockIdx.y]);
}

// ============================================================================================== launchers
// the dynamic shared memory of a format synthesis: synthSmemBytes + the blend inputs of the output pixels
static size_t fmtSynthSmem(int format, int fs) {
    const size_t mix = format == kFmtNv12 || format == kFmtP010
                           ? (size_t)kSyTH * kSyE * 4 + (size_t)((kSyTH + 1) / 2) * (kSyE / 2) * 8
                           : (size_t)3 * kSyTH * kSyE * 4;
    return synthSmemBytes(fs) + mix;
}

cudaError_t prepareFormatKernels() {
    const int smem = (int)fmtSynthSmem(kFmtRgb10, 1);   // the largest
    cudaError_t e = cudaFuncSetAttribute(k_synth_fmt<kFmtRgb10>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt<kFmtF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt<kFmtNv12>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt<kFmtP010>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_batch<kFmtRgb10>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_batch<kFmtF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_batch<kFmtNv12>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_batch<kFmtP010>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_ui<kFmtRgb10>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_ui<kFmtF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_ui<kFmtNv12>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_fmt_ui<kFmtP010>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtNv12, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtP010, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtRgb10, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtF16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtRgb10>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtNv12>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_blur_fmt<kFmtP010>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

cudaError_t launchLumaFmt(const LumaPyrParams& p, cudaStream_t s) {
    const dim3 grid(divUp(p.lw[0], 32), divUp(p.lh[0], 32));
    switch (p.f.format) {
        case kFmtRgb10: return launchPdl(k_luma_fmt<kFmtRgb10>, grid, dim3(256), 0, s, p);
        case kFmtF16: return launchPdl(k_luma_fmt<kFmtF16>, grid, dim3(256), 0, s, p);
        case kFmtNv12: return launchPdl(k_luma_fmt<kFmtNv12>, grid, dim3(256), 0, s, p);
        case kFmtP010: return launchPdl(k_luma_fmt<kFmtP010>, grid, dim3(256), 0, s, p);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchLumaFmtMerged(Merged<LumaPyrParams>& m, int format, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    int total = 0;
    for (int i = 0; i < m.n; i++) {
        m.first[i] = total;
        m.gx[i] = (int)divUp(m.item[i].lw[0], 32);
        total += m.gx[i] * (int)divUp(m.item[i].lh[0], 32);
    }
    m.first[m.n] = total;
    switch (format) {
        case kFmtRgb10: return launchPdl(k_luma_fmt_m<kFmtRgb10>, dim3(total), dim3(256), 0, s, m);
        case kFmtF16: return launchPdl(k_luma_fmt_m<kFmtF16>, dim3(total), dim3(256), 0, s, m);
        case kFmtNv12: return launchPdl(k_luma_fmt_m<kFmtNv12>, dim3(total), dim3(256), 0, s, m);
        case kFmtP010: return launchPdl(k_luma_fmt_m<kFmtP010>, dim3(total), dim3(256), 0, s, m);
        default: return cudaErrorInvalidValue;
    }
}

// CrosshairV2's estimate fill (gpu/shaders/ui_v2_lumafill.comp) for Rgb10 / RgbaF16 frames, as k_ui_v2_fill for 8-bit
// RGBA with the format's luma: a level-0 cell holding a UI pixel takes the luma of its not-UI pixels, the window
// widened by fs px per step up to 8 px while it has none, formed as the luma pass forms a cell (quarter levels summed,
// rneDiv(4 sum, n) / 16, so the estimate's sums stay exact)
template <int F>
__global__ void __launch_bounds__(64) k_ui_fill_fmt(const UiFillParams p) {
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
                sum += lumaQ<F>(p.f, f, p.pitch, x, y, p.pq);
                n++;
            }
        if (n > 0) {
            (isC ? p.lc : p.la)[(size_t)cy * p.fw + cx] = __fmul_rn(i2f(rneDiv(4 * sum, n)), 1.0f / 16.0f);
            return;
        }
    }
}
cudaError_t launchUiFillFmt(const UiFillParams& p, cudaStream_t s) {
    const dim3 grid(divUp(p.ncx, 8), divUp(p.ncy, 8), 2);
    switch (p.f.format) {
        case kFmtRgb10: return launchPdl(k_ui_fill_fmt<kFmtRgb10>, grid, dim3(64), 0, s, p);
        case kFmtF16: return launchPdl(k_ui_fill_fmt<kFmtF16>, grid, dim3(64), 0, s, p);
        case kFmtNv12: return launchPdl(k_ui_fill_fmt<kFmtNv12>, grid, dim3(64), 0, s, p);
        case kFmtP010: return launchPdl(k_ui_fill_fmt<kFmtP010>, grid, dim3(64), 0, s, p);
        default: return cudaErrorInvalidValue;
    }
}

__global__ void __launch_bounds__(256) k_pq_table(float* tab, float kWhite) {
    const int i = blockIdx.x * 256 + threadIdx.x;   // the half's bits
    tab[i] = fmtPq255(h2f((uint32_t)i), kWhite);
}
cudaError_t launchPqTable(float* tab, float kWhite, cudaStream_t s) {
    k_pq_table<<<65536 / 256, 256, 0, s>>>(tab, kWhite);
    return cudaGetLastError();
}

cudaError_t launchSynthFmt(const SynthParams& p, cudaStream_t s) {
    const dim3 grid(divUp(p.W, kSyT), divUp(p.H, kSyTH));
    const size_t smem = fmtSynthSmem(p.f.format, p.fs);
    if (p.uiA || p.uiC) {   // CrosshairV2: the tap rejection compiled in
        switch (p.f.format) {
            case kFmtRgb10: return launchPdl(k_synth_fmt_ui<kFmtRgb10>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtF16: return launchPdl(k_synth_fmt_ui<kFmtF16>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtNv12: return launchPdl(k_synth_fmt_ui<kFmtNv12>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtP010: return launchPdl(k_synth_fmt_ui<kFmtP010>, grid, dim3(kSyThreads), smem, s, p);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (p.f.format) {
        case kFmtRgb10: return launchPdl(k_synth_fmt<kFmtRgb10>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtF16: return launchPdl(k_synth_fmt<kFmtF16>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtNv12: return launchPdl(k_synth_fmt<kFmtNv12>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtP010: return launchPdl(k_synth_fmt<kFmtP010>, grid, dim3(kSyThreads), smem, s, p);
        default: return cudaErrorInvalidValue;
    }
}

size_t synthFmtKernelSmem(int format, int fs) { return fmtSynthSmem(format, fs); }
template <int F>
static int fmtBatchOcc(size_t smem) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_synth_fmt_batch<F>, kSyThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ;
}
int synthFmtBatchCtasPerSm(int format, size_t smem) {
    switch (format) {
        case kFmtRgb10: return fmtBatchOcc<kFmtRgb10>(smem);
        case kFmtF16: return fmtBatchOcc<kFmtF16>(smem);
        case kFmtNv12: return fmtBatchOcc<kFmtNv12>(smem);
        case kFmtP010: return fmtBatchOcc<kFmtP010>(smem);
        default: return 0;
    }
}
cudaError_t launchSynthFmtBatch(const SynthBatchArgs& b, int format, int grid, size_t smem, cudaStream_t s) {
    switch (format) {
        case kFmtRgb10: return launchPdl(k_synth_fmt_batch<kFmtRgb10>, dim3(grid), dim3(kSyThreads), smem, s, b);
        case kFmtF16: return launchPdl(k_synth_fmt_batch<kFmtF16>, dim3(grid), dim3(kSyThreads), smem, s, b);
        case kFmtNv12: return launchPdl(k_synth_fmt_batch<kFmtNv12>, dim3(grid), dim3(kSyThreads), smem, s, b);
        case kFmtP010: return launchPdl(k_synth_fmt_batch<kFmtP010>, dim3(grid), dim3(kSyThreads), smem, s, b);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t launchFallbackFmtBatch(const FallbackParams* items, int nItems, cudaStream_t s) {
    return launchPdl(k_fallback_fmt_batch, dim3(smCount(), nItems), dim3(256), 0, s, items);
}

cudaError_t launchFallbackFmt(const FallbackParams& p, cudaStream_t s) {
    return launchPdl(k_fallback_fmt, dim3(smCount() * 4), dim3(256), 0, s, p);
}

cudaError_t launchSynthBlurFmt(const BlurParams& bp, int fix, cudaStream_t s) {
    const size_t smem = fmtSynthSmem(bp.base.f.format, bp.base.fs);
    const dim3 grid(divUp(bp.base.W, kSyT), divUp(bp.base.H, kSyTH));
    BlurParams p = bp;
    p.fix = fix;
    if (bp.base.uiA || bp.base.uiC) {   // CrosshairV2: the tap rejection compiled in
        switch (bp.base.f.format) {
            case kFmtRgb10: return launchPdl(k_synth_blur_fmt<kFmtRgb10, true>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtF16: return launchPdl(k_synth_blur_fmt<kFmtF16, true>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtNv12: return launchPdl(k_synth_blur_fmt<kFmtNv12, true>, grid, dim3(kSyThreads), smem, s, p);
            case kFmtP010: return launchPdl(k_synth_blur_fmt<kFmtP010, true>, grid, dim3(kSyThreads), smem, s, p);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (bp.base.f.format) {
        case kFmtRgb10: return launchPdl(k_synth_blur_fmt<kFmtRgb10>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtF16: return launchPdl(k_synth_blur_fmt<kFmtF16>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtNv12: return launchPdl(k_synth_blur_fmt<kFmtNv12>, grid, dim3(kSyThreads), smem, s, p);
        case kFmtP010: return launchPdl(k_synth_blur_fmt<kFmtP010>, grid, dim3(kSyThreads), smem, s, p);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace fgk
