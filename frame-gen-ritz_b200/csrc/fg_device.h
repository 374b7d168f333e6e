// fg_device.h -- device helpers shared by the kernels of the V1 path (fg_kernels.cu: 8-bit RGBA, fg_formats.cu: the
// other frame formats), the synthesis tile shape and its field stage, and the launch helper.
#pragma once
#include <cfloat>
#include <cstdint>

#include "fg_params.h"

namespace fgk {

// Programmatic dependent launch: every kernel is launched with programmatic stream serialisation, lets the next kernel
// of the stream be scheduled at once (its CTAs only occupy the slots this grid frees) and then waits for the previous
// grid to complete and its memory to be visible before touching anything an earlier kernel wrote. The launch latency
// of each small dependent pass overlaps the tail of the one before it.
__device__ __forceinline__ void pdlEnter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// the item of this CTA in a merged launch and the CTA's coordinates in the item's own grid
template <class P>
__device__ __forceinline__ int mergedItem(const Merged<P>& m, int& bx, int& by) {
    const int b = (int)blockIdx.x;
    int lo = 0, hi = m.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (m.first[mid] <= b) lo = mid; else hi = mid - 1;
    }
    const int l = b - m.first[lo], gx = m.gx[lo];
    bx = l % gx;
    by = l / gx;
    return lo;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// luma texel with clamp-to-edge (== cv2 BORDER_REPLICATE and the replicate pad_to_block, interp.py:68-70)
__device__ __forceinline__ float Lc(const float* __restrict__ L, int w, int h, int x, int y) {
    return __ldg(L + (size_t)clampi(y, 0, h - 1) * w + clampi(x, 0, w - 1));
}

// cv2.remap INTER_LINEAR / BORDER_REPLICATE of a float plane at (x, y): coordinates rounded half-even to 1/32 px,
// taps clamped one by one, ((p00 w00 + p01 w01) + p10 w10) + p11 w11 with w = (1 - fy)(1 - fx) ... in float.
__device__ __forceinline__ float remapF(const float* __restrict__ L, int w, int h, float x, float y) {
    const int X = __float2int_rn(__fmul_rn(x, 32.0f)), Y = __float2int_rn(__fmul_rn(y, 32.0f));
    const int ix = X >> 5, iy = Y >> 5;
    const float fx = (float)(X & 31) * (1.0f / 32.0f), fy = (float)(Y & 31) * (1.0f / 32.0f);
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    const int x0 = clampi(ix, 0, w - 1), x1 = clampi(ix + 1, 0, w - 1);
    const size_t r0 = (size_t)clampi(iy, 0, h - 1) * w, r1 = (size_t)clampi(iy + 1, 0, h - 1) * w;
    const float p00 = __ldg(L + r0 + x0), p01 = __ldg(L + r0 + x1), p10 = __ldg(L + r1 + x0), p11 = __ldg(L + r1 + x1);
    float r = __fmul_rn(p00, __fmul_rn(gy, gx));
    r = __fadd_rn(r, __fmul_rn(p01, __fmul_rn(gy, fx)));
    r = __fadd_rn(r, __fmul_rn(p10, __fmul_rn(fy, gx)));
    r = __fadd_rn(r, __fmul_rn(p11, __fmul_rn(fy, fx)));
    return r;
}

// the same on the 2-channel float field (fw x fh float2)
__device__ __forceinline__ float2 remapF2(const float2* __restrict__ F, int w, int h, float x, float y) {
    const int X = __float2int_rn(__fmul_rn(x, 32.0f)), Y = __float2int_rn(__fmul_rn(y, 32.0f));
    const int ix = X >> 5, iy = Y >> 5;
    const float fx = (float)(X & 31) * (1.0f / 32.0f), fy = (float)(Y & 31) * (1.0f / 32.0f);
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    const float w00 = __fmul_rn(gy, gx), w01 = __fmul_rn(gy, fx), w10 = __fmul_rn(fy, gx), w11 = __fmul_rn(fy, fx);
    const int x0 = clampi(ix, 0, w - 1), x1 = clampi(ix + 1, 0, w - 1);
    const size_t r0 = (size_t)clampi(iy, 0, h - 1) * w, r1 = (size_t)clampi(iy + 1, 0, h - 1) * w;
    const float2 p00 = __ldg(F + r0 + x0), p01 = __ldg(F + r0 + x1), p10 = __ldg(F + r1 + x0), p11 = __ldg(F + r1 + x1);
    float2 r;
    r.x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.x, w00), __fmul_rn(p01.x, w01)), __fmul_rn(p10.x, w10)), __fmul_rn(p11.x, w11));
    r.y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.y, w00), __fmul_rn(p01.y, w01)), __fmul_rn(p10.y, w10)), __fmul_rn(p11.y, w11));
    return r;
}

// cv2.cvtColor BGR2GRAY on 8-bit input as OpenCV 4.13 computes it (15-bit fixed point; checked on all 2^24 colours)
__device__ __forceinline__ int gray8(uint32_t px, int ri, int gi, int bi) {
    const int r = (px >> (8 * ri)) & 255, g = (px >> (8 * gi)) & 255, b = (px >> (8 * bi)) & 255;
    return (b * 3735 + g * 19235 + r * 9798 + 16384) >> 15;
}
// the same with the weights in 16-bit lanes for the two-way dot products (byte 0, byte 1) and (byte 2, byte 3) of a
// pixel: wlo = w(byte 0) | w(byte 1) << 16, whi = w(byte 2) (byte 3, alpha, weighs 0); exact integer arithmetic
__device__ __forceinline__ int gray8dp(uint32_t px, uint32_t wlo, uint32_t whi) {
    return (int)(__dp2a_hi(whi, px, __dp2a_lo(wlo, px, 16384u)) >> 15);
}

// Paired fp32 multiply / add (two IEEE operations per instruction). The compiler may fuse a paired multiply and add into
// one paired FMA whatever rounding is asked for, so these are used only where every product and sum is exact (dyadic
// operands with few significant bits): there a fused and an unfused evaluation give the same bits. Chains that round
// (the field at t, its upsampling, the warp positions) use the scalar __fmul_rn / __fadd_rn, which are never fused.
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }

// round-half-even(x * 32) for |x * 32| < 2^22 (cv2's saturate_cast<int>(x * INTER_TAB_SIZE)), as the float's bits
// CrosshairV2's warp-tap rejection (gpu/shaders/ui_reject.glsl): does the bilinear tap whose position rounded to
// 1/32 px is (X, Y) (in 1/32 px) read, with a non-zero weight, a pixel that the UI mask m (header + bytes, fg_params.h
// UiV2Params) marks? The tap reads lo = (X >> 5, Y >> 5) .. lo + (the fraction is not 0) per axis.
__device__ __forceinline__ bool uiHitMask(const uint32_t* __restrict__ m, int X, int Y) {
    const uint32_t wh = __ldg(m + 2);
    if (wh == 0u) return false;
    const uint32_t o = __ldg(m + 1);
    const int ox = (int)(o & 0xFFFFu), oy = (int)(o >> 16), w = (int)(wh & 0xFFFFu), h = (int)(wh >> 16);
    const int stride = (int)__ldg(m + 3);
    const int lx = X >> 5, ly = Y >> 5;
    const int x0 = max(lx - ox, 0), y0 = max(ly - oy, 0);
    const int x1 = min(lx + ((X & 31) != 0) - ox, w - 1), y1 = min(ly + ((Y & 31) != 0) - oy, h - 1);
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++)
            if ((__ldg(m + 4 + y * stride + (x >> 2)) >> (8 * (x & 3))) & 255u) return true;
    return false;
}

// is the frame pixel (x, y) a UI pixel of the mask (header + bytes)?
__device__ __forceinline__ bool uiPx(const uint32_t* __restrict__ m, int x, int y) {
    const uint32_t o = __ldg(m + 1), wh = __ldg(m + 2);
    x -= (int)(o & 0xFFFFu);
    y -= (int)(o >> 16);
    if (x < 0 || y < 0 || x >= (int)(wh & 0xFFFFu) || y >= (int)(wh >> 16)) return false;
    return ((__ldg(m + kUiMaskHeader + y * (int)__ldg(m + 3) + (x >> 2)) >> (8 * (x & 3))) & 255u) != 0u;
}

// the same for a YUV sample (gpu/shaders/ui_reject.glsl uiFootprint, FG_YUV): the 2x2 texels of the half-resolution
// chroma plane around it, c = X - 16 in 1/64 chroma texels, i = c >> 6, the second texel only if the fraction is not
// 0: the pixels 2 i .. 2 (i + n) + 1 per axis, which contain the luma taps too
__device__ __forceinline__ bool uiHitMaskYuv(const uint32_t* __restrict__ m, int X, int Y) {
    const uint32_t wh = __ldg(m + 2);
    if (wh == 0u) return false;
    const uint32_t o = __ldg(m + 1);
    const int ox = (int)(o & 0xFFFFu), oy = (int)(o >> 16), w = (int)(wh & 0xFFFFu), h = (int)(wh >> 16);
    const int stride = (int)__ldg(m + 3);
    const int cx = X - 16, cy = Y - 16, ix = cx >> 6, iy = cy >> 6;
    const int x0 = max(2 * ix - ox, 0), y0 = max(2 * iy - oy, 0);
    const int x1 = min(2 * (ix + ((cx & 63) != 0)) + 1 - ox, w - 1), y1 = min(2 * (iy + ((cy & 63) != 0)) + 1 - oy, h - 1);
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++)
            if ((__ldg(m + 4 + y * stride + (x >> 2)) >> (8 * (x & 3))) & 255u) return true;
    return false;
}

__device__ __forceinline__ float2 rne32bits(float2 v) {
    return __ffma2_rn(v, make_float2(32.0f, 32.0f), make_float2(12582912.0f, 12582912.0f));
}
__device__ __forceinline__ int rne32(float x) { return __float_as_int(__fmaf_rn(x, 32.0f, 12582912.0f)) - 0x4B400000; }
// exact float of 0 <= i < 2^23
__device__ __forceinline__ float i2f(int i) { return __int_as_float(0x4B000000 | i) - 8388608.0f; }
// floor of 0 <= v < 2^23
__device__ __forceinline__ int floorPos(float v) { return __float_as_int(__fadd_rz(v, 8388608.0f)) - 0x4B000000; }

__device__ __forceinline__ float warpSum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ============================================================================================== luma tower
constexpr int kTowerFloats = 1024 + 256 + 64 + 16 + 4 + 1;   // a 32x32 level-0 tile and its 16x16 .. 1x1 levels above

// round half-even to a multiple of 2^-10 (the grid of the other formats' coarse pyramid levels)
__device__ __forceinline__ float round10(float v) { return __fmul_rn(rintf(__fmul_rn(v, 1024.0f)), 1.0f / 1024.0f); }

// interp.pyramid :73-77 above one 32x32 level-0 tile held in sl[.][0..1023] (tx0, ty0: the tile's origin): levels
// 1 .. p.nlev-1 of the tile's tower, each pixel the mean of the valid 2x2 pixels below it (sum * 1/4 when full,
// sum / count at the odd edges), written to p.la / p.lc and kept in sl for the next level. ROUND: rounded to 2^-10.
template <bool ROUND>
__device__ __forceinline__ void lumaTower(const LumaPyrParams& p, float (*sl)[kTowerFloats], int tx0, int ty0) {
    int off = 0, side = 32;
    for (int l = 1; l < p.nlev; l++) {
        const int noff = off + side * side, ns = side >> 1;
        const int X0 = tx0 >> l, Y0 = ty0 >> l;
        const int pw = p.lw[l - 1], ph = p.lh[l - 1];
        for (int i = threadIdx.x; i < ns * ns; i += 256) {
            const int lx = i % ns, ly = i / ns, X = X0 + lx, Y = Y0 + ly;
            float va = 0.0f, vc = 0.0f;
            if (X < p.lw[l] && Y < p.lh[l]) {
                float sa = 0.0f, sc = 0.0f;
                int n = 0;
                for (int j = 0; j < 2; j++)
                    for (int k = 0; k < 2; k++)
                        if (2 * X + k < pw && 2 * Y + j < ph) {
                            const int ci = off + (2 * ly + j) * side + 2 * lx + k;
                            sa = __fadd_rn(sa, sl[0][ci]);
                            sc = __fadd_rn(sc, sl[1][ci]);
                            n++;
                        }
                va = n == 4 ? __fmul_rn(sa, 0.25f) : __fdiv_rn(sa, (float)n);
                vc = n == 4 ? __fmul_rn(sc, 0.25f) : __fdiv_rn(sc, (float)n);
                if (ROUND) { va = round10(va); vc = round10(vc); }
                p.la[l][(size_t)Y * p.lw[l] + X] = va;
                p.lc[l][(size_t)Y * p.lw[l] + X] = vc;
            }
            sl[0][noff + i] = va;
            sl[1][noff + i] = vc;
        }
        __syncthreads();
        off = noff;
        side = ns;
    }
}

// ============================================================================================== synthesis tile
// 64 x 64 mismatch region -> 58 x 58 output tile: the square tile recomputes the least halo (1.22 region pixels per
// output pixel, against 1.29 for 128 x 32) within the shared memory of 3 CTAs per SM
constexpr int kSyE = 64, kSyEH = 64, kSyAp = 3;
constexpr int kSyT = kSyE - 2 * kSyAp, kSyTH = kSyEH - 2 * kSyAp;
constexpr int kSyThreads = 512, kSyK = kSyEH / (kSyThreads / kSyE);   // region rows per thread (512 = 64 columns x 8)
constexpr size_t kSyWarpBytes = (size_t)2 * kSyTH * kSyE * 4;   // k_synth: both warps of the output rows, after the row sums
// the output row (tile coordinates) of a thread's k-th output pixel: thread rows ey0 = 0..7 take kSyK consecutive rows
// each (the last only kSyTH - 7 kSyK of them), so the vertical 7-sums run as a sliding window
__device__ __forceinline__ int syOutRow(int ey0, int k) { return ey0 * kSyK + k; }
// row strides of the mismatch plane e (bytes) and of its horizontal 7-sums (uint16): one word of padding per row, so
// that the lanes of a warp can walk 32 different rows of one column group without bank conflicts
constexpr int kSyES = kSyE + 4, kSyHS = kSyE + 2;

// cv2.remap INTER_LINEAR / BORDER_REPLICATE of the 2-channel float field at (x, y): quantisation and weights paired
// (exact), the taps' weighted sum as cv2 rounds it, ((p00 w00 + p01 w01) + p10 w10) + p11 w11 per channel
__device__ __forceinline__ float2 remapF2m(const float2* __restrict__ F, int w, int h, float x, float y) {
    const float2 bits = rne32bits(make_float2(x, y));
    const int X = __float_as_int(bits.x) - 0x4B400000, Y = __float_as_int(bits.y) - 0x4B400000;
    const int ix = X >> 5, iy = Y >> 5;
    const float2 f = pmul(make_float2(i2f(X & 31), i2f(Y & 31)), make_float2(1.0f / 32.0f, 1.0f / 32.0f));
    const float2 g = padd(make_float2(1.0f, 1.0f), make_float2(-f.x, -f.y));
    const float2 wA = pmul(make_float2(g.y, g.y), make_float2(g.x, f.x));   // (w00, w01)
    const float2 wB = pmul(make_float2(f.y, f.y), make_float2(g.x, f.x));   // (w10, w11)
    const int x0 = clampi(ix, 0, w - 1), x1 = clampi(ix + 1, 0, w - 1);
    const size_t r0 = (size_t)clampi(iy, 0, h - 1) * w, r1 = (size_t)clampi(iy + 1, 0, h - 1) * w;
    const float2 p00 = __ldg(F + r0 + x0), p01 = __ldg(F + r0 + x1), p10 = __ldg(F + r1 + x0), p11 = __ldg(F + r1 + x1);
    float2 r;
    r.x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.x, wA.x), __fmul_rn(p01.x, wA.y)), __fmul_rn(p10.x, wB.x)), __fmul_rn(p11.x, wB.y));
    r.y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.y, wA.x), __fmul_rn(p01.y, wA.y)), __fmul_rn(p10.y, wB.x)), __fmul_rn(p11.y, wB.y));
    return r;
}

struct SyCoef {   // one region column (or row): upsampling taps (relative to the tile's field region) and weights
    int i0, i1;
    float a0, a1;   // rows: already x fs (scaling by a power of 2 commutes with the rounding)
    float pos;      // the clamped pixel coordinate
    int pi;
};

__device__ __forceinline__ SyCoef syCoef(int e, int origin, int n, int un, int fn, int g0, float invfs, float wscale, bool xaxis) {
    SyCoef c;
    const int p = clampi(origin - kSyAp + e, 0, n - 1);
    const int d = min(p, un - 1);   // crop [:H, :W] / edge pad of the upsampled field
    float f = __fsub_rn(__fmul_rn((float)d + 0.5f, invfs), 0.5f);   // exact for fs = 1, 2, 4
    int s = (int)floorf(f);
    f = __fsub_rn(f, (float)s);
    if (xaxis) {   // cv2 resize: x weights forced to (1, 0) beyond the borders; y rows clamped, weights kept
        if (s < 0) { s = 0; f = 0.0f; }
        if (s >= fn - 1) { s = fn - 1; f = 0.0f; }
    }
    c.i0 = clampi(s, 0, fn - 1) - g0;
    c.i1 = clampi(s + 1, 0, fn - 1) - g0;
    c.a0 = __fmul_rn(1.0f - f, wscale);
    c.a1 = __fmul_rn(f, wscale);
    c.pos = (float)p;
    c.pi = p;
    return c;
}

// Stages 0-1b of a synthesis tile, shared by the kernels of every format: the tile's field region, the row
// coefficients (rowc) and this thread's column coefficients (returned); the field at t on the region (interp.field_at:
// g <- pf(q - s g), twice, from g = pf(q)); the horizontal stage of its upsampling (cv2 resize: h = S0 a0 + S1 a1 per
// row) into hrow. Carves the dynamic shared memory sm into the field region, hrow, the mismatch plane e and the row
// sums hsum. Ends with a barrier.
__device__ __forceinline__ SyCoef syFieldStage(const SynthParams& p, int X0, int Y0, int tid, int ex, int ey0, SyCoef* rowc,
                                               int* gReg, unsigned char* sm, float2*& hrow, uint8_t*& e,
                                               unsigned short*& hsum) {
    const int fs = p.fs, uw = p.fw * fs, uh = p.fh * fs;
    const float invfs = 1.0f / (float)fs, fsf = (float)fs;
    if (tid == 0) {
        const SyCoef lo = syCoef(0, X0, p.W, uw, p.fw, 0, invfs, 1.0f, true);
        const SyCoef hi = syCoef(kSyE - 1, X0, p.W, uw, p.fw, 0, invfs, 1.0f, true);
        const SyCoef rlo = syCoef(0, Y0, p.H, uh, p.fh, 0, invfs, 1.0f, false);
        const SyCoef rhi = syCoef(kSyEH - 1, Y0, p.H, uh, p.fh, 0, invfs, 1.0f, false);
        gReg[0] = lo.i0; gReg[1] = hi.i1 - lo.i0 + 1; gReg[2] = rlo.i0; gReg[3] = rhi.i1 - rlo.i0 + 1;
    }
    __syncthreads();
    const int gx0 = gReg[0], GW = gReg[1], gy0 = gReg[2], GH = gReg[3];
    if (tid < kSyEH) rowc[tid] = syCoef(tid, Y0, p.H, uh, p.fh, gy0, invfs, fsf, false);
    const SyCoef cx = syCoef(ex, X0, p.W, uw, p.fw, gx0, invfs, 1.0f, true);
    float2* g = reinterpret_cast<float2*>(sm);             // GH x GW
    hrow = g + GW * GH;                                    // GH x kSyE
    e = reinterpret_cast<uint8_t*>(hrow + GH * kSyE);      // kSyEH rows of kSyES bytes
    hsum = reinterpret_cast<unsigned short*>(e + kSyEH * kSyES);   // kSyEH rows of kSyHS (columns < kSyT used)
    // the region's GW x GH samples spread over all threads (GW is about half the CTA's width at flowScale 2): row
    // r = floor((i + 0.5) / GW), exact in float for these sizes (the quotient stays >= 0.5 / GW from an integer)
    const float invGW = 1.0f / (float)GW;
    for (int i = tid; i < GW * GH; i += kSyThreads) {
        const int r = (int)__fmul_rz(__int2float_rn(i) + 0.5f, invGW), c = i - r * GW;
        const int qx = gx0 + c, qy = gy0 + r;
        float2 v = __ldg(p.pf + (size_t)qy * p.fw + qx);
        if (p.lookup) {
            const float fx = (float)qx, fy = (float)qy;
#pragma unroll
            for (int it = 0; it < 2; it++)
                v = remapF2m(p.pf, p.fw, p.fh, __fsub_rn(fx, __fmul_rn(p.s, v.x)), __fsub_rn(fy, __fmul_rn(p.s, v.y)));
        }
        g[r * GW + c] = v;
    }
    __syncthreads();
    for (int r = ey0; r < GH; r += kSyThreads / kSyE) {
        const float2 s0 = g[r * GW + cx.i0], s1 = g[r * GW + cx.i1];
        hrow[r * kSyE + ex] = make_float2(__fadd_rn(__fmul_rn(s0.x, cx.a0), __fmul_rn(s1.x, cx.a1)),
                                          __fadd_rn(__fmul_rn(s0.y, cx.a0), __fmul_rn(s1.y, cx.a1)));
    }
    __syncthreads();
    return cx;
}

// Stage 3 of a synthesis tile: the horizontal 7-sums of the mismatch plane, one region row and 8 output columns per
// thread (a running window); the lanes of a warp take the 32 rows of one column group (conflict-free strides)
__device__ __forceinline__ void syRowSums(const uint8_t* e, unsigned short* hsum, int tid) {
    const int r = tid & (kSyEH - 1), c0 = (tid / kSyEH) * 8;
    const uint8_t* q = e + r * kSyES + c0;
    unsigned short* o = hsum + r * kSyHS + c0;
    unsigned int sum = q[0] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6];
    o[0] = (unsigned short)sum;
#pragma unroll
    for (int c = 1; c < 8; c++) {
        if (c0 + c + 6 < kSyE) sum += q[c + 6] - q[c - 1];
        o[c] = (unsigned short)sum;
    }
}

// the half-vector of region row ey in this thread's column (vertical stage of the upsampling, x fs folded in)
__device__ __forceinline__ float2 syHalfVec(const SyCoef& cy, const float2* hrow, int ex) {
    const float2 h0 = hrow[cy.i0 * kSyE + ex], h1 = hrow[cy.i1 * kSyE + ex];
    return make_float2(__fadd_rn(__fmul_rn(h0.x, cy.a0), __fmul_rn(h1.x, cy.a1)),
                       __fadd_rn(__fmul_rn(h0.y, cy.a0), __fmul_rn(h1.y, cy.a1)));
}

inline unsigned int divUp(int a, int b) { return (unsigned int)((a + b - 1) / b); }

template <typename... KArgs, typename... Args>
cudaError_t launchPdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace fgk
