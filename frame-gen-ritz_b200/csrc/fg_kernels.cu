// CUDA kernels of the MotionVersion::V1 interpolation path (sm_100a).
//
// Each kernel reproduces the arithmetic of frame-gen-ritz's proto/interp.py as executed by numpy and OpenCV 4.13
// (cvtColor, resize, remap, blur, medianBlur), bit for bit:
//   - estimate values are dyadic rationals (luma multiples of 4^-(l+1) at flowScale 2, bilinear weights multiples of
//     1/32 per axis), so every SAD, tap and box sum below is exact in float32 / int32 whatever the summation order;
//   - where values are not dyadic (the field at time t, its upsampling, the blend), the kernels follow OpenCV's and
//     numpy's operation order with explicit round-to-nearest intrinsics (no contraction);
//   - reductions whose rounding depends on order (the scene-cut mean) follow numpy's pairwise tree.
// The whole library is compiled with -fmad=false as a second guard against contraction.
#include <algorithm>
#include <atomic>
#include <cooperative_groups.h>

#include "fg_device.h"

namespace fgk {

// ============================================================================================== luma + pyramid
// interp.flow :149-152 + interp.pyramid :73-77. One CTA = a 32x32 tile of level 0 (32 fs x 32 fs frame pixels) and
// the aligned 16x16 .. 1x1 tiles of levels 1..5 above it: a level-(l+1) pixel only averages the 2x2 level-l pixels
// below it, so the whole tower stays inside the tile. Mean of the valid pixels: sum * 1/n^2 when full, sum / count
// at the frame's odd edges (cv2's INTER_AREA fast path).
__device__ __forceinline__ void lumaPyrCta(const LumaPyrParams& p, int bx, int by) {
    __shared__ float sl[2][kTowerFloats];
    const int tx0 = bx * 32, ty0 = by * 32;
    const int fw = p.lw[0], fh = p.lh[0], fs = p.fs;
    if (p.vec16 && tx0 + 32 <= fw && ty0 + 32 <= fh) {
        // flowScale 2, 16-byte aligned rows, a full tile: thread = 4 frame pixels (one uint4) x 2 rows = 2 level-0
        // pixels; a warp reads 2 x 256 contiguous bytes per frame and row pair
        const int cg = threadIdx.x & 15, rp = threadIdx.x >> 4;
        // luma weights by byte position for the dot-product form (G is byte 1 in both orders)
        const uint32_t wlo = (p.ri == 0 ? 9798u : 3735u) | (19235u << 16), whi = p.ri == 0 ? 3735u : 9798u;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int ly = rp + 16 * j, y = ty0 + ly;
            const size_t o0 = (size_t)(2 * y) * p.pitch + (size_t)(2 * tx0 + 4 * cg) * 4;
            const uint4 a0 = __ldg(reinterpret_cast<const uint4*>(p.a + o0)), a1 = __ldg(reinterpret_cast<const uint4*>(p.a + o0 + p.pitch));
            const uint4 c0 = __ldg(reinterpret_cast<const uint4*>(p.c + o0)), c1 = __ldg(reinterpret_cast<const uint4*>(p.c + o0 + p.pitch));
            const int sa0 = gray8dp(a0.x, wlo, whi) + gray8dp(a0.y, wlo, whi) + gray8dp(a1.x, wlo, whi) + gray8dp(a1.y, wlo, whi);
            const int sa1 = gray8dp(a0.z, wlo, whi) + gray8dp(a0.w, wlo, whi) + gray8dp(a1.z, wlo, whi) + gray8dp(a1.w, wlo, whi);
            const int sc0 = gray8dp(c0.x, wlo, whi) + gray8dp(c0.y, wlo, whi) + gray8dp(c1.x, wlo, whi) + gray8dp(c1.y, wlo, whi);
            const int sc1 = gray8dp(c0.z, wlo, whi) + gray8dp(c0.w, wlo, whi) + gray8dp(c1.z, wlo, whi) + gray8dp(c1.w, wlo, whi);
            // sum * 0.25 (integer sums of 4 lumas: exact)
            const float2 va = make_float2(i2f(sa0) * 0.25f, i2f(sa1) * 0.25f), vc = make_float2(i2f(sc0) * 0.25f, i2f(sc1) * 0.25f);
            *reinterpret_cast<float2*>(p.la[0] + (size_t)y * fw + tx0 + 2 * cg) = va;
            *reinterpret_cast<float2*>(p.lc[0] + (size_t)y * fw + tx0 + 2 * cg) = vc;
            sl[0][ly * 32 + 2 * cg] = va.x; sl[0][ly * 32 + 2 * cg + 1] = va.y;
            sl[1][ly * 32 + 2 * cg] = vc.x; sl[1][ly * 32 + 2 * cg + 1] = vc.y;
        }
    } else {
        for (int i = threadIdx.x; i < 1024; i += 256) {
            const int x = tx0 + (i & 31), y = ty0 + (i >> 5);
            float va = 0.0f, vc = 0.0f;
            if (x < fw && y < fh) {
                int sa = 0, sc = 0, n = 0;
                for (int j = 0; j < fs; j++) {
                    const int yy = y * fs + j;
                    if (yy >= p.H) break;
                    const uint32_t* ra = reinterpret_cast<const uint32_t*>(p.a + (size_t)yy * p.pitch);
                    const uint32_t* rc = reinterpret_cast<const uint32_t*>(p.c + (size_t)yy * p.pitch);
                    for (int k = 0; k < fs; k++) {
                        const int xx = x * fs + k;
                        if (xx >= p.W) break;
                        sa += gray8(__ldg(ra + xx), p.ri, p.gi, p.bi);
                        sc += gray8(__ldg(rc + xx), p.ri, p.gi, p.bi);
                        n++;
                    }
                }
                if (fs == 1) {
                    va = (float)sa;
                    vc = (float)sc;
                } else if (n == fs * fs) {
                    const float inv = 1.0f / (float)(fs * fs);
                    va = __fmul_rn((float)sa, inv);
                    vc = __fmul_rn((float)sc, inv);
                } else {
                    va = __fdiv_rn((float)sa, (float)n);
                    vc = __fdiv_rn((float)sc, (float)n);
                }
                p.la[0][(size_t)y * fw + x] = va;
                p.lc[0][(size_t)y * fw + x] = vc;
            }
            sl[0][i] = va;
            sl[1][i] = vc;
        }
    }
    __syncthreads();
    lumaTower<false>(p, sl, tx0, ty0);
}
__global__ void __launch_bounds__(256) k_luma_pyr(const LumaPyrParams p) {
    pdlEnter();
    lumaPyrCta(p, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(256) k_luma_pyr_m(const __grid_constant__ Merged<LumaPyrParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    lumaPyrCta(m.item[i], bx, by);
}

// a pyramid level beyond the luma kernel's tower (interp.py:76); round10: the other formats' 2^-10 grid
__global__ void __launch_bounds__(256) k_down(const DownParams p) {
    pdlEnter();
    const int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= p.dw || y >= p.dh) return;
    float sa = 0.0f, sc = 0.0f;
    int n = 0;
    for (int j = 0; j < 2; j++)
        for (int k = 0; k < 2; k++)
            if (2 * x + k < p.sw && 2 * y + j < p.sh) {
                const size_t i = (size_t)(2 * y + j) * p.sw + 2 * x + k;
                sa = __fadd_rn(sa, p.sa[i]);
                sc = __fadd_rn(sc, p.sc[i]);
                n++;
            }
    float va = n == 4 ? __fmul_rn(sa, 0.25f) : __fdiv_rn(sa, (float)n);
    float vc = n == 4 ? __fmul_rn(sc, 0.25f) : __fdiv_rn(sc, (float)n);
    if (p.round10) { va = round10(va); vc = round10(vc); }
    p.da[(size_t)y * p.dw + x] = va;
    p.dc[(size_t)y * p.dw + x] = vc;
}

// ============================================================================================== seed + search
// interp.seed_from :131-144 and interp.search :116-124 at integer steps, one warp per 8x8 block.
// Seed: own parent, the 3 nearest other parents, zero, the global median (all 2x the parent level's vectors),
// scored by block SAD + (0 for own, lambda otherwise); the first minimum wins.
// Search: every integer offset within +-R of the seed; the (8+2R)^2 windows of a and c (bilateral: a at q - v, c at
// q + v) are staged in shared memory; lane i scores candidates i, i+32, ...; cost = SAD + lambda |d|_1; the warp
// keeps the lowest (cost, raster index) pair, i.e. the first minimum in interp's (dy, dx) order.
template <bool kLat>
__device__ __forceinline__ void searchSeed(const SearchParams& p, int bx, int by, int lane, int& sx, int& sy);

__device__ __forceinline__ void searchCta(const SearchParams& p, int cta) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = cta * 4 + warp;
    if (b >= p.bw * p.bh) return;
    const int R = p.R, T = 8 + 2 * R, D = 2 * R + 1;
    float* sA = smem + warp * 2 * T * T;
    float* sC = sA + T * T;
    const int bx = b % p.bw, by = b / p.bw, b0x = bx * kBlock, b0y = by * kBlock;
    int sx, sy;
    searchSeed<false>(p, bx, by, lane, sx, sy);
    for (int i = lane; i < T * T; i += 32) {
        const int x = i % T, y = i / T;
        sA[i] = Lc(p.la, p.w, p.h, b0x - sx - R + x, b0y - sy - R + y);
        sC[i] = Lc(p.lc, p.w, p.h, b0x + sx - R + x, b0y + sy - R + y);
    }
    __syncwarp();
    float bc = FLT_MAX, bsad = 0.0f;
    int bci = 0x7fffffff;
    for (int ci = lane; ci < D * D; ci += 32) {
        const int dx = ci % D - R, dy = ci / D - R;
        const float* pa = sA + (R - dy) * T + (R - dx);
        const float* pc = sC + (R + dy) * T + (R + dx);
        float sum = 0.0f;
#pragma unroll
        for (int y = 0; y < 8; y++)
#pragma unroll
            for (int x = 0; x < 8; x++) sum += fabsf(pa[y * T + x] - pc[y * T + x]);
        const float sad = __fmul_rn(sum, 1.0f / 64.0f);
        const float cost = __fadd_rn(sad, p.pen[abs(dx) + abs(dy)]);
        if (cost < bc) { bc = cost; bci = ci; bsad = sad; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, o), os = __shfl_xor_sync(0xffffffffu, bsad, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bci, o);
        if (oc < bc || (oc == bc && oi < bci)) { bc = oc; bci = oi; bsad = os; }
    }
    if (lane == 0) {
        p.out[b] = make_float2((float)(sx + bci % D - R), (float)(sy + bci / D - R));
        if (p.sadOut) p.sadOut[b] = bsad;
    }
}
__global__ void __launch_bounds__(128) k_search(const SearchParams p) {
    pdlEnter();
    searchCta(p, blockIdx.x);
}
__global__ void __launch_bounds__(128) k_search_m(const __grid_constant__ Merged<SearchParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    searchCta(m.item[i], bx);
}

// The seed of a block (interp.seed_from :131-144 for one fine block), shared by both search kernels. A candidate equal
// to an earlier one is skipped: its cost would equal that one's (or exceed it by lambda), so under the first-minimum
// rule it could never be picked.
template <bool kLat>
__device__ __forceinline__ void searchSeed(const SearchParams& p, int bx, int by, int lane, int& sx, int& sy) {
    sx = 0;
    sy = 0;
    if (p.top) return;
    const int b0x = bx * kBlock, b0y = by * kBlock;
    int cxs[6], cys[6];
    bool pen0 = false;   // the first candidate pays lambda too
    if (p.cnn) {
        // seed-net level: its two candidates (rounded half-even, clamped to +-256), then zero; the first is free of
        // the penalty only when the net is confident (logit >= 0). Slots 3..5 repeat zero and are skipped as such.
        const float* o = p.cnn + (size_t)(by * p.bw + bx) * kSeedNetOut;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            cxs[k] = k < 2 ? __float2int_rn(fminf(fmaxf(o[2 * k], -256.0f), 256.0f)) : 0;
            cys[k] = k < 2 ? __float2int_rn(fminf(fmaxf(o[2 * k + 1], -256.0f), 256.0f)) : 0;
        }
        pen0 = !(o[4] >= 0.0f);
    } else {
        const int px = min(bx >> 1, p.pw - 1), py = min(by >> 1, p.ph - 1);
        const int oy = (by & 1) ? 1 : -1, ox = (bx & 1) ? 1 : -1;
#pragma unroll
        for (int k = 0; k < 6; k++) {   // own, (0, oy), (ox, 0), (ox, oy) parents x 2; zero; the global median
            int cx = 0, cy = 0;
            if (k < 4) {
                const int dx = (k & 2) ? ox : 0, dy = (k & 1) ? oy : 0;
                const float2 v = p.parent[clampi(py + dy, 0, p.ph - 1) * p.pw + clampi(px + dx, 0, p.pw - 1)];
                cx = 2 * __float2int_rn(v.x);
                cy = 2 * __float2int_rn(v.y);
            } else if (k == 5) {
                cx = __float2int_rn(p.med[0]);
                cy = __float2int_rn(p.med[1]);
            }
            cxs[k] = cx;
            cys[k] = cy;
        }
    }
    const int qx = b0x + (lane & 7), qy0 = b0y + (lane >> 3), qy1 = qy0 + 4;
    if (!kLat) {   // large levels (throughput bound): candidates scored one after another, duplicates skipped
        float best = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            bool dup = false;
#pragma unroll
            for (int j = 0; j < k; j++) dup |= cxs[j] == cxs[k] && cys[j] == cys[k];
            if (dup) continue;   // warp-uniform
            const int cx = cxs[k], cy = cys[k];
            float s;
            if (b0x - abs(cx) >= 0 && b0x + 7 + abs(cx) < p.w && b0y - abs(cy) >= 0 && b0y + 7 + abs(cy) < p.h) {
                const float* ra = p.la + (size_t)(qy0 - cy) * p.w + (qx - cx);
                const float* rc = p.lc + (size_t)(qy0 + cy) * p.w + (qx + cx);
                s = fabsf(__ldg(ra) - __ldg(rc)) + fabsf(__ldg(ra + 4 * p.w) - __ldg(rc + 4 * p.w));
            } else {
                s = fabsf(Lc(p.la, p.w, p.h, qx - cx, qy0 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy0 + cy));
                s += fabsf(Lc(p.la, p.w, p.h, qx - cx, qy1 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy1 + cy));
            }
            s = warpSum(s);   // exact: at most 24 significant bits
            float cost = __fmul_rn(s, 1.0f / 64.0f);
            if (k > 0 || pen0) cost = __fadd_rn(cost, p.lambda);
            if (k == 0 || cost < best) { best = cost; sx = cx; sy = cy; }
        }
        return;
    }
    // small levels (latency bound): every candidate's two pixel pairs per lane are loaded before any is reduced
    // (clamped addressing = the replicate border), so the six scores cost one memory round trip rather than six
    bool dup[6];
    float sk[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        dup[k] = false;
#pragma unroll
        for (int j = 0; j < k; j++) dup[k] |= cxs[j] == cxs[k] && cys[j] == cys[k];
        const int cx = cxs[k], cy = cys[k];
        sk[k] = fabsf(Lc(p.la, p.w, p.h, qx - cx, qy0 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy0 + cy)) +
                fabsf(Lc(p.la, p.w, p.h, qx - cx, qy1 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy1 + cy));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)   // six warp sums side by side (exact: at most 24 significant bits)
#pragma unroll
        for (int k = 0; k < 6; k++) sk[k] += __shfl_xor_sync(0xffffffffu, sk[k], o);
    float best = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (dup[k]) continue;   // warp-uniform
        float cost = __fmul_rn(sk[k], 1.0f / 64.0f);
        if (k > 0 || pen0) cost = __fadd_rn(cost, p.lambda);
        if (k == 0 || cost < best) { best = cost; sx = cxs[k]; sy = cys[k]; }
    }
}

// levels of at most this many blocks are latency bound (a few CTAs per SM): their seeds load every candidate at once
constexpr int kSearchLatBlocks = 2048;

// interp.search at integer steps, radius R known at compile time (1..6), one warp per 8x8 block. The (8+2R)^2 windows
// of a and c are staged in shared memory. Lane = (dy, block row y): it holds a's row y - dy and c's row y + dy in
// registers and scores every dx from them; the 8 rows of a dy are summed by shuffles (all sums exact).
template <int R, bool kLat>
__device__ __forceinline__ void searchRCta(const SearchParams& p, int cta) {
    constexpr int T = 8 + 2 * R, D = 2 * R + 1, NI = 8 * D, ROUNDS = (NI + 31) / 32;
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = cta * 4 + warp;
    if (b >= p.bw * p.bh) return;
    float* sA = smem + warp * (2 * T * T + D * D);
    float* sC = sA + T * T;
    float* sad = sC + T * T;   // D x D window SADs (sums over the 64 pixels)
    const int bx = b % p.bw, by = b / p.bw, b0x = bx * kBlock, b0y = by * kBlock;
    int sx, sy;
    searchSeed<kLat>(p, bx, by, lane, sx, sy);
    const int ax0 = b0x - sx - R, ay0 = b0y - sy - R, cx0 = b0x + sx - R, cy0 = b0y + sy - R;
    if (ax0 >= 0 && ay0 >= 0 && ax0 + T <= p.w && ay0 + T <= p.h && cx0 >= 0 && cy0 >= 0 && cx0 + T <= p.w && cy0 + T <= p.h) {
        for (int i = lane; i < T * T; i += 32) {
            const int x = i % T, y = i / T;
            sA[i] = __ldg(p.la + (size_t)(ay0 + y) * p.w + ax0 + x);
            sC[i] = __ldg(p.lc + (size_t)(cy0 + y) * p.w + cx0 + x);
        }
    } else {
        for (int i = lane; i < T * T; i += 32) {
            const int x = i % T, y = i / T;
            sA[i] = Lc(p.la, p.w, p.h, ax0 + x, ay0 + y);
            sC[i] = Lc(p.lc, p.w, p.h, cx0 + x, cy0 + y);
        }
    }
    __syncwarp();
#pragma unroll
    for (int rd = 0; rd < ROUNDS; rd++) {
        const int it = rd * 32 + lane;
        const bool act = it < NI;
        const int dyi = act ? (it >> 3) : 0, y = it & 7, dy = dyi - R;
        const float* ra = sA + (y - dy + R) * T;
        const float* rc = sC + (y + dy + R) * T;
        float a[T], c[T];
#pragma unroll
        for (int i = 0; i < T; i++) { a[i] = ra[i]; c[i] = rc[i]; }
#pragma unroll
        for (int dxi = 0; dxi < D; dxi++) {
            const int dx = dxi - R;
            float sum = 0.0f;
#pragma unroll
            for (int x = 0; x < 8; x++) sum += fabsf(a[x - dx + R] - c[x + dx + R]);
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 2);
            sum += __shfl_xor_sync(0xffffffffu, sum, 4);
            if (act && y == 0) sad[dyi * D + dxi] = sum;
        }
    }
    __syncwarp();
    float bc = FLT_MAX, bsad = 0.0f;
    int bci = 0x7fffffff;
    for (int ci = lane; ci < D * D; ci += 32) {
        const int dx = ci % D - R, dy = ci / D - R;
        const float sd = __fmul_rn(sad[ci], 1.0f / 64.0f);
        const float cost = __fadd_rn(sd, p.pen[abs(dx) + abs(dy)]);
        if (cost < bc) { bc = cost; bci = ci; bsad = sd; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, o), os = __shfl_xor_sync(0xffffffffu, bsad, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bci, o);
        if (oc < bc || (oc == bc && oi < bci)) { bc = oc; bci = oi; bsad = os; }
    }
    if (lane == 0) {
        p.out[b] = make_float2((float)(sx + bci % D - R), (float)(sy + bci / D - R));
        if (p.sadOut) p.sadOut[b] = bsad;
    }
}
template <int R, bool kLat>
__global__ void __launch_bounds__(128) k_search_r(const SearchParams p) {
    pdlEnter();
    searchRCta<R, kLat>(p, blockIdx.x);
}
template <int R, bool kLat>
__global__ void __launch_bounds__(128) k_search_r_m(const __grid_constant__ Merged<SearchParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    searchRCta<R, kLat>(m.item[i], bx);
}

// ============================================================================================== median3 + global median
__device__ __forceinline__ void cswap(float& a, float& b) {
    const float lo = fminf(a, b), hi = fmaxf(a, b);
    a = lo;
    b = hi;
}
// exact median of 9 (a 19-exchange selection network)
__device__ __forceinline__ float med9(float v[9]) {
    cswap(v[1], v[2]); cswap(v[4], v[5]); cswap(v[7], v[8]);
    cswap(v[0], v[1]); cswap(v[3], v[4]); cswap(v[6], v[7]);
    cswap(v[1], v[2]); cswap(v[4], v[5]); cswap(v[7], v[8]);
    cswap(v[0], v[3]); cswap(v[5], v[8]); cswap(v[4], v[7]);
    cswap(v[3], v[6]); cswap(v[1], v[4]); cswap(v[2], v[5]);
    cswap(v[4], v[7]); cswap(v[4], v[2]); cswap(v[6], v[4]);
    cswap(v[4], v[2]);
    return v[4];
}

// interp.median3 :127-128 (cv2.medianBlur ksize 3 per component, replicate border) over one level's block field.
// With doHist, also the global-median seed candidate of the next finer level (interp.py:141-142, np.median of the
// fine blocks' own-parent vectors): every parent vector is added to an exact histogram with the number of fine blocks
// that take it as their own parent; the last CTA reads off the order statistics k1 = (n-1)/2, k2 = n/2 and writes
// 2 x the median = v_k1 + v_k2, then clears the histogram for the next estimate.
__device__ __forceinline__ void median3Cta(const Median3Params& p, int cta, int ctas) {
    const int b = cta * 256 + threadIdx.x;
    const int n = p.bw * p.bh;
    if (b < n) {
        const int bx = b % p.bw, by = b / p.bw;
        float xs[9], ys[9];
        int k = 0;
#pragma unroll
        for (int j = -1; j <= 1; j++)
#pragma unroll
            for (int i = -1; i <= 1; i++) {
                const float2 v = p.in[clampi(by + j, 0, p.bh - 1) * p.bw + clampi(bx + i, 0, p.bw - 1)];
                xs[k] = v.x;
                ys[k] = v.y;
                k++;
            }
        const float2 m = make_float2(med9(xs), med9(ys));
        p.out[b] = m;
        if (p.doHist) {
            const int wx = bx < p.bw - 1 ? max(0, min(2, p.fbw - 2 * bx)) : max(0, p.fbw - 2 * bx);
            const int wy = by < p.bh - 1 ? max(0, min(2, p.fbh - 2 * by)) : max(0, p.fbh - 2 * by);
            const unsigned int wgt = (unsigned int)(wx * wy);
            if (wgt) {
                int ix = __float2int_rn(m.x) + p.B, iy = __float2int_rn(m.y) + p.B;
                if (ix < 0 || ix > 2 * p.B || iy < 0 || iy > 2 * p.B) {
                    atomicOr(p.err, kErrHistRange);
                    ix = clampi(ix, 0, 2 * p.B);
                    iy = clampi(iy, 0, 2 * p.B);
                }
                atomicAdd(p.hist + ix, wgt);
                atomicAdd(p.hist + (2 * p.B + 1) + iy, wgt);
            }
        }
    }
    if (!p.doHist) return;
    __shared__ unsigned int ticket;
    __shared__ unsigned int part[256];
    __shared__ int found[4];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) ticket = atomicAdd(p.done, 1u);
    __syncthreads();
    if (ticket != (unsigned int)ctas - 1u) return;
    __threadfence();
    if (threadIdx.x < 4) found[threadIdx.x] = 0;
    const int nb = 2 * p.B + 1;
    const unsigned int N = (unsigned int)(p.fbw * p.fbh), ks[2] = {(N - 1) / 2, N / 2};
    const int per = (nb + 255) / 256;
    const unsigned int lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    for (int axis = 0; axis < 2; axis++) {
        const unsigned int* h = p.hist + axis * nb;
        const int s0 = threadIdx.x * per, s1 = min(s0 + per, nb);
        unsigned int loc = 0;
        for (int i = s0; i < s1; i++) loc += __ldcg(h + i);
        unsigned int inc = loc;   // inclusive scan of the 256 partial sums: within each warp, then across the 8 warps
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int n = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (unsigned int)o) inc += n;
        }
        if (lane == 31) part[wid] = inc;
        __syncthreads();
        unsigned int wofs = 0;
        for (unsigned int w = 0; w < wid; w++) wofs += part[w];
        unsigned int acc = wofs + inc - loc;
        for (int i = s0; i < s1; i++) {
            const unsigned int hv = __ldcg(h + i);
            for (int q = 0; q < 2; q++)
                if (acc <= ks[q] && ks[q] < acc + hv) found[axis * 2 + q] = i - p.B;
            acc += hv;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        p.medOut[0] = (float)(found[0] + found[1]);
        p.medOut[1] = (float)(found[2] + found[3]);
        *p.done = 0;
    }
    for (int i = threadIdx.x; i < 2 * nb; i += 256) p.hist[i] = 0;
}
__global__ void __launch_bounds__(256) k_median3(const Median3Params p) {
    pdlEnter();
    median3Cta(p, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) k_median3_m(const __grid_constant__ Merged<Median3Params> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    median3Cta(m.item[i], bx, m.first[i + 1] - m.first[i]);
}

// One block of k_median3's work for the shared-memory forms below: the block's 3x3 medians (written to p.out), and
// its own-parent weight added to the histogram hist (2 * nb bins in shared memory: x then y).
__device__ __forceinline__ void med3Block(const Median3Params& p, int b, unsigned int* hist, int nb) {
    const int bx = b % p.bw, by = b / p.bw;
    float xs[9], ys[9];
    int k = 0;
#pragma unroll
    for (int j = -1; j <= 1; j++)
#pragma unroll
        for (int i = -1; i <= 1; i++) {
            const float2 v = p.in[clampi(by + j, 0, p.bh - 1) * p.bw + clampi(bx + i, 0, p.bw - 1)];
            xs[k] = v.x;
            ys[k] = v.y;
            k++;
        }
    const float2 m = make_float2(med9(xs), med9(ys));
    p.out[b] = m;
    const int wx = bx < p.bw - 1 ? max(0, min(2, p.fbw - 2 * bx)) : max(0, p.fbw - 2 * bx);
    const int wy = by < p.bh - 1 ? max(0, min(2, p.fbh - 2 * by)) : max(0, p.fbh - 2 * by);
    const unsigned int wgt = (unsigned int)(wx * wy);
    if (wgt) {
        int ix = __float2int_rn(m.x) + p.B, iy = __float2int_rn(m.y) + p.B;
        if (ix < 0 || ix > 2 * p.B || iy < 0 || iy > 2 * p.B) {
            atomicOr(p.err, kErrHistRange);
            ix = clampi(ix, 0, 2 * p.B);
            iy = clampi(iy, 0, 2 * p.B);
        }
        atomicAdd(hist + ix, wgt);
        atomicAdd(hist + nb + iy, wgt);
    }
}

constexpr int kMed1Threads = 1024, kMed1Blocks = 2048, kMed1MaxBins = 4097;

// The global median from a complete histogram in shared memory, by all kMed1Threads threads of the CTA: the order
// statistics k1 = (N - 1) / 2, k2 = N / 2 of each axis (chunk sums, a block-wide scan, a walk of the chunk), written
// as 2 x the median = v_k1 + v_k2 to p.medOut.
__device__ __forceinline__ void medianFromHist(const Median3Params& p, const unsigned int* hist, int nb) {
    __shared__ unsigned int part[32];
    __shared__ int found[4];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid < 4) found[tid] = 0;
    const unsigned int N = (unsigned int)(p.fbw * p.fbh), ks[2] = {(N - 1) / 2, N / 2};
    const int per = (nb + kMed1Threads - 1) / kMed1Threads;
    for (int axis = 0; axis < 2; axis++) {
        const unsigned int* h = hist + axis * nb;
        const int s0 = tid * per, s1 = min(s0 + per, nb);
        unsigned int loc = 0;
        for (int i = s0; i < s1; i++) loc += h[i];
        unsigned int inc = loc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) part[wid] = inc;
        __syncthreads();
        if (wid == 0) {   // the warps' totals -> their exclusive offsets
            const unsigned int tot = part[lane];
            unsigned int x = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int v = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += v;
            }
            part[lane] = x - tot;
        }
        __syncthreads();
        unsigned int acc = part[wid] + inc - loc;
        for (int i = s0; i < s1; i++) {
            const unsigned int hv = h[i];
            for (int q = 0; q < 2; q++)
                if (acc <= ks[q] && ks[q] < acc + hv) found[axis * 2 + q] = i - p.B;
            acc += hv;
        }
        __syncthreads();
    }
    if (tid == 0) {
        p.medOut[0] = (float)(found[0] + found[1]);
        p.medOut[1] = (float)(found[2] + found[3]);
    }
}

// k_median3 for a level small enough for one CTA (at most kMed1Blocks blocks; the histogram fits in shared memory):
// the same medians and the same global median, with the histogram in shared memory and the order statistics read
// off by the same CTA, so no global atomics, no fence and no last-block ticket stand in the estimate's critical path
// (the coarse levels are latency bound).
__device__ __forceinline__ void median3OneCta(const Median3Params& p) {
    extern __shared__ unsigned int hs1[];   // 2 * nb bins: x then y
    const int nb = 2 * p.B + 1, tid = threadIdx.x;
    for (int i = tid; i < 2 * nb; i += kMed1Threads) hs1[i] = 0;
    __syncthreads();
    const int n = p.bw * p.bh;
#pragma unroll 2
    for (int b = tid; b < n; b += kMed1Threads) med3Block(p, b, hs1, nb);
    __syncthreads();
    medianFromHist(p, hs1, nb);
}
__global__ void __launch_bounds__(kMed1Threads, 1) k_median3_one(const Median3Params p) {
    pdlEnter();
    median3OneCta(p);
}
__global__ void __launch_bounds__(kMed1Threads, 1) k_median3_one_m(const __grid_constant__ Merged<Median3Params> m) {
    pdlEnter();
    median3OneCta(m.item[blockIdx.x]);   // one CTA per item
}

// k_median3 for mid-size levels (at most kMedClBlocks blocks): a cluster of kMedCl CTAs, each with its own histogram
// in shared memory; after the cluster barrier CTA 0 adds the others' histograms through distributed shared memory and
// reads off the order statistics. No global atomics, no fence, no last-block ticket; the other CTAs stay resident
// (a second cluster barrier) until CTA 0 has read their shared memory.
constexpr int kMedCl = 8, kMedClBlocks = kMedCl * kMed1Threads * 2;
__device__ __forceinline__ void median3ClusterCta(const Median3Params& p) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ unsigned int hs1[];
    const int nb = 2 * p.B + 1, tid = threadIdx.x;
    const unsigned int rank = cl.block_rank();
    for (int i = tid; i < 2 * nb; i += kMed1Threads) hs1[i] = 0;
    __syncthreads();
    const int n = p.bw * p.bh;
#pragma unroll 2
    for (int b = (int)rank * kMed1Threads + tid; b < n; b += kMedCl * kMed1Threads) med3Block(p, b, hs1, nb);
    cl.sync();   // every CTA's histogram is complete
    if (rank == 0) {
        for (int i = tid; i < 2 * nb; i += kMed1Threads) {
            unsigned int sum = hs1[i];
#pragma unroll
            for (int r = 1; r < kMedCl; r++) sum += cl.map_shared_rank(hs1, r)[i];
            hs1[i] = sum;
        }
        __syncthreads();
        medianFromHist(p, hs1, nb);
    }
    cl.sync();
}
__global__ void __cluster_dims__(kMedCl, 1, 1) __launch_bounds__(kMed1Threads, 1) k_median3_cluster(const Median3Params p) {
    pdlEnter();
    median3ClusterCta(p);
}
__global__ void __cluster_dims__(kMedCl, 1, 1) __launch_bounds__(kMed1Threads, 1)
    k_median3_cluster_m(const __grid_constant__ Merged<Median3Params> m) {
    pdlEnter();
    median3ClusterCta(m.item[blockIdx.x / kMedCl]);   // one cluster per item
}

// ============================================================================================== scene-cut mean
// numpy's pairwise float32 sum of a leaf: fewer than 8 elements summed from 0, else 8 running sums, folded
// ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the remainder in order (numpy pairwise_sum).
__device__ float pairwiseLeaf(const float* a, int n) {
    if (n < 8) {
        float r = 0.0f;
        for (int i = 0; i < n; i++) r = __fadd_rn(r, __ldcg(a + i));
        return r;
    }
    float r[8];
#pragma unroll
    for (int j = 0; j < 8; j++) r[j] = __ldcg(a + j);
    int i = 8;
    for (; i < n - (n % 8); i += 8)
#pragma unroll
        for (int j = 0; j < 8; j++) r[j] = __fadd_rn(r[j], __ldcg(a + i + j));
    float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])), __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; i++) res = __fadd_rn(res, __ldcg(a + i));
    return res;
}

// interp.estimate :189-190 (sad.mean() > CUT_SAD): the pairwise tree of the host-built plan, leaves in parallel,
// then one step per tree height; the float32 division by n; plus the debug counter's sum of roundEven(sad * 256).
// Runs in one CTA of `nt` threads; `vals` holds nLeaves + nInner floats.
__device__ void cutMeanBlock(const float* sads, int n, const CutPlan& plan, float cutSad, DevState* st, float* vals,
                             unsigned int* red) {
    const int nt = blockDim.x, tid = threadIdx.x;
    for (int i = tid; i < plan.nLeaves; i += nt) {
        const int2 lf = plan.leaves[i];
        vals[i] = pairwiseLeaf(sads + lf.x, lf.y);
    }
    unsigned int s256 = 0;
    for (int i = tid; i < n; i += nt) s256 += (unsigned int)__float2int_rn(__fmul_rn(__ldcg(sads + i), 256.0f));
    red[tid] = s256;
    __syncthreads();
    for (int d = 0; d < plan.nSteps; d++) {
        for (int j = plan.depthStart[d] + tid; j < plan.depthStart[d + 1]; j += nt) {
            const int2 c = plan.inner[j];
            vals[plan.nLeaves + j] = __fadd_rn(vals[c.x], vals[c.y]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        unsigned int tot = 0;
        for (int i = 0; i < nt; i++) tot += red[i];
        const float mean = __fdiv_rn(vals[plan.root], (float)n);
        st->sadMean = mean;
        st->cut = mean > cutSad ? 1u : 0u;
        st->sadSum256 = tot;
    }
}

__global__ void __launch_bounds__(256) k_cutmean(const CutMeanParams p) {
    pdlEnter();
    extern __shared__ float vals[];
    __shared__ unsigned int red[256];
    const bool inSmem = (size_t)(p.plan.nLeaves + p.plan.nInner) * sizeof(float) <= kPlanSmemMax;
    cutMeanBlock(p.sads, p.n, p.plan, p.cutSad, p.st, inSmem ? vals : p.plan.gvals, red);
}

// ============================================================================================== sub-pixel refinement
// interp.flow :162-163: search(., 1, 0.5) then search(., 1, 0.25) around the median-filtered integer vector s, one
// warp per finest-level block. Both frames' 13x13 windows (block +- 2 px around q -+ s) are staged in shared memory.
// Every pass samples each frame on a 24 x 24 lattice: per axis, the 8 pixel positions times the pass's 3 offsets
// (base + step * {-1, 0, 1}, quarter-pixel units). The lattice is built separably (horizontal then vertical, weights
// multiples of 1/4: every product and sum is exact, so it equals cv2's bilinear tap), after which a candidate's SAD is
// two shared loads per pixel. The scene-cut mean of the winners' SADs (numpy's pairwise sum) is spread over the grid:
// the warp that writes the last SAD of a leaf of the summation tree sums that leaf, and the warp that completes the
// last leaf adds the inner nodes.
constexpr int kSubT = 13, kSubO = 2, kSubL = 24, kSubRows = 10;   // tile, its margin, lattice side, tile rows used
constexpr int kSubWarpFloats = 2 * kSubT * kSubT + 2 * kSubRows * kSubL + 72;

// One leaf of the pairwise tree by one warp, in numpy's order: lanes 0..7 are its 8 accumulators (independent loads),
// combined as ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the tail; leaves under 8 elements by lane 0
// alone. Also returns (in every lane) the leaf's sum of roundEven(sad * 256), the debug counter's share.
__device__ __forceinline__ float warpLeafSum(const float* a, int n, int lane, unsigned int& s256) {
    unsigned int s = 0;
    for (int i = lane; i < n; i += 32) s += (unsigned int)__float2int_rn(__fmul_rn(__ldcg(a + i), 256.0f));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    s256 = s;
    float res = 0.0f;
    if (n < 8) {
        if (lane == 0)
            for (int i = 0; i < n; i++) res = __fadd_rn(res, __ldcg(a + i));
        return __shfl_sync(0xffffffffu, res, 0);
    }
    const int body = n - (n % 8);
    float r = 0.0f;
    if (lane < 8) {
        r = __ldcg(a + lane);
        for (int i = 8 + lane; i < body; i += 8) r = __fadd_rn(r, __ldcg(a + i));
    }
    const float r1 = __shfl_down_sync(0xffffffffu, r, 1);   // lane 2k: r[2k] + r[2k+1]
    const float p2 = __fadd_rn(r, r1);
    const float p2b = __shfl_down_sync(0xffffffffu, p2, 2);  // lane 4k: (r0 + r1) + (r2 + r3)
    const float p4 = __fadd_rn(p2, p2b);
    const float p4b = __shfl_down_sync(0xffffffffu, p4, 4);
    if (lane == 0) {
        res = __fadd_rn(p4, p4b);
        for (int i = body; i < n; i++) res = __fadd_rn(res, __ldcg(a + i));
    }
    return __shfl_sync(0xffffffffu, res, 0);
}

// the scene-cut mean's share of the warp that wrote the SAD of block b (warp-uniform call)
__device__ __forceinline__ void cutMeanShare(const SubpixParams& p, int b, int nb, int lane) {
    const CutPlan& pl = p.plan;
    const int leaf = pl.leafOf[b];
    unsigned int old = 0;
    if (lane == 0) {
        __threadfence();   // this warp's SAD before its arrival
        old = atomicAdd(pl.leafCnt + leaf, 1u);
    }
    old = __shfl_sync(0xffffffffu, old, 0);
    const int2 lf = pl.leaves[leaf];
    if (old != (unsigned int)lf.y - 1u) return;
    __threadfence();
    unsigned int s256;
    const float v = warpLeafSum(p.sads + lf.x, lf.y, lane, s256);
    unsigned int done = 0;
    if (lane == 0) {
        pl.gvals[leaf] = v;
        pl.leafS256[leaf] = s256;
        pl.leafCnt[leaf] = 0;
        __threadfence();
        done = atomicAdd(&p.st->subDone, 1u);
    }
    done = __shfl_sync(0xffffffffu, done, 0);
    if (done != (unsigned int)pl.nLeaves - 1u) return;
    // the last leaf: the inner nodes, one height per step, then the mean and the debug counter
    __threadfence();
    for (int d = 0; d < pl.nSteps; d++) {
        for (int j = pl.depthStart[d] + lane; j < pl.depthStart[d + 1]; j += 32) {
            const int2 c = pl.inner[j];
            pl.gvals[pl.nLeaves + j] = __fadd_rn(__ldcg(pl.gvals + c.x), __ldcg(pl.gvals + c.y));
        }
        __threadfence_block();
        __syncwarp();
    }
    unsigned int tot = 0;
    for (int i = lane; i < pl.nLeaves; i += 32) tot += __ldcg(pl.leafS256 + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) {
        const float mean = __fdiv_rn(__ldcg(pl.gvals + pl.root), (float)nb);
        p.st->sadMean = mean;
        p.st->cut = mean > p.cutSad ? 1u : 0u;
        p.st->sadSum256 = tot;
        p.st->subDone = 0;
    }
}

__device__ __forceinline__ void subpixCta(const SubpixParams& p, int cta) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = cta * 4 + warp;
    const int nb = p.bw * p.bh;
    if (b < nb) {
        float* tA = smem + warp * kSubWarpFloats;
        float* tC = tA + kSubT * kSubT;
        float2* H = reinterpret_cast<float2*>(tC + kSubT * kSubT);   // kSubRows x kSubL: (a, c) at tile rows 1..10
        float* rows = reinterpret_cast<float*>(H + kSubRows * kSubL);
        const int bx = b % p.bw, by = b / p.bw, b0x = bx * kBlock, b0y = by * kBlock;
        const float2 v0 = p.in[b];
        const int sx = __float2int_rn(v0.x), sy = __float2int_rn(v0.y);
        const int ax0 = b0x - sx - kSubO, ay0 = b0y - sy - kSubO, cx0 = b0x + sx - kSubO, cy0 = b0y + sy - kSubO;
        if (ax0 >= 0 && ay0 >= 0 && ax0 + kSubT <= p.w && ay0 + kSubT <= p.h && cx0 >= 0 && cy0 >= 0 &&
            cx0 + kSubT <= p.w && cy0 + kSubT <= p.h) {   // both windows inside the level: no clamps
            const float* ra = p.la + (size_t)ay0 * p.w + ax0;
            const float* rc = p.lc + (size_t)cy0 * p.w + cx0;
#pragma unroll
            for (int j = 0; j < (kSubT * kSubT + 31) / 32; j++) {
                const int i = lane + 32 * j;
                if (i < kSubT * kSubT) {
                    const int x = i % kSubT, y = i / kSubT;
                    tA[i] = __ldg(ra + y * p.w + x);
                    tC[i] = __ldg(rc + y * p.w + x);
                }
            }
        } else {
            for (int i = lane; i < kSubT * kSubT; i += 32) {
                const int x = i % kSubT, y = i / kSubT;
                tA[i] = Lc(p.la, p.w, p.h, ax0 + x, ay0 + y);
                tC[i] = Lc(p.lc, p.w, p.h, cx0 + x, cy0 + y);
            }
        }
        __syncwarp();
        // lane constants: lattice column u = 3 x + (d + 1) (lanes 24..31 only help with the reductions)
        const int u = lane < kSubL ? lane : kSubL - 1, ux = u / 3, ud = u % 3 - 1;
        int b4x = 0, b4y = 0;   // the offset chosen so far, quarter pixels
        float sadBest = 0.0f;
        for (int pass = 0; pass < 2; pass++) {
            const int s4 = pass ? 1 : 2;
            if (lane < kSubL) {
                // horizontal stage of column u: a at tile column x + 2 - o, c at x + 2 + o, o = (b4x + s4 d) / 4
                const int oA = 4 * (ux + kSubO) - (b4x + s4 * ud), oC = 4 * (ux + kSubO) + (b4x + s4 * ud);
                const float fA = (float)(oA & 3) * 0.25f, fC = (float)(oC & 3) * 0.25f;
                const float2 w0 = make_float2(1.0f - fA, 1.0f - fC), w1 = make_float2(fA, fC);
                const float* ra = tA + kSubT + (oA >> 2);
                const float* rc = tC + kSubT + (oC >> 2);
#pragma unroll
                for (int r = 0; r < kSubRows; r++) {   // exact: dyadic values, <= 16 significant bits
                    const float2 s0 = make_float2(ra[r * kSubT], rc[r * kSubT]), s1 = make_float2(ra[r * kSubT + 1], rc[r * kSubT + 1]);
                    H[r * kSubL + u] = __ffma2_rn(s1, w1, pmul(s0, w0));
                }
            }
            __syncwarp();
            if (lane < kSubL) {
                // vertical stage fused with the SADs: lattice row v = 3 y + (d + 1) reads the horizontal rows
                // y + rA[d] and y + rA[d] + 1 (rA in {0, 1}); lane u = 3 x + (dx + 1) adds |a - c| of pixel (x, y)
                // to candidate (dx, d - 1) for every y
                int rA[3], rC[3];
                float2 w0[3], w1[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int oA = -(b4y + s4 * (d - 1)), oC = b4y + s4 * (d - 1);
                    const float fA = (float)(oA & 3) * 0.25f, fC = (float)(oC & 3) * 0.25f;
                    rA[d] = 1 + (oA >> 2);
                    rC[d] = 1 + (oC >> 2);
                    w0[d] = make_float2(1.0f - fA, 1.0f - fC);
                    w1[d] = make_float2(fA, fC);
                }
                float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
#pragma unroll
                for (int y = 0; y < 8; y++) {
                    const float2 r0 = H[y * kSubL + u], r1 = H[(y + 1) * kSubL + u], r2 = H[(y + 2) * kSubL + u];
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const float2 ta = rA[d] ? r1 : r0, tb = rA[d] ? r2 : r1;   // a rows
                        const float2 tc = rC[d] ? r1 : r0, td = rC[d] ? r2 : r1;   // c rows
                        const float2 q = __ffma2_rn(make_float2(tb.x, td.y), w1[d], pmul(make_float2(ta.x, tc.y), w0[d]));
                        const float dd = fabsf(q.x - q.y);
                        if (d == 0) acc0 += dd; else if (d == 1) acc1 += dd; else acc2 += dd;
                    }
                }
                rows[(0 * 3 + ud + 1) * 8 + ux] = acc0;
                rows[(1 * 3 + ud + 1) * 8 + ux] = acc1;
                rows[(2 * 3 + ud + 1) * 8 + ux] = acc2;
            }
            __syncwarp();
            float cost = FLT_MAX, sad = 0.0f;
            if (lane < 9) {
                float sum = 0.0f;
#pragma unroll
                for (int y = 0; y < 8; y++) sum += rows[lane * 8 + y];
                sad = __fmul_rn(sum, 1.0f / 64.0f);
                cost = __fadd_rn(sad, p.pen[pass][abs(lane % 3 - 1) + abs(lane / 3 - 1)]);
            }
            int bi = lane;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float oc = __shfl_xor_sync(0xffffffffu, cost, o), os = __shfl_xor_sync(0xffffffffu, sad, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (oc < cost || (oc == cost && oi < bi)) { cost = oc; bi = oi; sad = os; }
            }
            b4x += s4 * (bi % 3 - 1);
            b4y += s4 * (bi / 3 - 1);
            sadBest = sad;
            if (pass == 0 && p.out0 && lane == 0)
                p.out0[b] = make_float2(__fadd_rn((float)sx, (float)b4x * 0.25f), __fadd_rn((float)sy, (float)b4y * 0.25f));
            __syncwarp();
        }
        if (lane == 0) {
            p.out[b] = make_float2(__fadd_rn((float)sx, (float)b4x * 0.25f), __fadd_rn((float)sy, (float)b4y * 0.25f));
            p.sads[b] = sadBest;
        }
        cutMeanShare(p, b, nb, lane);
    }
}
__global__ void __launch_bounds__(128) k_subpix(const SubpixParams p) {
    pdlEnter();
    subpixCta(p, blockIdx.x);
}
__global__ void __launch_bounds__(128) k_subpix_m(const __grid_constant__ Merged<SubpixParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    subpixCta(m.item[i], bx);
}

// ============================================================================================== per-pixel field
// interp.pixel_field :167-183 at flow resolution. Candidates per pixel: the bilinear block field (cv2.resize x8,
// INTER_LINEAR), the own block, the blocks above / below / left / right (edge-clamped), zero. Each candidate's cost is
// the 5x5 replicate-border box of |a(q - h) - c(q + h)| where every window pixel uses its own candidate (cv2.blur over
// the per-candidate error image). One CTA = a 64 x 32 region (60 x 28 outputs + a 2 px apron), one candidate at a
// time through one error plane. A vector h enters the taps only through R = rne(32 h): cv2 samples a at 32 q - R and c
// at 32 q + R (1/32 units; q - h is exact in float here). The taps are exact (dyadic luma, integer weights), the errors
// are exact multiples of 2^-14 summed as int32, and the mean is formed as cv2's box filter does: (S 2^-14) * (1/25) in
// double, then to float.
constexpr int kPfE = 64, kPfEH = 32, kPfAp = 2, kPfTW = kPfE - 2 * kPfAp, kPfTH = kPfEH - 2 * kPfAp, kPfNC = 7;
constexpr int kPfK = kPfEH / 4;                  // region rows per thread
constexpr int kPfBX = kPfE / 8 + 3, kPfBY = kPfEH / 8 + 3;   // block-field region (with the +-1 neighbours)

// one luma tap at 1/32 position (X, Y) of both frames at once: (a at (XA, YA), c at (XC, YC)); returns 1024 x the tap
__device__ __forceinline__ float2 tapPair(const float* __restrict__ ya, const float* __restrict__ yc, int w, int h,
                                          int XA, int YA, int XC, int YC) {
    const int iax = XA >> 5, iay = YA >> 5, icx = XC >> 5, icy = YC >> 5;
    float2 p00, p01, p10, p11;
    if ((unsigned)iax < (unsigned)(w - 1) && (unsigned)iay < (unsigned)(h - 1) && (unsigned)icx < (unsigned)(w - 1) &&
        (unsigned)icy < (unsigned)(h - 1)) {
        const float* qa = ya + iay * w + iax;
        const float* qc = yc + icy * w + icx;
        p00 = make_float2(__ldg(qa), __ldg(qc));
        p01 = make_float2(__ldg(qa + 1), __ldg(qc + 1));
        p10 = make_float2(__ldg(qa + w), __ldg(qc + w));
        p11 = make_float2(__ldg(qa + w + 1), __ldg(qc + w + 1));
    } else {
        const int ax0 = clampi(iax, 0, w - 1), ax1 = clampi(iax + 1, 0, w - 1), ay0 = clampi(iay, 0, h - 1) * w, ay1 = clampi(iay + 1, 0, h - 1) * w;
        const int cx0 = clampi(icx, 0, w - 1), cx1 = clampi(icx + 1, 0, w - 1), cy0 = clampi(icy, 0, h - 1) * w, cy1 = clampi(icy + 1, 0, h - 1) * w;
        p00 = make_float2(__ldg(ya + ay0 + ax0), __ldg(yc + cy0 + cx0));
        p01 = make_float2(__ldg(ya + ay0 + ax1), __ldg(yc + cy0 + cx1));
        p10 = make_float2(__ldg(ya + ay1 + ax0), __ldg(yc + cy1 + cx0));
        p11 = make_float2(__ldg(ya + ay1 + ax1), __ldg(yc + cy1 + cx1));
    }
    const float2 wx1 = make_float2(i2f(XA & 31), i2f(XC & 31)), wy1 = make_float2(i2f(YA & 31), i2f(YC & 31));
    const float2 wx0 = padd(make_float2(32.0f, 32.0f), make_float2(-wx1.x, -wx1.y));
    const float2 wy0 = padd(make_float2(32.0f, 32.0f), make_float2(-wy1.x, -wy1.y));
    // exact: luma (dyadic, <= 10 significant bits) x integer weights <= 32 per stage
    const float2 h0 = __ffma2_rn(p01, wx1, pmul(p00, wx0));
    const float2 h1 = __ffma2_rn(p11, wx1, pmul(p10, wx0));
    return __ffma2_rn(h1, wy1, pmul(h0, wy0));
}

// the horizontal stage of one tap row of both frames: a at row ra (columns ax0, ax1), c at row rc (cx0, cx1), rows
// clamped; returns 32 x the row's value of each (tapPair's h0 / h1)
__device__ __forceinline__ float2 tapRowPair(const float* __restrict__ ya, const float* __restrict__ yc, int w, int h,
                                             int ra, int rc, int ax0, int ax1, int cx0, int cx1, float2 wx0, float2 wx1) {
    const float* qa = ya + clampi(ra, 0, h - 1) * w;
    const float* qc = yc + clampi(rc, 0, h - 1) * w;
    return __ffma2_rn(make_float2(__ldg(qa + ax1), __ldg(qc + cx1)), wx1, pmul(make_float2(__ldg(qa + ax0), __ldg(qc + cx0)), wx0));
}

// Candidates 1..5 (the vector of the pixel's own block or of a 4-neighbour) are constant over a block: the thread walks
// down kPfK consecutive region rows of its column with one set of taps and weights per block, each row's lower tap row
// being the next row's upper one (the rows are the same for every lane, so the branches are uniform). Same taps,
// weights and operation order as tapPair.
__device__ __forceinline__ void pfBlockCandidate(const PixfieldParams& p, int k, int qx, int Y0, int ey0, int ex, int bx0,
                                                 int by0, const int2 (*bR)[kPfBX], int (*plane)[kPfE + 1]) {
    const int dxk = k == 4 ? -1 : (k == 5 ? 1 : 0), dyk = k == 2 ? -1 : (k == 3 ? 1 : 0);
    const int bx = clampi((qx >> 3) + dxk, 0, p.bw - 1) - bx0;
    int ax0 = 0, ax1 = 0, cx0 = 0, cx1 = 0, dya = 0, dyc = 0, by = -1, qyPrev = -1, E = 0;
    float2 wx0 = make_float2(0.0f, 0.0f), wx1 = wx0, wy0 = wx0, wy1 = wx0, top = wx0, bot = wx0;
#pragma unroll
    for (int j = 0; j < kPfK; j++) {
        const int ey = ey0 * kPfK + j;
        const int qy = clampi(Y0 - kPfAp + ey, 0, p.h - 1);
        if (qy != qyPrev) {   // a clamped row repeats the previous one
            const int b = clampi((qy >> 3) + dyk, 0, p.bh - 1) - by0;
            if (b != by) {    // a new block row: this lane's vector, taps and weights; both tap rows
                by = b;
                const int2 R = bR[b][bx];
                const int ia = qx + ((-R.x) >> 5), ic = qx + (R.x >> 5);
                ax0 = clampi(ia, 0, p.w - 1);
                ax1 = clampi(ia + 1, 0, p.w - 1);
                cx0 = clampi(ic, 0, p.w - 1);
                cx1 = clampi(ic + 1, 0, p.w - 1);
                dya = (-R.y) >> 5;
                dyc = R.y >> 5;
                wx1 = make_float2(i2f((-R.x) & 31), i2f(R.x & 31));
                wy1 = make_float2(i2f((-R.y) & 31), i2f(R.y & 31));
                wx0 = padd(make_float2(32.0f, 32.0f), make_float2(-wx1.x, -wx1.y));
                wy0 = padd(make_float2(32.0f, 32.0f), make_float2(-wy1.x, -wy1.y));
                top = tapRowPair(p.ya, p.yc, p.w, p.h, qy + dya, qy + dyc, ax0, ax1, cx0, cx1, wx0, wx1);
            } else {
                top = bot;    // qy = qyPrev + 1 in the same block row
            }
            bot = tapRowPair(p.ya, p.yc, p.w, p.h, qy + dya + 1, qy + dyc + 1, ax0, ax1, cx0, cx1, wx0, wx1);
            const float2 t = __ffma2_rn(bot, wy1, pmul(top, wy0));
            E = __float_as_int(__fmaf_rn(fabsf(t.x - t.y), 16.0f, 12582912.0f)) - 0x4B400000;   // E * 2^14
            qyPrev = qy;
        }
        plane[ey][ex] = E;
    }
}

__device__ __forceinline__ void pixfieldCta(const PixfieldParams& p, int ctaX, int ctaY) {
    // rows padded by one word: the horizontal sums below read down the rows of a column group, one row per lane
    __shared__ int plane[kPfEH][kPfE + 1];
    __shared__ int plane0[kPfEH][kPfE + 1];   // the zero candidate's errors, computed once
    __shared__ int hs[kPfEH][kPfE + 1];
    __shared__ float2 bv[kPfBY][kPfBX];
    __shared__ int2 bR[kPfBY][kPfBX];
    __shared__ float4 rowc[kPfEH];   // bilinear candidate, y: (row0, row1 relative to the block region, weights)
    const int tid = threadIdx.x, ex = tid & (kPfE - 1), ey0 = tid >> 6;
    const int X0 = ctaX * kPfTW, Y0 = ctaY * kPfTH;
    // the block-field region: every block a region pixel's candidates can name
    const int qx0 = clampi(X0 - kPfAp, 0, p.w - 1), qy0 = clampi(Y0 - kPfAp, 0, p.h - 1);
    const int bx0 = max((qx0 >> 3) - 1, 0), by0 = max((qy0 >> 3) - 1, 0);
    for (int i = tid; i < kPfBX * kPfBY; i += 256) {
        const int bx = min(bx0 + i % kPfBX, p.bw - 1), by = min(by0 + i / kPfBX, p.bh - 1);
        const float2 v = __ldg(p.v + by * p.bw + bx);
        bv[i / kPfBX][i % kPfBX] = v;
        const float2 r = rne32bits(v);
        bR[i / kPfBX][i % kPfBX] = make_int2(__float_as_int(r.x) - 0x4B400000, __float_as_int(r.y) - 0x4B400000);
    }
    // cv2.resize x8 coefficients: x per thread column (weights (1, 0) beyond the borders), y per region row (rows
    // clamped, weights kept)
    const int qx = clampi(X0 - kPfAp + ex, 0, p.w - 1);
    int cx0, cx1;
    float ca0, ca1;
    {
        float f = __fsub_rn(__fmul_rn((float)qx + 0.5f, 0.125f), 0.5f);
        int sft = (int)floorf(f);
        f = __fsub_rn(f, (float)sft);
        if (sft < 0) { sft = 0; f = 0.0f; }
        if (sft >= p.bw - 1) { sft = p.bw - 1; f = 0.0f; }
        cx0 = clampi(sft, 0, p.bw - 1) - bx0;
        cx1 = clampi(sft + 1, 0, p.bw - 1) - bx0;
        ca0 = 1.0f - f;
        ca1 = f;
    }
    if (tid < kPfEH) {
        const int qy = clampi(Y0 - kPfAp + tid, 0, p.h - 1);
        float f = __fsub_rn(__fmul_rn((float)qy + 0.5f, 0.125f), 0.5f);
        const int sft = (int)floorf(f);
        f = __fsub_rn(f, (float)sft);
        rowc[tid] = make_float4(__int_as_float(clampi(sft, 0, p.bh - 1) - by0), __int_as_float(clampi(sft + 1, 0, p.bh - 1) - by0),
                                1.0f - f, f);
    }
    __syncthreads();
    const int bxq = (qx >> 3) - bx0;   // this column's block in the region
    const int qx32 = 32 * qx;
    float best[kPfK];
    int bestk[kPfK];
    const double C = 0x1p-14 * (1.0 / 25.0);   // cv2's box scale with the 2^-14 units folded in (exact scaling)
#pragma unroll
    for (int j = 0; j < kPfK; j++) {   // the zero candidate: both taps at q itself (weights 32 x 32)
        const int ey = ey0 + 4 * j;
        const int qy = clampi(Y0 - kPfAp + ey, 0, p.h - 1);
        const float ta = __fmul_rn(__ldg(p.ya + qy * p.w + qx), 1024.0f), tc = __fmul_rn(__ldg(p.yc + qy * p.w + qx), 1024.0f);
        plane0[ey][ex] = __float_as_int(__fmaf_rn(fabsf(ta - tc), 16.0f, 12582912.0f)) - 0x4B400000;
    }
    for (int k = 0; k < kPfNC; k++) {
        // 1. candidate k's error at this thread's region pixels (the zero candidate's is plane0 already)
        if (k == 0) {   // the upsampled field: a vector per pixel
#pragma unroll
            for (int j = 0; j < kPfK; j++) {
                const int ey = ey0 + 4 * j;
                const int qy = clampi(Y0 - kPfAp + ey, 0, p.h - 1);
                const float4 ry = rowc[ey];
                const int r0 = __float_as_int(ry.x), r1 = __float_as_int(ry.y);
                const float2 h0 = padd(pmul(bv[r0][cx0], make_float2(ca0, ca0)), pmul(bv[r0][cx1], make_float2(ca1, ca1)));
                const float2 h1 = padd(pmul(bv[r1][cx0], make_float2(ca0, ca0)), pmul(bv[r1][cx1], make_float2(ca1, ca1)));
                const float2 r = rne32bits(padd(pmul(h0, make_float2(ry.z, ry.z)), pmul(h1, make_float2(ry.w, ry.w))));
                const int2 R = make_int2(__float_as_int(r.x) - 0x4B400000, __float_as_int(r.y) - 0x4B400000);
                const int qy32 = 32 * qy;
                const float2 t = tapPair(p.ya, p.yc, p.w, p.h, qx32 - R.x, qy32 - R.y, qx32 + R.x, qy32 + R.y);
                plane[ey][ex] = __float_as_int(__fmaf_rn(fabsf(t.x - t.y), 16.0f, 12582912.0f)) - 0x4B400000;   // E * 2^14
            }
        } else if (k < kPfNC - 1) {
            pfBlockCandidate(p, k, qx, Y0, ey0, ex, bx0, by0, bR, plane);
        }
        __syncthreads();
        // 2. horizontal 5-sums: one region row, 8 output columns per thread (a running window); the lanes of a warp
        //    take the 32 rows of one column group (conflict-free with the padded rows)
        {
            const int r = tid & 31, c0 = (tid >> 5) * 8;
            const int* q = k == kPfNC - 1 ? &plane0[r][c0] : &plane[r][c0];
            int sum = q[0] + q[1] + q[2] + q[3] + q[4];
            hs[r][c0] = sum;
#pragma unroll
            for (int c = 1; c < 8; c++) {
                if (c0 + c + 4 < kPfE) sum += q[c + 4] - q[c - 1];
                hs[r][c0 + c] = sum;
            }
        }
        __syncthreads();
        // 3. vertical 5-sums (a running window down this thread's kPfK consecutive output rows), the cost, the running
        //    first minimum
        const int lx = ex - kPfAp;
        if ((unsigned)lx < (unsigned)kPfTW) {
            const int ly0 = ey0 * kPfK;
            int S = hs[ly0][lx] + hs[ly0 + 1][lx] + hs[ly0 + 2][lx] + hs[ly0 + 3][lx];
#pragma unroll
            for (int j = 0; j < kPfK; j++) {
                const int ly = ly0 + j;
                if (ly >= kPfTH) break;   // uniform over the warp; later rows are out too
                S += hs[ly + 4][lx] - (j ? hs[ly - 1][lx] : 0);
                float c = (float)(__dadd_rn(__hiloint2double(0x43300000, S), -4503599627370496.0) * C);
                if (k == 0) c = __fsub_rn(c, p.smooth);
                if (k == kPfNC - 1) c = __fsub_rn(c, p.zero);
                if (k == 0 || c < best[j]) { best[j] = c; bestk[j] = k; }
            }
        }
    }
    // 4. the chosen candidate's vector
    const int lx = ex - kPfAp, x = X0 + lx;
    if ((unsigned)lx >= (unsigned)kPfTW || x >= p.w) return;
#pragma unroll
    for (int j = 0; j < kPfK; j++) {
        const int ly = ey0 * kPfK + j, ey = ly + kPfAp, y = Y0 + ly;
        if (ly >= kPfTH || y >= p.h) break;
        const int k = bestk[j];
        float2 v;
        if (k == 0) {
            const float4 ry = rowc[ey];
            const int r0 = __float_as_int(ry.x), r1 = __float_as_int(ry.y);
            const float2 h0 = padd(pmul(bv[r0][cx0], make_float2(ca0, ca0)), pmul(bv[r0][cx1], make_float2(ca1, ca1)));
            const float2 h1 = padd(pmul(bv[r1][cx0], make_float2(ca0, ca0)), pmul(bv[r1][cx1], make_float2(ca1, ca1)));
            v = padd(pmul(h0, make_float2(ry.z, ry.z)), pmul(h1, make_float2(ry.w, ry.w)));
        } else if (k == kPfNC - 1) {
            v = make_float2(0.0f, 0.0f);
        } else {
            const int dx = k == 4 ? -1 : (k == 5 ? 1 : 0), dy = k == 2 ? -1 : (k == 3 ? 1 : 0);
            v = bv[clampi((y >> 3) + dy, 0, p.bh - 1) - by0][clampi((x >> 3) + dx, 0, p.bw - 1) - bx0];
        }
        p.pf[(size_t)y * p.w + x] = v;
    }
    (void)bxq;
}
__global__ void __launch_bounds__(256) k_pixfield(const PixfieldParams p) {
    pdlEnter();
    pixfieldCta(p, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(256) k_pixfield_m(const __grid_constant__ Merged<PixfieldParams> m) {
    pdlEnter();
    int bx, by;
    const int i = mergedItem(m, bx, by);
    pixfieldCta(m.item[i], bx, by);
}

// ============================================================================================== synthesis
// interp.synth :219-246 for one time t, fused: the field at t (interp.field_at, flow res, recomputed per tile with
// its halo), its upsampling to full resolution (cv2.resize x fs INTER_LINEAR, crop / edge pad, x fs), the two
// bilinear 8-bit warps (cv2.remap of uint8: 5-bit fractions, integer weights, round half up), the max-channel
// mismatch, its 7x7 replicate box, the trust ramp, the untrusted count and the blend. One CTA = kSyTW x kSyTH output
// pixels; the mismatch is also computed on the 3-pixel halo the box needs. A scene cut (decided by the estimate)
// copies the nearer frame instead; the untrusted-share decision needs every CTA's count and is taken by k_fallback.
//
// Float <-> int conversions run on the FP32 pipe (magic-number additions, exact in the ranges used here) rather than
// the conversion units; the bilinear taps run two channels per 32-bit multiply (R|B lanes, G) and the mismatch and the
// t = 0.5 blend use byte-SIMD instructions.

// one cv2.remap INTER_LINEAR / BORDER_REPLICATE sample of a 4-byte-per-pixel 8-bit frame of at least 2 x 2 pixels
// at the position whose rne32 bits are (bx, by): channels 0..2 of the result (byte 3 = 0; also unpacked in ch).
// Borders: the 1/32-pixel position is clamped to [0, 32 (W - 1)], the left tap is min(X >> 5, W - 2) and the right
// weight X - 32 ix (0..32): at the right edge the taps (W - 2, W - 1) with weights (0, 32), the same products as cv2's
// (W - 1, W - 1) pair, so the four taps are always (ix, iy) + {0, 1}^2 (one address, fixed offsets). Filter: cv2's
// 15-bit weights of 5-bit bilinear fractions are 32 wx wy, and (sum p 32 wx wy + 2^14) >> 15 == (sum p wx wy + 512) >> 10
// with wx wy <= 1024; per channel two 16-bit x 8-bit dot products (dp2a) on tap bytes gathered by byte permutes, exact
// in 32 bits.
__device__ __forceinline__ uint32_t sampleU8(const uint32_t* __restrict__ img, uint32_t pw, int W, int H, float bxf, float byf,
                                             int ch[3]) {
    const int X = clampi(__float_as_int(bxf) - 0x4B400000, 0, 32 * (W - 1));
    const int Y = clampi(__float_as_int(byf) - 0x4B400000, 0, 32 * (H - 1));
    const int ix = min(X >> 5, W - 2), iy = min(Y >> 5, H - 2);
    const uint32_t fx = (uint32_t)(X - 32 * ix), fy = (uint32_t)(Y - 32 * iy);
    const uint32_t* q = img + ((uint32_t)iy * pw + (uint32_t)ix);
    const uint32_t p00 = __ldg(q), p01 = __ldg(q + 1), p10 = __ldg(q + pw), p11 = __ldg(q + pw + 1);
    const uint32_t wx = (32u - fx) | (fx << 16);            // (left, right) weights as 16-bit lanes
    const uint32_t w0 = wx * (32u - fy), w1 = wx * fy;      // (w00, w01), (w10, w11): lanes <= 1024, no carry
    const uint32_t rg0 = __byte_perm(p00, p01, 0x5140), rg1 = __byte_perm(p10, p11, 0x5140);   // R00 R01 G00 G01
    const uint32_t b0 = __byte_perm(p00, p01, 0x0062), b1 = __byte_perm(p10, p11, 0x6200);     // B00 B01 / - - B10 B11
    const uint32_t c0 = __dp2a_lo(w1, rg1, __dp2a_lo(w0, rg0, 512u)) >> 10;
    const uint32_t c1 = __dp2a_hi(w1, rg1, __dp2a_hi(w0, rg0, 512u)) >> 10;
    const uint32_t c2 = __dp2a_hi(w1, b1, __dp2a_lo(w0, b0, 512u)) >> 10;
    ch[0] = (int)c0;
    ch[1] = (int)c1;
    ch[2] = (int)c2;
    return c2 * 65536u + (c1 * 256u + c0);
}

// one output tile (bx, by) of one synthesis; all threads of the CTA take part. Each output pixel goes to
// sink(k, x, y, ly, o): k = this thread's region-row slot, (x, y) the pixel, ly its tile row, o the packed result
// (alpha = the nearer frame's). The untrusted count is added to *p.untrusted unless that is null. kCut: under a scene
// cut the tile is a copy of the nearer frame to p.out (and the core returns at once); without kCut the caller has
// taken the cut into account.
template <bool kCut, bool kUi = false, class Sink>
__device__ __forceinline__ void synthTileCore(const SynthParams& p, int bx, int by, Sink&& sink) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ SyCoef rowc[kSyEH];
    __shared__ float TA[256], TC[256];
    __shared__ unsigned int cnt;
    __shared__ int gReg[4];
    const int X0 = bx * kSyT, Y0 = by * kSyTH;
    const int tid = threadIdx.x, ex = tid & (kSyE - 1), ey0 = tid / kSyE;
    const uint8_t* nearF = p.nearC ? p.c : p.a;
    const uint32_t pitch = (uint32_t)p.pitch, pw = pitch >> 2;
    const uint32_t* fa32 = reinterpret_cast<const uint32_t*>(p.a);
    const uint32_t* fc32 = reinterpret_cast<const uint32_t*>(p.c);
    if (kCut && p.st->cut) {   // scene cut (interp.py:225-226): the nearer real frame
        for (int i = tid; i < kSyT * kSyTH; i += kSyThreads) {
            const int x = X0 + (i % kSyT), y = Y0 + (i / kSyT);
            if (x < p.W && y < p.H)
                reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] =
                    __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * pitch) + x);
        }
        return;
    }
    if (tid == 0) cnt = 0;
    if (tid < 256) {
        TA[tid] = __fmul_rn(p.wA, (float)tid);
        TC[tid] = __fmul_rn(p.wC, (float)tid);
    }
    float2* hrow;
    uint8_t* e;
    unsigned short* hsum;
    const SyCoef cx = syFieldStage(p, X0, Y0, tid, ex, ey0, rowc, gReg, sm, hrow, e, hsum);
    // 2. this thread's region column: half-vector (vertical stage, x fs folded in), both warps, mismatch. The warps
    //    wait in shared memory for the blend (in registers they would leave too few for the sample loads in flight).
    uint32_t* sWA = reinterpret_cast<uint32_t*>(hsum + kSyEH * kSyHS);   // the output rows: kSyTH x kSyE
    uint32_t* sWC = sWA + kSyTH * kSyE;
    const float kA = p.mid ? 1.0f : p.ka, kC = p.mid ? 1.0f : p.kc;   // t = 0.5: the products by 1 are exact
#pragma unroll
    for (int k = 0; k < kSyK; k++) {
        const int ey = ey0 + (kSyThreads / kSyE) * k;
        const SyCoef cy = rowc[ey];
        const float2 h0 = hrow[cy.i0 * kSyE + ex], h1 = hrow[cy.i1 * kSyE + ex];
        const float hx = __fadd_rn(__fmul_rn(h0.x, cy.a0), __fmul_rn(h1.x, cy.a1));
        const float hy = __fadd_rn(__fmul_rn(h0.y, cy.a0), __fmul_rn(h1.y, cy.a1));
        // a(q - 2t h), c(q + 2(1 - t) h): float32 products, then the sums (numpy's order)
        const float2 ba = rne32bits(make_float2(__fsub_rn(cx.pos, __fmul_rn(kA, hx)), __fsub_rn(cy.pos, __fmul_rn(kA, hy))));
        const float2 bc = rne32bits(make_float2(__fadd_rn(cx.pos, __fmul_rn(kC, hx)), __fadd_rn(cy.pos, __fmul_rn(kC, hy))));
        int ca[3], cc[3];
        uint32_t A = sampleU8(fa32, pw, p.W, p.H, ba.x, ba.y, ca), C = sampleU8(fc32, pw, p.W, p.H, bc.x, bc.y, cc);
        if (kUi) {   // CrosshairV2: a tap on its own frame's UI takes the other frame's tap (both or neither: kept)
            const bool ha = p.uiA && uiHitMask(p.uiA, __float_as_int(ba.x) - 0x4B400000, __float_as_int(ba.y) - 0x4B400000);
            const bool hc = p.uiC && uiHitMask(p.uiC, __float_as_int(bc.x) - 0x4B400000, __float_as_int(bc.y) - 0x4B400000);
            if (ha != hc) {
                if (ha) {
                    A = C;
                    ca[0] = cc[0]; ca[1] = cc[1]; ca[2] = cc[2];
                } else {
                    C = A;
                    cc[0] = ca[0]; cc[1] = ca[1]; cc[2] = ca[2];
                }
            }
        }
        if ((unsigned)(ey - kSyAp) < (unsigned)kSyTH) {   // warp-uniform
            sWA[(ey - kSyAp) * kSyE + ex] = A;
            sWC[(ey - kSyAp) * kSyE + ex] = C;
        }
        const int m = max(max(abs(ca[0] - cc[0]), abs(ca[1] - cc[1])), abs(ca[2] - cc[2]));
        e[ey * kSyES + ex] = (uint8_t)m;
    }
    const int lx = ex - kSyAp, x = X0 + lx;
    const bool colOk = (unsigned)lx < (unsigned)kSyT && x < p.W;   // this thread's output column
    __syncthreads();
    // 3. horizontal 7-sums: one region row and 8 output columns per thread, a running window
    syRowSums(e, hsum, tid);
    __syncthreads();
    // 4. this thread's output pixels: vertical 7-sum (a running window), trust, blend, store
    unsigned int myCnt = 0;
    // Weights that are multiples of 1/256 (t = k/256: 1/4, 3/4, ...) make every step of the blend exact (8-bit x 8-bit
    // products, sums below 2^17), so fl(fl(wA a) + fl(wC c)) + 0.5 floored is (WA a + WC c + 128) >> 8 with WA = 256 wA,
    // WC = 256 wC: two channels per 32-bit multiply-add (16-bit lanes, no carry while WA + WC <= 256)
    const float wa256 = __fmul_rn(p.wA, 256.0f), wc256 = __fmul_rn(p.wC, 256.0f);
    const bool dyad = !p.mid && wa256 == truncf(wa256) && wc256 == truncf(wc256) && wa256 >= 0.0f && wc256 >= 0.0f &&
                      __fadd_rn(wa256, wc256) <= 256.0f;
    const uint32_t WA = dyad ? (uint32_t)wa256 : 0u, WC = dyad ? (uint32_t)wc256 : 0u;
    if (colOk) {
        const unsigned short* q = hsum + syOutRow(ey0, 0) * kSyHS + lx;
        int S = q[0] + q[kSyHS] + q[2 * kSyHS] + q[3 * kSyHS] + q[4 * kSyHS] + q[5 * kSyHS];
#pragma unroll
        for (int k = 0; k < kSyK; k++) {
            const int ly = syOutRow(ey0, k), y = Y0 + ly;
            if (ly >= kSyTH || y >= p.H) break;   // uniform over the warp; later rows are out too
            S += q[(k + 6) * kSyHS] - (k ? q[(k - 1) * kSyHS] : 0);
            const uint32_t nq = __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * pitch) + x);
            const uint32_t wak = sWA[ly * kSyE + ex], wck = sWC[ly * kSyE + ex];
            uint32_t o;
            if (S <= p.sZero) {   // u = 0: out = the blend rounded
                if (p.mid) {
                    // floor(0.5 (a + c) + 0.5) per byte: (a | c) - ((a ^ c) >> 1), no borrow between bytes
                    o = (wak | wck) - (((wak ^ wck) >> 1) & 0x7F7F7F7Fu);
                } else if (dyad) {
                    const uint32_t M = 0x00FF00FFu;
                    const uint32_t rb = (wak & M) * WA + ((wck & M) * WC + 0x00800080u);
                    const uint32_t g = ((wak >> 8) & M) * WA + (((wck >> 8) & M) * WC + 0x00800080u);
                    o = ((rb >> 8) & M) | (g & 0x0000FF00u);
                } else {
                    // fl32(fl32((1 - t) a) + fl32(t c)) + 0.5, floored (never above 255.5 here, so no clamp is needed): the
                    // products come from the tables, the adds are paired (adds alone cannot be fused), the floor is a
                    // round-toward-zero add of 2^23 whose low mantissa byte is the result
                    const uint32_t A = wak, C = wck;
                    const float2 m01 = padd(make_float2(TA[A & 255u], TA[(A >> 8) & 255u]), make_float2(TC[C & 255u], TC[(C >> 8) & 255u]));
                    const float m2 = __fadd_rn(TA[(A >> 16) & 255u], TC[(C >> 16) & 255u]);
                    const float2 f01 = __ffma2_rz(padd(m01, make_float2(0.5f, 0.5f)), make_float2(1.0f, 1.0f), make_float2(8388608.0f, 8388608.0f));
                    const float f2 = __fadd_rz(__fadd_rn(m2, 0.5f), 8388608.0f);
                    o = __byte_perm(__byte_perm(__float_as_uint(f01.x), __float_as_uint(f01.y), 0x0040), __float_as_uint(f2), 0x0410);
                }
            } else if (S >= p.sOne) {   // u = 1: the nearer frame
                o = nq;
                myCnt++;
            } else {
                const float eb = (float)((double)S * (1.0 / 49.0));   // cv2.blur: double sum * (1/49), to float
                float u = __fdiv_rn(__fsub_rn(eb, p.trust0), p.trustSpan);
                u = fminf(fmaxf(u, 0.0f), 1.0f);
                myCnt += u > 0.5f;
                const float iu = 1.0f - u;
                o = 0;
#pragma unroll
                for (int k2 = 0; k2 < 3; k2++) {
                    const int sh = 8 * k2;
                    const uint32_t ca = (wak >> sh) & 255u, cc = (wck >> sh) & 255u;
                    const float fa = i2f((int)ca), fc = i2f((int)cc), fn = i2f((int)((nq >> sh) & 255u));
                    const float mix = p.mid ? __fmul_rn(0.5f, __fadd_rn(fa, fc)) : __fadd_rn(TA[ca], TC[cc]);
                    const float v = __fadd_rn(__fadd_rn(__fmul_rn(mix, iu), __fmul_rn(fn, u)), 0.5f);
                    o |= (uint32_t)floorPos(fminf(fmaxf(v, 0.0f), 255.0f)) << sh;
                }
            }
            o = (o & 0x00FFFFFFu) | (nq & 0xFF000000u);   // alpha (byte 3 in both pixel orders): the nearer frame's
            sink(k, x, y, ly, o);
            if (p.emap) p.emap[(size_t)y * ((p.W + 3) & ~3) + x] = e[(ly + kSyAp) * kSyES + ex];
        }
    }
    if (myCnt) atomicAdd(&cnt, myCnt);
    __syncthreads();
    if (tid == 0 && cnt && p.untrusted) atomicAdd(p.untrusted, cnt);
}

// one output tile of one synthesis, stored to p.out
template <bool kUi = false>
__device__ __forceinline__ void synthTile(const SynthParams& p, int bx, int by) {
    synthTileCore<true, kUi>(p, bx, by, [&](int, int x, int y, int, uint32_t o) {
        reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] = o;
    });
}

__global__ void __launch_bounds__(kSyThreads, 3) k_synth(const SynthParams p) {
    pdlEnter();
    synthTile(p, blockIdx.x, blockIdx.y);
}

// the same with CrosshairV2's warp-tap rejection (p.uiA / p.uiC); a separate kernel so the plain one is unchanged
__global__ void __launch_bounds__(kSyThreads, 3) k_synth_ui(const SynthParams p) {
    pdlEnter();
    synthTile<true>(p, blockIdx.x, blockIdx.y);
}

// Motion blur (gpu/framegen.h:553-573, gpu/shaders/blur_resolve.comp): out = round(sum_k w_k frame_k), frame_k the
// 8-bit frame recordSynth(t_k) gives (the nearer real frame under a scene cut or a whole-frame flick; prev / curr at
// t_k <= 0 / >= 1). One CTA per output tile runs the synthesis of every sample on the tile and accumulates it in
// registers (no sub-frame is written): per pixel and colour channel acc = sum q_k v_k, the weights q_k integers
// summing to 2^16; out = (acc + 2^15) >> 16. Alpha is the nearer frame's in every sub-frame, so it is the weighted
// mean of prev's and curr's alpha. A flick (more than globalFallback of a sample's pixels untrusted) is known only
// when every tile has counted: the main pass (fix = 0) assumes none and counts per sample; the fix-up pass (fix = 1)
// exits at once unless some synthesized sample flicked, and then redoes every tile with those samples replaced.
template <bool kUi>
__global__ void __launch_bounds__(kSyThreads, 2) k_synth_blur_t(const BlurParams bp) {
    pdlEnter();
    __shared__ __align__(16) SynthParams sp;
    __shared__ unsigned int sRepl, sRedo;   // samples replaced by a real frame; whether this pass has work
    __shared__ uint32_t sWp, sWc, sWap;     // weights of the replaced samples taking prev / curr; alpha weight of prev
    const int tid = threadIdx.x, ex = tid & (kSyE - 1), ey0 = tid / kSyE;
    const SynthParams& b = bp.base;
    if (tid == 0) {
        const bool cut = b.st->cut != 0;
        unsigned int repl = 0, flick = 0;
        uint32_t wp = 0, wc = 0, wap = 0;
        for (int k = 0; k < bp.n; k++) {
            const BlurSample& m = bp.smp[k];
            const bool nearC = m.mode == 2 || (m.mode == 0 && m.nearC);
            bool r = m.mode != 0 || cut;
            if (!r && bp.fix && (double)bp.cnt[k] / ((double)b.W * (double)b.H) > bp.frac) {
                r = true;
                flick |= 1u << k;
            }
            if (r) {
                repl |= 1u << k;
                if (nearC) wc += m.q; else wp += m.q;
            }
            if (!nearC) wap += m.q;
        }
        sRepl = repl;
        sRedo = !bp.fix || flick != 0;
        sWp = wp; sWc = wc; sWap = wap;
    }
    __syncthreads();
    if (!sRedo) return;
    const unsigned int repl = sRepl;
    uint32_t acc[kSyK][3];
#pragma unroll
    for (int k = 0; k < kSyK; k++) acc[k][0] = acc[k][1] = acc[k][2] = 0u;
    for (int j = 0; j < bp.n; j++) {
        if ((repl >> j) & 1u) continue;   // uniform over the CTA
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
        const uint32_t q = bp.smp[j].q;
        synthTileCore<false, kUi>(sp, blockIdx.x, blockIdx.y, [&](int k, int, int, int, uint32_t o) {
            acc[k][0] += q * (o & 255u);
            acc[k][1] += q * ((o >> 8) & 255u);
            acc[k][2] += q * ((o >> 16) & 255u);
        });
        __syncthreads();   // the tile's shared memory and sp are free again
    }
    // the output: the synthesized samples' sums plus the replaced samples' real pixels, rounded once
    const uint32_t wp = sWp, wc = sWc, wap = sWap, wac = 65536u - wap;
    const uint32_t pitch = (uint32_t)b.pitch;
    const int lx = ex - kSyAp, x = blockIdx.x * kSyT + lx;
    if ((unsigned)lx >= (unsigned)kSyT || x >= b.W) return;
#pragma unroll
    for (int k = 0; k < kSyK; k++) {   // the pixels synthTileCore gave this thread's slot k
        const int ly = syOutRow(ey0, k), y = blockIdx.y * kSyTH + ly;
        if (ly >= kSyTH || y >= b.H) break;
        const uint32_t pa = __ldg(reinterpret_cast<const uint32_t*>(b.a + (size_t)y * pitch) + x);
        const uint32_t pc = __ldg(reinterpret_cast<const uint32_t*>(b.c + (size_t)y * pitch) + x);
        uint32_t o = 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const uint32_t v = acc[k][c] + wp * ((pa >> (8 * c)) & 255u) + wc * ((pc >> (8 * c)) & 255u) + 32768u;
            o |= (v >> 16) << (8 * c);
        }
        o |= ((wap * (pa >> 24) + wac * (pc >> 24) + 32768u) >> 16) << 24;
        reinterpret_cast<uint32_t*>(b.out + (size_t)y * b.outPitch)[x] = o;
    }
}

// Many syntheses (of several frame pairs and times) in one persistent launch: every CTA takes the next tile of the
// work list (items in the host's order, each item's tiles in raster order) from an atomic counter until the list is
// exhausted; an item's parameters are staged in shared memory per tile. Mixed sizes balance across the SMs.
__global__ void __launch_bounds__(kSyThreads, 3) k_synth_batch(const SynthBatchArgs b) {
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
        static_assert(sizeof(SynthParams) % 4 == 0, "SynthParams copies as words");
        for (int i = threadIdx.x; i < (int)(sizeof(SynthParams) / 4); i += kSyThreads)
            reinterpret_cast<uint32_t*>(&sp)[i] = __ldg(reinterpret_cast<const uint32_t*>(b.items + it) + i);
        __syncthreads();
        const int t = w - b.tileStart[it], tx = b.tilesX[it];
        synthTile(sp, t % tx, t / tx);
        __syncthreads();   // the tile's shared memory is free again
    }
}

// the untrusted-share decision of many syntheses (grid.y = item), the batched k_fallback (the item counters are
// zeroed by the host before the batch's synth launch)
__global__ void __launch_bounds__(256) k_fallback_batch(const FallbackParams* __restrict__ items) {
    pdlEnter();   // the counters are complete only when the synthesis launch is
    const FallbackParams& p = items[blockIdx.y];
    const unsigned int cnt = *p.untrusted;
    if (!((double)cnt / ((double)p.W * (double)p.H) > p.frac)) return;
    const uint8_t* nearF = p.nearC ? p.c : p.a;
    const size_t n = (size_t)p.W * p.H;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) {
        const int x = (int)(i % p.W), y = (int)(i / p.W);
        reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] =
            __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * p.pitch) + x);
    }
}

// interp.py:238-239: more than globalFallback of the pixels untrusted -> the nearer real frame over the output.
// Every CTA exits at once in the normal case. Also clears the next synth's counter.
__global__ void __launch_bounds__(256) k_fallback(const FallbackParams p) {
    pdlEnter();
    const unsigned int cnt = *p.untrusted;
    if (blockIdx.x == 0 && threadIdx.x == 0) *p.untrustedNext = 0;
    if (!((double)cnt / ((double)p.W * (double)p.H) > p.frac)) return;
    const uint8_t* nearF = p.nearC ? p.c : p.a;
    const size_t n = (size_t)p.W * p.H;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) {
        const int x = (int)(i % p.W), y = (int)(i / p.W);
        reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] =
            __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * p.pitch) + x);
    }
}

// ============================================================================================== launchers
cudaError_t launchLumaPyr(const LumaPyrParams& p, cudaStream_t s) {
    return launchPdl(k_luma_pyr, dim3(divUp(p.lw[0], 32), divUp(p.lh[0], 32)), dim3(256), 0, s, p);
}
cudaError_t launchDown(const DownParams& p, cudaStream_t s) {
    return launchPdl(k_down, dim3(divUp(p.dw, 16), divUp(p.dh, 16)), dim3(256), 0, s, p);
}
template <int R>
static cudaError_t launchSearchR(const SearchParams& p, cudaStream_t s) {
    constexpr int T = 8 + 2 * R, D = 2 * R + 1;
    const dim3 grid(divUp(p.bw * p.bh, 4));
    const size_t smem = (size_t)4 * (2 * T * T + D * D) * sizeof(float);
    if (p.bw * p.bh <= kSearchLatBlocks) return launchPdl(k_search_r<R, true>, grid, dim3(128), smem, s, p);
    return launchPdl(k_search_r<R, false>, grid, dim3(128), smem, s, p);
}
cudaError_t launchSearch(const SearchParams& p, cudaStream_t s) {
    switch (p.R) {
        case 1: return launchSearchR<1>(p, s);
        case 2: return launchSearchR<2>(p, s);
        case 3: return launchSearchR<3>(p, s);
        case 4: return launchSearchR<4>(p, s);
        case 5: return launchSearchR<5>(p, s);
        case 6: return launchSearchR<6>(p, s);
        default: {   // radii 7..12 (settings beyond the defaults): the runtime-radius kernel
            const int T = 8 + 2 * p.R;
            return launchPdl(k_search, dim3(divUp(p.bw * p.bh, 4)), dim3(128), (size_t)4 * 2 * T * T * sizeof(float), s, p);
        }
    }
}
cudaError_t launchMedian3(const Median3Params& p, cudaStream_t s) {
    const int nb = 2 * p.B + 1;
    if (p.doHist && p.bw * p.bh <= kMed1Blocks && nb <= kMed1MaxBins)
        return launchPdl(k_median3_one, dim3(1), dim3(kMed1Threads), (size_t)2 * nb * 4, s, p);
    if (p.doHist && p.bw * p.bh <= kMedClBlocks && nb <= kMed1MaxBins)
        return launchPdl(k_median3_cluster, dim3(kMedCl), dim3(kMed1Threads), (size_t)2 * nb * 4, s, p);
    return launchPdl(k_median3, dim3(divUp(p.bw * p.bh, 256)), dim3(256), 0, s, p);
}
// ---- merged launches: the items' CTA ranges, then one launch (every item of m takes the same kernel variant)
template <class P, class F>
static int layoutMerged(Merged<P>& m, F ctasOf) {   // ctasOf(item, gx&) -> the item's CTA count
    int total = 0;
    for (int i = 0; i < m.n; i++) {
        int gx = 1;
        const int c = ctasOf(m.item[i], gx);
        m.first[i] = total;
        m.gx[i] = gx;
        total += c;
    }
    m.first[m.n] = total;
    return total;
}
cudaError_t launchLumaPyrMerged(Merged<LumaPyrParams>& m, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    const int total = layoutMerged(m, [](const LumaPyrParams& p, int& gx) {
        gx = (int)divUp(p.lw[0], 32);
        return gx * (int)divUp(p.lh[0], 32);
    });
    return launchPdl(k_luma_pyr_m, dim3(total), dim3(256), 0, s, m);
}
int searchVariant(const SearchParams& p) {
    if (p.R >= 1 && p.R <= 6) return 2 * p.R + (p.bw * p.bh <= kSearchLatBlocks ? 1 : 0);
    return 100 + p.R;
}
template <int R>
static cudaError_t launchSearchRMerged(Merged<SearchParams>& m, int total, cudaStream_t s) {
    constexpr int T = 8 + 2 * R, D = 2 * R + 1;
    const size_t smem = (size_t)4 * (2 * T * T + D * D) * sizeof(float);
    if (searchVariant(m.item[0]) & 1) return launchPdl(k_search_r_m<R, true>, dim3(total), dim3(128), smem, s, m);
    return launchPdl(k_search_r_m<R, false>, dim3(total), dim3(128), smem, s, m);
}
cudaError_t launchSearchMerged(Merged<SearchParams>& m, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    const int v = searchVariant(m.item[0]);
    for (int i = 1; i < m.n; i++)
        if (searchVariant(m.item[i]) != v) return cudaErrorInvalidValue;
    const int total = layoutMerged(m, [](const SearchParams& p, int& gx) {
        gx = (int)divUp(p.bw * p.bh, 4);
        return gx;
    });
    switch (m.item[0].R) {
        case 1: return launchSearchRMerged<1>(m, total, s);
        case 2: return launchSearchRMerged<2>(m, total, s);
        case 3: return launchSearchRMerged<3>(m, total, s);
        case 4: return launchSearchRMerged<4>(m, total, s);
        case 5: return launchSearchRMerged<5>(m, total, s);
        case 6: return launchSearchRMerged<6>(m, total, s);
        default: {
            const int T = 8 + 2 * m.item[0].R;
            return launchPdl(k_search_m, dim3(total), dim3(128), (size_t)4 * 2 * T * T * sizeof(float), s, m);
        }
    }
}
int median3Variant(const Median3Params& p) {
    const int nb = 2 * p.B + 1;
    if (p.doHist && p.bw * p.bh <= kMed1Blocks && nb <= kMed1MaxBins) return 0;
    if (p.doHist && p.bw * p.bh <= kMedClBlocks && nb <= kMed1MaxBins) return 1;
    return 2;
}
cudaError_t launchMedian3Merged(Merged<Median3Params>& m, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    const int v = median3Variant(m.item[0]);
    size_t smem = 0;
    for (int i = 0; i < m.n; i++) {
        if (median3Variant(m.item[i]) != v) return cudaErrorInvalidValue;
        smem = std::max(smem, (size_t)2 * (2 * m.item[i].B + 1) * 4);
    }
    if (v == 0) {
        layoutMerged(m, [](const Median3Params&, int& gx) { gx = 1; return 1; });
        return launchPdl(k_median3_one_m, dim3(m.n), dim3(kMed1Threads), smem, s, m);
    }
    if (v == 1) {
        layoutMerged(m, [](const Median3Params&, int& gx) { gx = kMedCl; return kMedCl; });
        return launchPdl(k_median3_cluster_m, dim3(kMedCl * m.n), dim3(kMed1Threads), smem, s, m);
    }
    const int total = layoutMerged(m, [](const Median3Params& p, int& gx) {
        gx = (int)divUp(p.bw * p.bh, 256);
        return gx;
    });
    return launchPdl(k_median3_m, dim3(total), dim3(256), 0, s, m);
}
cudaError_t launchSubpixMerged(Merged<SubpixParams>& m, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    const int total = layoutMerged(m, [](const SubpixParams& p, int& gx) {
        gx = (int)divUp(p.bw * p.bh, 4);
        return gx;
    });
    return launchPdl(k_subpix_m, dim3(total), dim3(128), (size_t)4 * kSubWarpFloats * sizeof(float), s, m);
}
cudaError_t launchPixfieldMerged(Merged<PixfieldParams>& m, cudaStream_t s) {
    if (m.n < 1 || m.n > kMergeMax) return cudaErrorInvalidValue;
    const int total = layoutMerged(m, [](const PixfieldParams& p, int& gx) {
        gx = (int)divUp(p.w, kPfTW);
        return gx * (int)divUp(p.h, kPfTH);
    });
    return launchPdl(k_pixfield_m, dim3(total), dim3(256), 0, s, m);
}
static size_t planBytes(const CutPlan& c) {
    const size_t b = (size_t)(c.nLeaves + c.nInner) * sizeof(float);
    return b <= kPlanSmemMax ? b : 0;   // 0: the node values live in c.gvals
}
cudaError_t prepareKernels() {
    cudaError_t e = cudaFuncSetAttribute(k_subpix, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlanSmemMax);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_median3_one, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kMed1MaxBins * 4);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_median3_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kMed1MaxBins * 4);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_cutmean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlanSmemMax);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_subpix_m, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlanSmemMax);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_median3_one_m, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kMed1MaxBins * 4);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_median3_cluster_m, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kMed1MaxBins * 4);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(synthSmemBytes(1) + kSyWarpBytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(synthSmemBytes(1) + kSyWarpBytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_t<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(synthSmemBytes(1) + kSyWarpBytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_blur_t<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(synthSmemBytes(1) + kSyWarpBytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_synth_ui, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(synthSmemBytes(1) + kSyWarpBytes));
    return e;
}
cudaError_t launchSubpix(const SubpixParams& p, cudaStream_t s) {
    const size_t smem = (size_t)4 * kSubWarpFloats * sizeof(float);
    return launchPdl(k_subpix, dim3(divUp(p.bw * p.bh, 4)), dim3(128), smem, s, p);
}
cudaError_t launchCutMean(const CutMeanParams& p, cudaStream_t s) {
    return launchPdl(k_cutmean, dim3(1), dim3(256), planBytes(p.plan), s, p);
}
cudaError_t launchPixfield(const PixfieldParams& p, cudaStream_t s) {
    return launchPdl(k_pixfield, dim3(divUp(p.w, kPfTW), divUp(p.h, kPfTH)), dim3(256), 0, s, p);
}
size_t synthSmemBytes(int fs) {  // declared in fg_params.h
    // worst-case field region of a tile (GW x GH float2) + its horizontal stage + mismatch + row sums
    const int gw = (kSyE + fs - 1) / fs + 3, gh = (kSyEH + fs - 1) / fs + 3;
    return (size_t)gw * gh * 8 + (size_t)gh * kSyE * 8 + (size_t)kSyEH * kSyES + (size_t)kSyEH * kSyHS * 2;
}
size_t synthKernelSmem(int fs) { return synthSmemBytes(fs) + kSyWarpBytes; }
int synthTilesX(int W) { return (int)divUp(W, kSyT); }
int synthTilesY(int H) { return (int)divUp(H, kSyTH); }
cudaError_t launchSynth(const SynthParams& p, cudaStream_t s) {
    const size_t smem = synthSmemBytes(p.fs) + kSyWarpBytes;
    const dim3 grid(divUp(p.W, kSyT), divUp(p.H, kSyTH));
    if (p.uiA || p.uiC) return launchPdl(k_synth_ui, grid, dim3(kSyThreads), smem, s, p);
    return launchPdl(k_synth, grid, dim3(kSyThreads), smem, s, p);
}
cudaError_t launchSynthBlur(const BlurParams& bp, int fix, cudaStream_t s) {
    const size_t smem = synthSmemBytes(bp.base.fs) + kSyWarpBytes;
    const dim3 grid(divUp(bp.base.W, kSyT), divUp(bp.base.H, kSyTH));
    BlurParams p = bp;
    p.fix = fix;
    if (p.base.uiA || p.base.uiC) return launchPdl(k_synth_blur_t<true>, grid, dim3(kSyThreads), smem, s, p);
    return launchPdl(k_synth_blur_t<false>, grid, dim3(kSyThreads), smem, s, p);
}
cudaError_t launchSynthBatch(const SynthBatchArgs& b, int grid, size_t smem, cudaStream_t s) {
    return launchPdl(k_synth_batch, dim3(grid), dim3(kSyThreads), smem, s, b);
}
int synthBatchCtasPerSm(size_t smem) {   // resident k_synth_batch CTAs per SM with this dynamic shared memory
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_synth_batch, kSyThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ;
}
cudaError_t launchFallbackBatch(const FallbackParams* items, int nItems, cudaStream_t s) {
    return launchPdl(k_fallback_batch, dim3(smCount(), nItems), dim3(256), 0, s, items);
}
cudaError_t launchFallback(const FallbackParams& p, cudaStream_t s) {
    return launchPdl(k_fallback, dim3(smCount() * 4), dim3(256), 0, s, p);
}

int smCount() {
    constexpr int kDevices = 64;
    static std::atomic<int> cached[kDevices];   // 0: not queried yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
        cudaGetLastError();
        return 148;   // the grid-stride kernels stay correct with any grid; B200's count is a fair size
    }
    int n = cached[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return 148;
    }
    cached[dev].store(n, std::memory_order_relaxed);
    return n;
}

}  // namespace fgk
