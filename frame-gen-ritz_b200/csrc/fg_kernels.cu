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
#include <cfloat>
#include <cstdint>

#include "fg_params.h"

namespace fgk {

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

__device__ __forceinline__ float warpSum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ============================================================================================== luma + pyramid
// interp.flow :149-152 + interp.pyramid :73-77. One CTA = a 32x32 tile of level 0 (32 fs x 32 fs frame pixels) and
// the aligned 16x16 .. 1x1 tiles of levels 1..5 above it: a level-(l+1) pixel only averages the 2x2 level-l pixels
// below it, so the whole tower stays inside the tile. Mean of the valid pixels: sum * 1/n^2 when full, sum / count
// at the frame's odd edges (cv2's INTER_AREA fast path).
__global__ void __launch_bounds__(256) k_luma_pyr(const LumaPyrParams p) {
    __shared__ float sl[2][1024 + 256 + 64 + 16 + 4 + 1];
    const int tx0 = blockIdx.x * 32, ty0 = blockIdx.y * 32;
    const int fw = p.lw[0], fh = p.lh[0], fs = p.fs;
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
    __syncthreads();
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

// a pyramid level beyond the luma kernel's tower (interp.py:76)
__global__ void __launch_bounds__(256) k_down(const DownParams p) {
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
    p.da[(size_t)y * p.dw + x] = n == 4 ? __fmul_rn(sa, 0.25f) : __fdiv_rn(sa, (float)n);
    p.dc[(size_t)y * p.dw + x] = n == 4 ? __fmul_rn(sc, 0.25f) : __fdiv_rn(sc, (float)n);
}

// ============================================================================================== seed + search
// interp.seed_from :131-144 and interp.search :116-124 at integer steps, one warp per 8x8 block.
// Seed: own parent, the 3 nearest other parents, zero, the global median (all 2x the parent level's vectors),
// scored by block SAD + (0 for own, lambda otherwise); the first minimum wins.
// Search: every integer offset within +-R of the seed; the (8+2R)^2 windows of a and c (bilateral: a at q - v, c at
// q + v) are staged in shared memory; lane i scores candidates i, i+32, ...; cost = SAD + lambda |d|_1; the warp
// keeps the lowest (cost, raster index) pair, i.e. the first minimum in interp's (dy, dx) order.
__global__ void __launch_bounds__(128) k_search(const SearchParams p) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * 4 + warp;
    if (b >= p.bw * p.bh) return;
    const int R = p.R, T = 8 + 2 * R, D = 2 * R + 1;
    float* sA = smem + warp * 2 * T * T;
    float* sC = sA + T * T;
    const int bx = b % p.bw, by = b / p.bw, b0x = bx * kBlock, b0y = by * kBlock;
    int sx = 0, sy = 0;
    if (!p.top) {
        const int px = min(bx >> 1, p.pw - 1), py = min(by >> 1, p.ph - 1);
        const int oy = (by & 1) ? 1 : -1, ox = (bx & 1) ? 1 : -1;
        const int qx = b0x + (lane & 7), qy0 = b0y + (lane >> 3), qy1 = qy0 + 4;
        float best = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            int cx = 0, cy = 0;   // own, (0, oy), (ox, 0), (ox, oy) parents x 2; zero; the global median
            if (k < 4) {
                const int dx = (k & 2) ? ox : 0, dy = (k & 1) ? oy : 0;
                const float2 v = p.parent[clampi(py + dy, 0, p.ph - 1) * p.pw + clampi(px + dx, 0, p.pw - 1)];
                cx = 2 * __float2int_rn(v.x);
                cy = 2 * __float2int_rn(v.y);
            } else if (k == 5) {
                cx = __float2int_rn(p.med[0]);
                cy = __float2int_rn(p.med[1]);
            }
            float s = fabsf(Lc(p.la, p.w, p.h, qx - cx, qy0 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy0 + cy));
            s += fabsf(Lc(p.la, p.w, p.h, qx - cx, qy1 - cy) - Lc(p.lc, p.w, p.h, qx + cx, qy1 + cy));
            s = warpSum(s);   // exact: at most 24 significant bits
            float cost = __fmul_rn(s, 1.0f / 64.0f);
            if (k > 0) cost = __fadd_rn(cost, p.lambda);
            if (k == 0 || cost < best) { best = cost; sx = cx; sy = cy; }
        }
    }
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
__global__ void __launch_bounds__(256) k_median3(const Median3Params p) {
    const int b = blockIdx.x * 256 + threadIdx.x;
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
    if (ticket != gridDim.x - 1) return;
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
// two shared loads per pixel. The last CTA computes the scene-cut mean of the winners' SADs.
constexpr int kSubT = 13, kSubO = 2, kSubL = 24, kSubRows = 10;   // tile, its margin, lattice side, tile rows used
constexpr int kSubWarpFloats = 2 * kSubT * kSubT + 2 * kSubRows * kSubL + 2 * kSubL * kSubL + 72;

__global__ void __launch_bounds__(128) k_subpix(const SubpixParams p) {
    extern __shared__ float smem[];
    __shared__ unsigned int ticket;
    __shared__ unsigned int red[128];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * 4 + warp;
    const int nb = p.bw * p.bh;
    if (b < nb) {
        float* tA = smem + warp * kSubWarpFloats;
        float* tC = tA + kSubT * kSubT;
        float* hA = tC + kSubT * kSubT;      // kSubRows x kSubL: tile rows 1..10 sampled at the lattice columns
        float* hC = hA + kSubRows * kSubL;
        float* qA = hC + kSubRows * kSubL;   // kSubL x kSubL lattice
        float* qC = qA + kSubL * kSubL;
        float* rows = qC + kSubL * kSubL;
        const int bx = b % p.bw, by = b / p.bw, b0x = bx * kBlock, b0y = by * kBlock;
        const float2 v0 = p.in[b];
        const int sx = __float2int_rn(v0.x), sy = __float2int_rn(v0.y);
        for (int i = lane; i < kSubT * kSubT; i += 32) {
            const int x = i % kSubT, y = i / kSubT;
            tA[i] = Lc(p.la, p.w, p.h, b0x - sx - kSubO + x, b0y - sy - kSubO + y);
            tC[i] = Lc(p.lc, p.w, p.h, b0x + sx - kSubO + x, b0y + sy - kSubO + y);
        }
        __syncwarp();
        int b4x = 0, b4y = 0;   // the offset chosen so far, quarter pixels
        float sadBest = 0.0f;
        for (int pass = 0; pass < 2; pass++) {
            const int s4 = pass ? 1 : 2;
            // horizontal stage: a at tile x + 2 - o, c at x + 2 + o, o = (b4x + s4 d) / 4, lattice column u = 3x + d + 1
            for (int it = lane; it < kSubRows * kSubL; it += 32) {
                const int r = it / kSubL + 1, u = it % kSubL, x = u / 3, d = u % 3 - 1;
                const int PA = 4 * (x + kSubO) - (b4x + s4 * d), PC = 4 * (x + kSubO) + (b4x + s4 * d);
                const float fa = (float)(PA & 3) * 0.25f, fc = (float)(PC & 3) * 0.25f;
                const float* ra = tA + r * kSubT + (PA >> 2);
                const float* rc = tC + r * kSubT + (PC >> 2);
                hA[it] = __fmaf_rn(ra[1], fa, __fmul_rn(ra[0], 1.0f - fa));   // exact: dyadic, <= 16 significant bits
                hC[it] = __fmaf_rn(rc[1], fc, __fmul_rn(rc[0], 1.0f - fc));
            }
            __syncwarp();
            // vertical stage: lattice row v = 3y + d + 1
            for (int it = lane; it < kSubL * kSubL; it += 32) {
                const int v = it / kSubL, u = it % kSubL, y = v / 3, d = v % 3 - 1;
                const int PA = 4 * (y + kSubO) - (b4y + s4 * d), PC = 4 * (y + kSubO) + (b4y + s4 * d);
                const float fa = (float)(PA & 3) * 0.25f, fc = (float)(PC & 3) * 0.25f;
                const float* ca = hA + ((PA >> 2) - 1) * kSubL + u;
                const float* cc = hC + ((PC >> 2) - 1) * kSubL + u;
                qA[it] = __fmaf_rn(ca[kSubL], fa, __fmul_rn(ca[0], 1.0f - fa));
                qC[it] = __fmaf_rn(cc[kSubL], fc, __fmul_rn(cc[0], 1.0f - fc));
            }
            __syncwarp();
            // (candidate, row) partial sums: candidate k = (dy + 1) * 3 + (dx + 1)
            for (int it = lane; it < 72; it += 32) {
                const int k = it >> 3, y = it & 7, dx = k % 3, dy = k / 3;
                const float* ra = qA + (3 * y + dy) * kSubL + dx;
                const float* rc = qC + (3 * y + dy) * kSubL + dx;
                float sum = 0.0f;
#pragma unroll
                for (int x = 0; x < 8; x++) sum += fabsf(ra[3 * x] - rc[3 * x]);
                rows[it] = sum;
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
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) ticket = atomicAdd(&p.st->subDone, 1u);
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    const bool inSmem = (size_t)(p.plan.nLeaves + p.plan.nInner) * sizeof(float) <= kPlanSmemMax;
    cutMeanBlock(p.sads, nb, p.plan, p.cutSad, p.st, inSmem ? smem : p.plan.gvals, red);
    if (threadIdx.x == 0) p.st->subDone = 0;
}

// ============================================================================================== per-pixel field
// interp.pixel_field :167-183 at flow resolution. Candidates per pixel: the bilinear block field (cv2.resize x8,
// INTER_LINEAR), the own block, the blocks above / below / left / right (edge-clamped), zero. Each candidate's cost
// is the 5x5 replicate-border box of |a(q - h) - c(q + h)| where every window pixel uses its own candidate (cv2.blur
// over the per-candidate error image). Tile 32x16 + 2 px apron; the errors are exact multiples of 2^-14, so they
// are summed as int32 and the mean is formed in double as cv2's box filter does (sum * (1/25), then to float).
constexpr int kPfTW = 32, kPfTH = 16, kPfAp = 2, kPfEW = kPfTW + 2 * kPfAp, kPfEH = kPfTH + 2 * kPfAp, kPfNC = 7;

__device__ __forceinline__ float2 blockV(const float2* __restrict__ v, int bw, int bh, int bx, int by) {
    return __ldg(v + clampi(by, 0, bh - 1) * bw + clampi(bx, 0, bw - 1));
}

// cv2.resize INTER_LINEAR coefficient along one axis for a x8 upscale; clampw: the x rule (weights (1, 0) beyond the
// border), else the y rule (rows clamped, weights kept)
__device__ __forceinline__ void linCoef8(int d, int n, bool clampw, int& i0, int& i1, float& a0, float& a1) {
    float f = __fsub_rn(__fmul_rn((float)d + 0.5f, 0.125f), 0.5f);
    int s = (int)floorf(f);
    f = __fsub_rn(f, (float)s);
    if (clampw) {
        if (s < 0) { s = 0; f = 0.0f; }
        if (s >= n - 1) { s = n - 1; f = 0.0f; }
    }
    i0 = clampi(s, 0, n - 1);
    i1 = clampi(s + 1, 0, n - 1);
    a0 = 1.0f - f;
    a1 = f;
}

__device__ __forceinline__ float2 pfCand(const PixfieldParams& p, int k, int qx, int qy) {
    const int bx = qx >> 3, by = qy >> 3;
    switch (k) {
        case 0: {
            int x0, x1, y0, y1;
            float a0, a1, b0, b1;
            linCoef8(qx, p.bw, true, x0, x1, a0, a1);
            linCoef8(qy, p.bh, false, y0, y1, b0, b1);
            const float2 v00 = blockV(p.v, p.bw, p.bh, x0, y0), v01 = blockV(p.v, p.bw, p.bh, x1, y0);
            const float2 v10 = blockV(p.v, p.bw, p.bh, x0, y1), v11 = blockV(p.v, p.bw, p.bh, x1, y1);
            const float h0x = __fadd_rn(__fmul_rn(v00.x, a0), __fmul_rn(v01.x, a1)), h0y = __fadd_rn(__fmul_rn(v00.y, a0), __fmul_rn(v01.y, a1));
            const float h1x = __fadd_rn(__fmul_rn(v10.x, a0), __fmul_rn(v11.x, a1)), h1y = __fadd_rn(__fmul_rn(v10.y, a0), __fmul_rn(v11.y, a1));
            return make_float2(__fadd_rn(__fmul_rn(h0x, b0), __fmul_rn(h1x, b1)), __fadd_rn(__fmul_rn(h0y, b0), __fmul_rn(h1y, b1)));
        }
        case 1: return blockV(p.v, p.bw, p.bh, bx, by);
        case 2: return blockV(p.v, p.bw, p.bh, bx, by - 1);
        case 3: return blockV(p.v, p.bw, p.bh, bx, by + 1);
        case 4: return blockV(p.v, p.bw, p.bh, bx - 1, by);
        case 5: return blockV(p.v, p.bw, p.bh, bx + 1, by);
        default: return make_float2(0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(256) k_pixfield(const PixfieldParams p) {
    __shared__ int err[kPfNC][kPfEH * kPfEW];
    __shared__ int hs[kPfNC][kPfEH * kPfTW];
    const int tx0 = blockIdx.x * kPfTW - kPfAp, ty0 = blockIdx.y * kPfTH - kPfAp;
    for (int i = threadIdx.x; i < kPfEH * kPfEW; i += 256) {
        const int qx = clampi(tx0 + i % kPfEW, 0, p.w - 1), qy = clampi(ty0 + i / kPfEW, 0, p.h - 1);
        const float fx = (float)qx, fy = (float)qy;
#pragma unroll
        for (int k = 0; k < kPfNC; k++) {
            const float2 v = pfCand(p, k, qx, qy);
            const float e = fabsf(remapF(p.ya, p.w, p.h, __fsub_rn(fx, v.x), __fsub_rn(fy, v.y)) -
                                  remapF(p.yc, p.w, p.h, __fadd_rn(fx, v.x), __fadd_rn(fy, v.y)));
            err[k][i] = __float2int_rn(__fmul_rn(e, 16384.0f));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPfEH * kPfTW; i += 256) {
        const int r = i / kPfTW, c = i % kPfTW;
#pragma unroll
        for (int k = 0; k < kPfNC; k++) {
            const int* e = err[k] + r * kPfEW + c;
            hs[k][i] = e[0] + e[1] + e[2] + e[3] + e[4];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPfTW * kPfTH; i += 256) {
        const int lx = i % kPfTW, ly = i / kPfTW;
        const int qx = blockIdx.x * kPfTW + lx, qy = blockIdx.y * kPfTH + ly;
        if (qx >= p.w || qy >= p.h) continue;
        float best = 0.0f;
        int bk = 0;
#pragma unroll
        for (int k = 0; k < kPfNC; k++) {
            const int* h = hs[k] + ly * kPfTW + lx;
            const int S = h[0] + h[kPfTW] + h[2 * kPfTW] + h[3 * kPfTW] + h[4 * kPfTW];
            float c = (float)(((double)S * 0x1p-14) * (1.0 / 25.0));
            if (k == 0) c = __fsub_rn(c, p.smooth);
            if (k == kPfNC - 1) c = __fsub_rn(c, p.zero);
            if (k == 0 || c < best) { best = c; bk = k; }
        }
        p.pf[(size_t)qy * p.w + qx] = pfCand(p, bk, qx, qy);
    }
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
constexpr int kSyTW = 64, kSyTH = 32, kSyAp = 3, kSyEW = kSyTW + 2 * kSyAp, kSyEH = kSyTH + 2 * kSyAp;

// round-half-even(x * 32) for |x * 32| < 2^22 (cv2's saturate_cast<int>(x * INTER_TAB_SIZE))
__device__ __forceinline__ int rne32(float x) { return __float_as_int(__fmaf_rn(x, 32.0f, 12582912.0f)) - 0x4B400000; }
// exact float of 0 <= i < 2^23
__device__ __forceinline__ float i2f(int i) { return __int_as_float(0x4B000000 | i) - 8388608.0f; }
// floor of 0 <= v < 2^23
__device__ __forceinline__ int floorPos(float v) { return __float_as_int(__fadd_rz(v, 8388608.0f)) - 0x4B000000; }

// cv2.remap INTER_LINEAR / BORDER_REPLICATE of the 2-channel float field, conversions on the FP32 pipe
__device__ __forceinline__ float2 remapF2m(const float2* __restrict__ F, int w, int h, float x, float y) {
    const int X = rne32(x), Y = rne32(y);
    const int ix = X >> 5, iy = Y >> 5;
    const float fx = i2f(X & 31) * (1.0f / 32.0f), fy = i2f(Y & 31) * (1.0f / 32.0f);
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

// one cv2.remap INTER_LINEAR / BORDER_REPLICATE sample of a 4-byte-per-pixel 8-bit frame: channels 0..2 of the
// result (byte 3 = 0). Horizontal stage two channels per multiply (lanes of 16 bits hold at most 255 * 32), vertical
// stage per channel; (v + 512) >> 10 == cv2's (32 v + 2^14) >> 15 with its 15-bit weights.
__device__ __forceinline__ uint32_t sampleU8(const uint8_t* __restrict__ img, uint32_t pitch, int W, int H, float x, float y) {
    const int X = rne32(x), Y = rne32(y);
    const int ix = X >> 5, iy = Y >> 5;
    const uint32_t fx = (uint32_t)X & 31u, fy = (uint32_t)Y & 31u;
    uint32_t o00, o01, o10, o11;
    if ((unsigned)ix < (unsigned)(W - 1) && (unsigned)iy < (unsigned)(H - 1)) {
        o00 = (uint32_t)iy * pitch + (uint32_t)ix * 4u;
        o01 = o00 + 4u;
        o10 = o00 + pitch;
        o11 = o10 + 4u;
    } else {
        const uint32_t x0 = (uint32_t)clampi(ix, 0, W - 1) * 4u, x1 = (uint32_t)clampi(ix + 1, 0, W - 1) * 4u;
        const uint32_t r0 = (uint32_t)clampi(iy, 0, H - 1) * pitch, r1 = (uint32_t)clampi(iy + 1, 0, H - 1) * pitch;
        o00 = r0 + x0; o01 = r0 + x1; o10 = r1 + x0; o11 = r1 + x1;
    }
    const uint32_t p00 = __ldg(reinterpret_cast<const uint32_t*>(img + o00));
    const uint32_t p01 = __ldg(reinterpret_cast<const uint32_t*>(img + o01));
    const uint32_t p10 = __ldg(reinterpret_cast<const uint32_t*>(img + o10));
    const uint32_t p11 = __ldg(reinterpret_cast<const uint32_t*>(img + o11));
    const uint32_t M = 0x00FF00FFu, wx0 = 32u - fx, wy0 = 32u - fy;
    const uint32_t rb0 = (p00 & M) * wx0 + (p01 & M) * fx, rb1 = (p10 & M) * wx0 + (p11 & M) * fx;
    const uint32_t g0 = __byte_perm(p00, 0, 0x4441) * wx0 + __byte_perm(p01, 0, 0x4441) * fx;
    const uint32_t g1 = __byte_perm(p10, 0, 0x4441) * wx0 + __byte_perm(p11, 0, 0x4441) * fx;
    const uint32_t c0 = ((rb0 & 0xFFFFu) * wy0 + (rb1 & 0xFFFFu) * fy + 512u) >> 10;
    const uint32_t c2 = ((rb0 >> 16) * wy0 + (rb1 >> 16) * fy + 512u) >> 10;
    const uint32_t c1 = (g0 * wy0 + g1 * fy + 512u) >> 10;
    return c0 | (c1 << 8) | (c2 << 16);
}

struct SyCoef {   // one output column (or row) of the tile + halo: the upsampling taps and weights, the coordinate
    int i0, i1;   // flow taps relative to the tile's field region
    float a0, a1; // weights (rows: already x fs, which commutes with the rounding)
    float pos;    // the clamped pixel coordinate as a float
    int pi;       // ... as an int
};

__device__ __forceinline__ SyCoef syCoef(int e, int origin, int n, int un, int fn, int g0, float invfs, float fsf, bool xaxis) {
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
    c.a0 = __fmul_rn(1.0f - f, fsf);
    c.a1 = __fmul_rn(f, fsf);
    c.pos = (float)p;
    c.pi = p;
    return c;
}

__global__ void __launch_bounds__(256) k_synth(const SynthParams p) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ SyCoef colc[kSyEW], rowc[kSyEH];
    __shared__ float TA[256], TC[256];
    __shared__ unsigned int cnt;
    __shared__ int gReg[4];
    const int X0 = blockIdx.x * kSyTW, Y0 = blockIdx.y * kSyTH;
    const uint8_t* nearF = p.nearC ? p.c : p.a;
    const uint32_t pitch = (uint32_t)p.pitch;
    if (p.st->cut) {   // scene cut (interp.py:225-226): the nearer real frame
        for (int i = threadIdx.x; i < kSyTW * kSyTH; i += 256) {
            const int x = X0 + (i % kSyTW), y = Y0 + (i / kSyTW);
            if (x < p.W && y < p.H)
                reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] =
                    __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * pitch) + x);
        }
        return;
    }
    const int fs = p.fs, uw = p.fw * fs, uh = p.fh * fs;
    const float invfs = 1.0f / (float)fs, fsf = (float)fs;
    // 0. the field region of the tile + halo, the coefficient tables, the blend products
    if (threadIdx.x == 0) {
        const SyCoef lo = syCoef(0, X0, p.W, uw, p.fw, 0, invfs, 1.0f, true);
        const SyCoef hi = syCoef(kSyEW - 1, X0, p.W, uw, p.fw, 0, invfs, 1.0f, true);
        const SyCoef rlo = syCoef(0, Y0, p.H, uh, p.fh, 0, invfs, 1.0f, false);
        const SyCoef rhi = syCoef(kSyEH - 1, Y0, p.H, uh, p.fh, 0, invfs, 1.0f, false);
        gReg[0] = lo.i0; gReg[1] = hi.i1 - lo.i0 + 1; gReg[2] = rlo.i0; gReg[3] = rhi.i1 - rlo.i0 + 1;
        cnt = 0;
    }
    __syncthreads();
    const int gx0 = gReg[0], GW = gReg[1], gy0 = gReg[2], GH = gReg[3];
    for (int i = threadIdx.x; i < kSyEW + kSyEH; i += 256) {
        if (i < kSyEW) colc[i] = syCoef(i, X0, p.W, uw, p.fw, gx0, invfs, 1.0f, true);
        else rowc[i - kSyEW] = syCoef(i - kSyEW, Y0, p.H, uh, p.fh, gy0, invfs, fsf, false);
    }
    TA[threadIdx.x] = __fmul_rn(p.wA, (float)threadIdx.x);
    TC[threadIdx.x] = __fmul_rn(p.wC, (float)threadIdx.x);
    float2* g = reinterpret_cast<float2*>(sm);                                     // GH x GW
    float2* hrow = g + GW * GH;                                                    // GH x kSyEW
    uint2* wab = reinterpret_cast<uint2*>(hrow + GH * kSyEW);                      // kSyTH x kSyTW
    uint8_t* e = reinterpret_cast<uint8_t*>(wab + kSyTW * kSyTH);                  // kSyEH x kSyEW
    unsigned short* hsum = reinterpret_cast<unsigned short*>(e + ((kSyEH * kSyEW + 15) & ~15));   // kSyEH x kSyTW
    // 1. the field at t on the region (interp.field_at: g <- pf(q - s g), twice, from g = pf(q))
    for (int i = threadIdx.x; i < GW * GH; i += 256) {
        const int qx = gx0 + i % GW, qy = gy0 + i / GW;
        float2 v = __ldg(p.pf + (size_t)qy * p.fw + qx);
        if (p.lookup) {
            const float fx = (float)qx, fy = (float)qy;
#pragma unroll
            for (int it = 0; it < 2; it++)
                v = remapF2m(p.pf, p.fw, p.fh, __fsub_rn(fx, __fmul_rn(p.s, v.x)), __fsub_rn(fy, __fmul_rn(p.s, v.y)));
        }
        g[i] = v;
    }
    __syncthreads();
    // 1b. horizontal stage of the upsampling on the region's rows (cv2 resize: h = S0 a0 + S1 a1 per row)
    for (int i = threadIdx.x; i < GH * kSyEW; i += 256) {
        const int r = i / kSyEW, ex = i % kSyEW;
        const SyCoef c = colc[ex];
        const float2 s0 = g[r * GW + c.i0], s1 = g[r * GW + c.i1];
        hrow[i] = make_float2(__fadd_rn(__fmul_rn(s0.x, c.a0), __fmul_rn(s1.x, c.a1)),
                              __fadd_rn(__fmul_rn(s0.y, c.a0), __fmul_rn(s1.y, c.a1)));
    }
    __syncthreads();
    // 2. per pixel of tile + halo: half-vector (vertical stage, x fs folded into the row weights), both warps, mismatch
    for (int i = threadIdx.x; i < kSyEW * kSyEH; i += 256) {
        const int ex = i % kSyEW, ey = i / kSyEW;
        const SyCoef cx = colc[ex], cy = rowc[ey];
        const float2 h0 = hrow[cy.i0 * kSyEW + ex], h1 = hrow[cy.i1 * kSyEW + ex];
        const float hx = __fadd_rn(__fmul_rn(h0.x, cy.a0), __fmul_rn(h1.x, cy.a1));
        const float hy = __fadd_rn(__fmul_rn(h0.y, cy.a0), __fmul_rn(h1.y, cy.a1));
        float ax, ay, bx, by;
        if (p.mid) {
            ax = __fsub_rn(cx.pos, hx); ay = __fsub_rn(cy.pos, hy);
            bx = __fadd_rn(cx.pos, hx); by = __fadd_rn(cy.pos, hy);
        } else {
            ax = __fsub_rn(cx.pos, __fmul_rn(p.ka, hx)); ay = __fsub_rn(cy.pos, __fmul_rn(p.ka, hy));
            bx = __fadd_rn(cx.pos, __fmul_rn(p.kc, hx)); by = __fadd_rn(cy.pos, __fmul_rn(p.kc, hy));
        }
        const uint32_t wa = sampleU8(p.a, pitch, p.W, p.H, ax, ay);
        const uint32_t wc = sampleU8(p.c, pitch, p.W, p.H, bx, by);
        const uint32_t d = __vabsdiffu4(wa, wc);
        const uint32_t m = __vmaxu4(__vmaxu4(d, d >> 8), d >> 16);
        e[i] = (uint8_t)(m & 255u);
        const int lx = ex - kSyAp, ly = ey - kSyAp;
        if ((unsigned)lx < (unsigned)kSyTW && (unsigned)ly < (unsigned)kSyTH) wab[ly * kSyTW + lx] = make_uint2(wa, wc);
    }
    __syncthreads();
    // 3. horizontal 7-sums, a running window over 16 columns per item
    for (int it = threadIdx.x; it < kSyEH * (kSyTW / 16); it += 256) {
        const int r = it / (kSyTW / 16), c0 = (it % (kSyTW / 16)) * 16;
        const uint8_t* q = e + r * kSyEW + c0;
        unsigned int sum = q[0] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6];
        unsigned short* o = hsum + r * kSyTW + c0;
        o[0] = (unsigned short)sum;
#pragma unroll
        for (int c = 1; c < 16; c++) {
            sum += q[c + 6] - q[c - 1];
            o[c] = (unsigned short)sum;
        }
    }
    __syncthreads();
    // 4. vertical 7-sums (a running window down 8 rows per thread), trust, blend, store
    unsigned int myCnt = 0;
    {
        const int lx = threadIdx.x % kSyTW, ly0 = (threadIdx.x / kSyTW) * (kSyTH / 4);
        const int x = X0 + lx;
        const unsigned short* q = hsum + ly0 * kSyTW + lx;
        int S = q[0] + q[kSyTW] + q[2 * kSyTW] + q[3 * kSyTW] + q[4 * kSyTW] + q[5 * kSyTW];
        for (int k = 0; k < kSyTH / 4; k++) {
            const int ly = ly0 + k, y = Y0 + ly;
            S += q[(k + 6) * kSyTW];
            const int Sk = S;
            S -= q[k * kSyTW];
            if (x >= p.W || y >= p.H) continue;
            const uint2 w = wab[ly * kSyTW + lx];
            const uint32_t nq = __ldg(reinterpret_cast<const uint32_t*>(nearF + (size_t)y * pitch) + x);
            uint32_t o;
            if (Sk <= p.sZero) {   // u = 0: out = the blend rounded
                if (p.mid) {
                    o = __vavgu4(w.x, w.y);   // floor(0.5 (a + c) + 0.5) per byte
                } else {
                    o = 0;
#pragma unroll
                    for (int k2 = 0; k2 < 3; k2++) {
                        const float mix = __fadd_rn(TA[(w.x >> (8 * k2)) & 255u], TC[(w.y >> (8 * k2)) & 255u]);
                        o |= (uint32_t)floorPos(fminf(__fadd_rn(mix, 0.5f), 255.0f)) << (8 * k2);
                    }
                }
            } else if (Sk >= p.sOne) {   // u = 1: the nearer frame
                o = nq;
                myCnt++;
            } else {
                const float eb = (float)((double)Sk * (1.0 / 49.0));   // cv2.blur: double sum * (1/49), to float
                float u = __fdiv_rn(__fsub_rn(eb, p.trust0), p.trustSpan);
                u = fminf(fmaxf(u, 0.0f), 1.0f);
                myCnt += u > 0.5f;
                const float iu = 1.0f - u;
                o = 0;
#pragma unroll
                for (int k2 = 0; k2 < 3; k2++) {
                    const int sh = 8 * k2;
                    const uint32_t ca = (w.x >> sh) & 255u, cc = (w.y >> sh) & 255u;
                    const float fa = i2f((int)ca), fc = i2f((int)cc), fn = i2f((int)((nq >> sh) & 255u));
                    const float mix = p.mid ? __fmul_rn(0.5f, __fadd_rn(fa, fc)) : __fadd_rn(TA[ca], TC[cc]);
                    const float v = __fadd_rn(__fadd_rn(__fmul_rn(mix, iu), __fmul_rn(fn, u)), 0.5f);
                    o |= (uint32_t)floorPos(fminf(fmaxf(v, 0.0f), 255.0f)) << sh;
                }
            }
            o = (o & 0x00FFFFFFu) | (nq & 0xFF000000u);   // alpha (byte 3 in both pixel orders): the nearer frame's
            reinterpret_cast<uint32_t*>(p.out + (size_t)y * p.outPitch)[x] = o;
            if (p.emap) p.emap[(size_t)y * ((p.W + 3) & ~3) + x] = e[(ly + kSyAp) * kSyEW + lx + kSyAp];
        }
    }
    if (myCnt) atomicAdd(&cnt, myCnt);
    __syncthreads();
    if (threadIdx.x == 0 && cnt) atomicAdd(p.untrusted, cnt);
}

// interp.py:238-239: more than globalFallback of the pixels untrusted -> the nearer real frame over the output.
// Every CTA exits at once in the normal case. Also clears the next synth's counter.
__global__ void __launch_bounds__(256) k_fallback(const FallbackParams p) {
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
static inline unsigned int divUp(int a, int b) { return (unsigned int)((a + b - 1) / b); }

cudaError_t launchLumaPyr(const LumaPyrParams& p, cudaStream_t s) {
    k_luma_pyr<<<dim3(divUp(p.lw[0], 32), divUp(p.lh[0], 32)), 256, 0, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchDown(const DownParams& p, cudaStream_t s) {
    k_down<<<dim3(divUp(p.dw, 16), divUp(p.dh, 16)), 256, 0, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchSearch(const SearchParams& p, cudaStream_t s) {
    const int T = 8 + 2 * p.R;
    const size_t smem = (size_t)4 * 2 * T * T * sizeof(float);
    k_search<<<divUp(p.bw * p.bh, 4), 128, smem, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchMedian3(const Median3Params& p, cudaStream_t s) {
    k_median3<<<divUp(p.bw * p.bh, 256), 256, 0, s>>>(p);
    return cudaGetLastError();
}
static size_t planBytes(const CutPlan& c) {
    const size_t b = (size_t)(c.nLeaves + c.nInner) * sizeof(float);
    return b <= kPlanSmemMax ? b : 0;   // 0: the node values live in c.gvals
}
cudaError_t prepareKernels() {
    cudaError_t e = cudaFuncSetAttribute(k_subpix, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlanSmemMax);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_cutmean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlanSmemMax);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)synthSmemBytes(1));
    return e;
}
cudaError_t launchSubpix(const SubpixParams& p, cudaStream_t s) {
    const size_t tiles = (size_t)4 * kSubWarpFloats * sizeof(float);
    const size_t smem = tiles > planBytes(p.plan) ? tiles : planBytes(p.plan);
    k_subpix<<<divUp(p.bw * p.bh, 4), 128, smem, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchCutMean(const CutMeanParams& p, cudaStream_t s) {
    k_cutmean<<<1, 256, planBytes(p.plan), s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchPixfield(const PixfieldParams& p, cudaStream_t s) {
    k_pixfield<<<dim3(divUp(p.w, kPfTW), divUp(p.h, kPfTH)), 256, 0, s>>>(p);
    return cudaGetLastError();
}
size_t synthSmemBytes(int fs) {  // declared in fg_params.h
    // worst-case field region of a tile (GW x GH float2) + its horizontal stage + interior warps + mismatch + row sums
    const int gw = (kSyEW + fs - 1) / fs + 3, gh = (kSyEH + fs - 1) / fs + 3;
    return (size_t)gw * gh * 8 + (size_t)gh * kSyEW * 8 + (size_t)kSyTW * kSyTH * 8 + (size_t)((kSyEH * kSyEW + 15) & ~15) +
           (size_t)kSyEH * kSyTW * 2;
}
cudaError_t launchSynth(const SynthParams& p, cudaStream_t s) {
    const size_t smem = synthSmemBytes(p.fs);
    k_synth<<<dim3(divUp(p.W, kSyTW), divUp(p.H, kSyTH)), 256, smem, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launchFallback(const FallbackParams& p, cudaStream_t s) {
    k_fallback<<<148 * 4, 256, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace fgk
