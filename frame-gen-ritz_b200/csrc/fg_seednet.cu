// The seed proposer: a 6-layer 3x3 convolutional net that reads the 2-channel luma (prev, curr) of one pyramid level
// and proposes, per 8x8 block of that level, two candidate half-vectors and a confidence for the integer block
// search. No counterpart in the reference's V1 path (its learned estimator, MotionVersion::Learned, is a different
// net that replaces the search); here the plain integer search keeps the decision, the net only adds candidates.
//
//   layer  in -> out  stride  activation     output grid (level w x h)
//   1      2  -> 32   2       ReLU           ceil(w/2) x ceil(h/2)
//   2      32 -> 32   2       ReLU           ceil(w/4) x ceil(h/4)
//   3      32 -> 32   2       ReLU           ceil(w/8) x ceil(h/8)   (= the level's block grid)
//   4, 5   32 -> 32   1       ReLU
//   6      32 -> 8    1       none           (c1x, c1y, c2x, c2y, confidence logit, 3 unused) per block
// 3x3 kernels, zero padding 1. Activations NHWC bfloat16; weights bfloat16 [cout][tap][cin] (tap = 3 ky + kx);
// biases and every accumulation float32.
//
// Forward: implicit GEMM on the tensor cores (mma.sync m16n8k16, bf16 x bf16 -> f32): M = output pixels, N = cout,
// K = 9 cin (layer 1: 18, zero-padded to 32); a CTA = 4 warps x 16 output pixels, the layer's weights staged once in
// shared memory. The GEMMs are small (a 4K frame's level 1: 1.2 GFLOP in all), so warp-level MMA with
// register-gathered A fragments is enough; no TMEM / TMA staging.
// Training: the backward's weight and input gradients are tcgen05 implicit GEMMs (fg_seednet_bwd.cu); the loss and
// Adam are elementwise kernels here. bf16 operands, float32 accumulation, gradients and master weights.
#include <cuda_bf16.h>

#include <algorithm>

#include "fg_device.h"
#include "fg_seednet.h"

namespace fgk {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t ldBf2(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// level luma (float, levels) -> the net's input: (v - 128) / 64 in bfloat16, channels (prev, curr)
__global__ void __launch_bounds__(256) k_sn_pack(const float* __restrict__ la, const float* __restrict__ lc, int n,
                                                bf16* __restrict__ x) {
    pdlEnter();
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float a = __fmul_rn(__fsub_rn(la[i], 128.0f), 1.0f / 64.0f), c = __fmul_rn(__fsub_rn(lc[i], 128.0f), 1.0f / 64.0f);
    reinterpret_cast<__nv_bfloat162*>(x)[i] = __floats2bfloat162_rn(a, c);
}

// One 3x3 convolution layer, forward, in tiles of 64 output pixels (4 warps x 16). in: [B][H][W][CIN] bf16 (layer 1
// with a.la set: the two float luma planes, normalised on the fly exactly as k_sn_pack does); out: [B][Ho][Wo][COUT]
// bf16 (ReLU) or float (last layer).
template <int CIN>
struct SnShape {
    static constexpr int K = 9 * CIN, KP = (K + 15) / 16 * 16, NKC = KP / 16;
};

// the layer's weights (bf16 [cout][9 cin], k zero-padded to a multiple of 16) and biases into shared memory
template <int CIN, int COUT>
__device__ __forceinline__ void snStage(const SnConvArgs& a, bf16* ws, float* bs) {
    constexpr int K = SnShape<CIN>::K, KP = SnShape<CIN>::KP;
    if (K == KP) {   // [cout][9 cin] is already the staged layout: a straight 16-byte copy
        const uint4* src = reinterpret_cast<const uint4*>(a.w);
        uint4* dst = reinterpret_cast<uint4*>(ws);
        for (int i = threadIdx.x; i < COUT * K / 8; i += blockDim.x) dst[i] = src[i];
    } else {
        const bf16* __restrict__ w = reinterpret_cast<const bf16*>(a.w);
        for (int i = threadIdx.x; i < COUT * KP; i += blockDim.x) {
            const int n = i / KP, k = i % KP;
            ws[i] = k < K ? w[n * K + k] : __float2bfloat16(0.0f);
        }
    }
    if (threadIdx.x < COUT) bs[threadIdx.x] = a.b[threadIdx.x];
}

// this thread's A fragments of every k chunk of tile `tile`, gathered up front (independent loads in flight together)
template <int CIN, int STRIDE>
__device__ __forceinline__ void snGather(const SnConvArgs& a, int tile, uint32_t (*af)[4]) {
    constexpr int K = SnShape<CIN>::K, NKC = SnShape<CIN>::NKC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int npix = a.B * a.Ho * a.Wo;
    const int p0 = (tile * 4 + warp) * 16;
    int base[2], oy[2], ox[2];
    bool val[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {   // the two output pixels of this thread's A rows
        const int p = p0 + gid + 8 * r;
        val[r] = p < npix;
        const int pp = val[r] ? p : 0;
        const int b = pp / (a.Ho * a.Wo), rem = pp % (a.Ho * a.Wo);
        oy[r] = (rem / a.Wo) * STRIDE - 1;
        ox[r] = (rem % a.Wo) * STRIDE - 1;
        base[r] = b * a.H * a.W;
    }
    const bf16* __restrict__ x = reinterpret_cast<const bf16*>(a.x);
#pragma unroll
    for (int kc = 0; kc < NKC; kc++)
#pragma unroll
        for (int q = 0; q < 4; q++) {   // register q: row gid (+8 for q odd), k columns +8 for q >= 2
            const int r = q & 1;
            // CIN = 32: a 16-wide k chunk lies in one tap; CIN = 2: pairs (tap, ci 0..1)
            const int k = kc * 16 + tig * 2 + ((q >> 1) << 3);
            const int tap = CIN == 32 ? (kc >> 1) : k / CIN;
            const int ci = CIN == 32 ? ((kc & 1) << 4) + tig * 2 + ((q >> 1) << 3) : 0;
            uint32_t v = 0;
            if ((CIN == 32 || k < K) && val[r]) {
                const int iy = oy[r] + tap / 3, ix = ox[r] + tap % 3;
                if ((unsigned)iy < (unsigned)a.H && (unsigned)ix < (unsigned)a.W) {
                    const size_t pix = (size_t)(base[r] + iy * a.W + ix);
                    if (CIN == 2 && a.la) {
                        const float la = __fmul_rn(__fsub_rn(__ldg(a.la + pix), 128.0f), 1.0f / 64.0f);
                        const float lc = __fmul_rn(__fsub_rn(__ldg(a.lc + pix), 128.0f), 1.0f / 64.0f);
                        const __nv_bfloat162 h = __floats2bfloat162_rn(la, lc);
                        v = *reinterpret_cast<const uint32_t*>(&h);
                    } else {
                        v = ldBf2(x + pix * CIN + ci);
                    }
                }
            }
            af[kc][q] = v;
        }
}

// the MMAs of one tile and its store (bias, ReLU or the float output)
template <int CIN, int COUT, bool LAST>
__device__ __forceinline__ void snMmaStore(const SnConvArgs& a, int tile, const uint32_t (*af)[4], const bf16* ws,
                                           const float* bs) {
    constexpr int KP = SnShape<CIN>::KP, NKC = SnShape<CIN>::NKC, NT = COUT / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int npix = a.B * a.Ho * a.Wo;
    const int p0 = (tile * 4 + warp) * 16;
    if (p0 >= npix) return;
    float acc[NT][4];
#pragma unroll
    for (int t = 0; t < NT; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0f;
#pragma unroll
    for (int kc = 0; kc < NKC; kc++)
#pragma unroll
        for (int t = 0; t < NT; t++) {
            const bf16* wb = ws + (t * 8 + gid) * KP + kc * 16 + tig * 2;
            mma16816(acc[t], af[kc], ldBf2(wb), ldBf2(wb + 8));
        }
#pragma unroll
    for (int t = 0; t < NT; t++) {
        const int n = t * 8 + tig * 2;
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int p = p0 + gid + 8 * r;
            if (p >= npix) continue;
            float v0 = acc[t][2 * r] + bs[n], v1 = acc[t][2 * r + 1] + bs[n + 1];
            if (LAST) {
                *reinterpret_cast<float2*>(a.yf + (size_t)p * COUT + n) = make_float2(v0, v1);
            } else {
                v0 = fmaxf(v0, 0.0f);
                v1 = fmaxf(v1, 0.0f);
                reinterpret_cast<__nv_bfloat162*>(a.y)[((size_t)p * COUT + n) >> 1] = __floats2bfloat162_rn(v0, v1);
            }
        }
    }
}

// one layer, one launch: a CTA per tile
template <int CIN, int COUT, int STRIDE, bool LAST>
__global__ void __launch_bounds__(128) k_sn_conv(const SnConvArgs a) {
    pdlEnter();
    __shared__ __align__(16) bf16 ws[COUT * SnShape<CIN>::KP];
    __shared__ float bs[COUT];
    uint32_t af[SnShape<CIN>::NKC][4];
    snGather<CIN, STRIDE>(a, blockIdx.x, af);
    snStage<CIN, COUT>(a, ws, bs);
    __syncthreads();
    snMmaStore<CIN, COUT, LAST>(a, blockIdx.x, af, ws, bs);
}

// ---------------------------------------------------------------------------------------------- training kernels
// the loss of one batch and its gradient at the last layer's output (per block: huber(c1 - truth) +
// huber(c2 - search) + BCE(confidence, |c1 - truth|_inf < 1), each block weighted by its target's weight; scale =
// 1 / blocks: the batch mean)
__global__ void __launch_bounds__(256) k_sn_loss(const float* __restrict__ out, const float* __restrict__ tgt, int n,
                                                float* __restrict__ dout, float* __restrict__ loss, float scale) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    float l = 0.0f;
    if (i < n) {
        const float* o = out + (size_t)i * kSnOut;
        const float* t = tgt + (size_t)i * kSnTargets;   // truth (2), search (2), weight, unused
        float* d = dout + (size_t)i * kSnOut;
        const float wgt = t[4];
        float err = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float e = o[k] - t[k];
            const float ae = fabsf(e);
            l += wgt * (ae < 1.0f ? 0.5f * e * e : ae - 0.5f);
            d[k] = scale * wgt * (ae < 1.0f ? e : copysignf(1.0f, e));
            if (k < 2) err = fmaxf(err, ae);
        }
        const float y = err < 1.0f ? 1.0f : 0.0f, z = o[4];
        const float sg = 1.0f / (1.0f + expf(-z));
        l += wgt * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
        d[4] = scale * wgt * (sg - y);
        d[5] = d[6] = d[7] = 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l * scale);
}

// Adam on the float32 master parameters; refreshes their bfloat16 copy (the forward's weights) and zeroes the gradient.
// The gradient is scaled by gscale as it is read (data-parallel training: the ranks' sum times 1 / ranks).
__global__ void __launch_bounds__(256) k_sn_adam(const SnAdamArgs a) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= a.n) return;
    const float g = a.grad[i] * a.gscale;
    const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
    const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    const float p = a.p[i] - a.lr * (m * a.c1) / (sqrtf(v * a.c2) + a.eps);
    a.p[i] = p;
    a.grad[i] = 0.0f;
    reinterpret_cast<bf16*>(a.wb)[i] = __float2bfloat16(p);
}

// ---------------------------------------------------------------------------------------------- launchers
cudaError_t launchSnPack(const float* la, const float* lc, int n, void* x, cudaStream_t s) {
    return launchPdl(k_sn_pack, dim3(divUp(n, 256)), dim3(256), 0, s, la, lc, n, reinterpret_cast<bf16*>(x));
}

cudaError_t launchSnConv(int layer, const SnConvArgs& a, cudaStream_t s) {
    const dim3 grid(divUp(a.B * a.Ho * a.Wo, 64));
    switch (layer) {
        case 0: return launchPdl(k_sn_conv<2, 32, 2, false>, grid, dim3(128), 0, s, a);
        case 1:
        case 2: return launchPdl(k_sn_conv<32, 32, 2, false>, grid, dim3(128), 0, s, a);
        case 3:
        case 4: return launchPdl(k_sn_conv<32, 32, 1, false>, grid, dim3(128), 0, s, a);
        case 5: return launchPdl(k_sn_conv<32, kSnOut, 1, true>, grid, dim3(128), 0, s, a);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchSnLoss(const float* out, const float* tgt, int n, float* dout, float* loss, float scale, cudaStream_t s) {
    k_sn_loss<<<divUp(n, 256), 256, 0, s>>>(out, tgt, n, dout, loss, scale);
    return cudaGetLastError();
}

cudaError_t launchSnAdam(const SnAdamArgs& a, cudaStream_t s) {
    k_sn_adam<<<divUp(a.n, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace fgk
