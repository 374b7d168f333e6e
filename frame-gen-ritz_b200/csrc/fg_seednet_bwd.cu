// The seed proposer's training backward on the fifth-generation tensor cores (tcgen05, bf16 operands in shared memory,
// f32 accumulators in tensor memory): the weight gradient and the input gradient of every 3x3 convolution layer as
// implicit GEMMs, replacing per-element loops. Same layouts and semantics as the per-layer forward in fg_seednet.cu.
//
//   k_sn_dw_tc<CIN, COUT, S>  dW[co][tap][ci] += sum_p x[S p + tap - 1][ci] dpre[p][co], db[co] += sum_p dpre[p][co]
//       GEMM D[m][n] = sum_k A[m][k] B[n][k] with m = tap * CIN + ci (plus one row of ones at m = 9 CIN, which makes
//       that row of D the bias gradient), n = co, k = output pixel. Every CTA reduces a contiguous slice of the output
//       pixels in chunks of 64 (4 MMAs of K = 16 per 128-row chunk of m), the operands double-buffered, and stores its
//       partial D; k_sn_dw_sum then adds the partials into dW / db in CTA order, so the gradient is deterministic.
//   k_sn_dx_tc<CIN, COUT, S>  dpre_in[q][ci] = [x[q][ci] > 0] sum_{tap, co} w[co][tap][ci] dpre[p(q, tap)][co], the
//       output pixels p with S p + tap - 1 = q: GEMM with m = input pixel q (128 per chunk), n = ci, k = tap * COUT + co
//       (padded to a multiple of 16); the weights are staged once per CTA.
// The gradient at a layer's output (float) enters the MMAs rounded to bf16, the way the forward's activations do;
// accumulation is f32. Operands are K-major without swizzle (fg_tc.h): a core matrix is 8 rows of 8 consecutive k.
// Waits on the MMAs' mbarriers are bounded (100 ms, then kErrSeedNet into *err, one more bounded wait, TMEM freed).
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "fg_device.h"
#include "fg_params.h"
#include "fg_seednet.h"
#include "fg_tc.h"

namespace fgk {
namespace {

using bf16 = __nv_bfloat16;
constexpr uint64_t kBwdWaitNs = 100000000ull;
constexpr int kBwdThreads = 256;
constexpr int kDwK = 64;   // output pixels per staged chunk of the weight gradient (8 k-groups)

__device__ __forceinline__ uint32_t bpack(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

template <int CIN, int COUT>
struct DwShape {
    static constexpr int MR = 9 * CIN + 1;                 // rows: (tap, ci), then the ones row (bias)
    static constexpr int NCH = (MR + 127) / 128;           // 128-row chunks of m
    static constexpr int NP = COUT < 16 ? 16 : COUT;       // N of the MMA (8 outputs padded to 16)
    static constexpr int KG = kDwK / 8;                    // k-groups per staged chunk
    static constexpr int A_BYTES = NCH * 16 * KG * 128;    // [m-group][k-group][8 rows][16 B]
    static constexpr int B_BYTES = NP / 8 * KG * 128;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int TCOLS = NCH * NP <= 32 ? 32 : NCH * NP <= 64 ? 64 : 128;
    static constexpr size_t SMEM = 2 * (size_t)STAGE + 64;
};

// waits for the mbarrier's next phase (bounded); false when it gave up
__device__ __forceinline__ bool waitPhase(uint64_t* bar, uint32_t& ph) {
    const bool ok = mbarWait(bar, ph, kBwdWaitNs);
    ph ^= 1u;
    return ok;
}

}  // namespace

template <int CIN, int COUT, int S>
__global__ void __launch_bounds__(kBwdThreads) k_sn_dw_tc(const SnBackArgs a, int chunksPerCta, unsigned int* err) {
    using Sh = DwShape<CIN, COUT>;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + 2 * Sh::STAGE);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 2 * Sh::STAGE + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int npix = a.B * a.Ho * a.Wo;
    const int nchunks = (npix + kDwK - 1) / kDwK;
    const int c0 = blockIdx.x * chunksPerCta, c1 = min(nchunks, c0 + chunksPerCta);
    if (warp == 0) tmemAlloc(tslot, Sh::TCOLS);
    if (tid == 0) {
        mbarInit(&bars[0], 1);
        mbarInit(&bars[1], 1);
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tbase = *tslot;
    const bf16* __restrict__ x = reinterpret_cast<const bf16*>(a.x);
    uint32_t ph[2] = {0u, 0u};
    bool ok = true;
    auto stage = [&](int chunk, int buf) {
        unsigned char* A = sm + buf * Sh::STAGE;
        unsigned char* Bm = A + Sh::A_BYTES;
        const int p0 = chunk * kDwK;
        // A: row m, 8 pixels per 16-byte row
        for (int i = tid; i < Sh::NCH * 16 * Sh::KG * 8; i += kBwdThreads) {
            const int r = i & 7, kg = (i >> 3) % Sh::KG, mg = (i >> 3) / Sh::KG;
            const int m = mg * 8 + r;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int p = p0 + kg * 8 + j;
                float e = 0.0f;
                if (p < npix && m <= 9 * CIN) {
                    if (m == 9 * CIN) {
                        e = 1.0f;
                    } else {
                        const int tap = m / CIN, ci = m % CIN;
                        const int b = p / (a.Ho * a.Wo), rem = p % (a.Ho * a.Wo);
                        const int iy = (rem / a.Wo) * S - 1 + tap / 3, ix = (rem % a.Wo) * S - 1 + tap % 3;
                        if ((unsigned)iy < (unsigned)a.H && (unsigned)ix < (unsigned)a.W)
                            e = __bfloat162float(x[((size_t)(b * a.H + iy) * a.W + ix) * CIN + ci]);
                    }
                }
                v[j] = e;
            }
            reinterpret_cast<uint4*>(A)[(mg * Sh::KG + kg) * 8 + r] =
                make_uint4(bpack(v[0], v[1]), bpack(v[2], v[3]), bpack(v[4], v[5]), bpack(v[6], v[7]));
        }
        // B: row co, 8 pixels of the output gradient
        for (int i = tid; i < Sh::NP / 8 * Sh::KG * 8; i += kBwdThreads) {
            const int r = i & 7, kg = (i >> 3) % Sh::KG, ng = (i >> 3) / Sh::KG;
            const int co = ng * 8 + r;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int p = p0 + kg * 8 + j;
                v[j] = (p < npix && co < COUT) ? a.dy[(size_t)p * COUT + co] : 0.0f;
            }
            reinterpret_cast<uint4*>(Bm)[(ng * Sh::KG + kg) * 8 + r] =
                make_uint4(bpack(v[0], v[1]), bpack(v[2], v[3]), bpack(v[4], v[5]), bpack(v[6], v[7]));
        }
    };
    const uint32_t idesc = tcIdescBf16(128, Sh::NP);
    for (int c = c0; c < c1 && ok; c++) {
        const int i = c - c0, buf = i & 1;
        if (i >= 2) ok = waitPhase(&bars[buf], ph[buf]) && ok;   // the MMAs of chunk c - 2 read this buffer
        ok = __syncthreads_and(ok);
        if (!ok) break;
        stage(c, buf);
        fenceAsyncShared();
        __syncthreads();
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t A = smemAddr(sm + buf * Sh::STAGE), Bm = A + Sh::A_BYTES;
            for (int ch = 0; ch < Sh::NCH; ch++)
                for (int s = 0; s < Sh::KG / 2; s++)
                    tcMma(tbase + ch * Sh::NP, tcDesc(A + (uint32_t)((ch * 16 * Sh::KG + 2 * s) * 128), 128, Sh::KG * 128),
                          tcDesc(Bm + (uint32_t)(2 * s * 128), 128, Sh::KG * 128), idesc, (i > 0 || s > 0) ? 1u : 0u);
            tcCommit(&bars[buf]);
        }
    }
    // the last (up to two) chunks' MMAs
    const int n = c1 - c0;
    for (int k = 0; k < 2; k++) {
        const int i = n - 1 - k;
        if (i < 0 || i < n - 2) continue;
        const bool w = waitPhase(&bars[i & 1], ph[i & 1]);
        ok = w && ok;
    }
    ok = __syncthreads_and(ok);
    tcFenceAfter();
    if (ok && n > 0) {   // epilogue: lanes 32 (warp % 4) .., columns half (warp / 4) of NP
        const int q = warp & 3, half = warp >> 2;
        for (int ch = 0; ch < Sh::NCH; ch++) {
            const int m = ch * 128 + 32 * q + lane;
            const uint32_t ta = tbase + ((uint32_t)(32 * q) << 16) + ch * Sh::NP + half * (Sh::NP / 2);
            float v[16];
            if (Sh::NP / 2 == 16) tmemLd16(ta, v);
            else tmemLd8(ta, v);
            float* part = a.part + (size_t)blockIdx.x * kSnPartFloats;
            for (int j = 0; j < Sh::NP / 2; j++) {
                const int co = half * (Sh::NP / 2) + j;
                if (co < COUT && m <= 9 * CIN) part[m * COUT + co] = v[j];
            }
        }
    }
    if (!ok && tid == 0 && err) atomicOr(err, kErrSeedNet);
    tcFenceBefore();
    __syncthreads();
    if (warp == 0) {
        tcFenceAfter();
        tmemFree(tbase, Sh::TCOLS);
    }
}

// dW / db += the sum of the CTAs' partial products, in CTA order (one thread per (row, co))
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_sn_dw_sum(const SnBackArgs a, int ctas) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= (9 * CIN + 1) * COUT) return;
    const int m = i / COUT, co = i % COUT;
    float s = 0.0f;
    for (int b = 0; b < ctas; b++) s += a.part[(size_t)b * kSnPartFloats + i];
    if (m < 9 * CIN) a.dw[(co * 9 + m / CIN) * CIN + m % CIN] += s;
    else a.db[co] += s;
}

template <int CIN, int COUT>
struct DxShape {
    static constexpr int K = 9 * COUT, KP = (K + 15) / 16 * 16, KG = KP / 8;
    static constexpr int A_BYTES = 16 * KG * 128;          // 128 rows (input pixels)
    static constexpr int B_BYTES = CIN / 8 * KG * 128;     // CIN rows
    static constexpr size_t SMEM = 2 * (size_t)A_BYTES + B_BYTES + 64;
};

template <int CIN, int COUT, int S>
__global__ void __launch_bounds__(kBwdThreads) k_sn_dx_tc(const SnBackArgs a, unsigned int* err) {
    static_assert(CIN == 32, "the input gradient is needed for the 32-channel inputs only");
    using Sh = DxShape<CIN, COUT>;
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char* Bm = sm + 2 * Sh::A_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Bm + Sh::B_BYTES);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(Bm + Sh::B_BYTES + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nq = a.B * a.H * a.W;
    const int nchunks = (nq + 127) / 128;
    const bf16* __restrict__ w = reinterpret_cast<const bf16*>(a.w);
    const bf16* __restrict__ x = reinterpret_cast<const bf16*>(a.x);
    if (warp == 0) tmemAlloc(tslot, 64);
    if (tid == 0) {
        mbarInit(&bars[0], 1);
        mbarInit(&bars[1], 1);
    }
    // B: row ci, k = tap * COUT + co: w[co][tap][ci]
    for (int i = tid; i < CIN / 8 * Sh::KG * 8; i += kBwdThreads) {
        const int r = i & 7, kg = (i >> 3) % Sh::KG, ng = (i >> 3) / Sh::KG;
        const int ci = ng * 8 + r;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int k = kg * 8 + j;
            v[j] = k < Sh::K ? __bfloat162float(w[((k % COUT) * 9 + k / COUT) * CIN + ci]) : 0.0f;
        }
        reinterpret_cast<uint4*>(Bm)[(ng * Sh::KG + kg) * 8 + r] =
            make_uint4(bpack(v[0], v[1]), bpack(v[2], v[3]), bpack(v[4], v[5]), bpack(v[6], v[7]));
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tbase = *tslot;
    uint32_t ph[2] = {0u, 0u};
    bool ok = true;
    auto stage = [&](int chunk, int buf) {   // A: row q, k = tap * COUT + co: dpre[p(q, tap)][co]
        unsigned char* A = sm + buf * Sh::A_BYTES;
        for (int i = tid; i < 16 * Sh::KG * 8; i += kBwdThreads) {
            const int r = i & 7, kg = (i >> 3) % Sh::KG, mg = (i >> 3) / Sh::KG;
            const int q = chunk * 128 + mg * 8 + r;
            const int k0 = kg * 8, tap = k0 / COUT, co0 = k0 % COUT;   // 8 consecutive k share a tap (COUT % 8 == 0)
            uint4 o = make_uint4(0, 0, 0, 0);
            if (q < nq && k0 < Sh::K) {
                const int b = q / (a.H * a.W), rem = q % (a.H * a.W), qy = rem / a.W, qx = rem % a.W;
                const int ty = qy + 1 - tap / 3, tx = qx + 1 - tap % 3;   // = S p
                if (ty >= 0 && tx >= 0 && ty % S == 0 && tx % S == 0 && ty / S < a.Ho && tx / S < a.Wo) {
                    const float4* g = reinterpret_cast<const float4*>(a.dy + ((size_t)(b * a.Ho + ty / S) * a.Wo + tx / S) * COUT + co0);
                    const float4 u = g[0], v = g[1];
                    o = make_uint4(bpack(u.x, u.y), bpack(u.z, u.w), bpack(v.x, v.y), bpack(v.z, v.w));
                }
            }
            reinterpret_cast<uint4*>(A)[(mg * Sh::KG + kg) * 8 + r] = o;
        }
    };
    const uint32_t idesc = tcIdescBf16(128, CIN);
    auto epi = [&](int chunk, int acc) {
        const int qw = warp & 3, half = warp >> 2;
        const int q = chunk * 128 + 32 * qw + lane;
        float v[16];
        tmemLd16(tbase + ((uint32_t)(32 * qw) << 16) + acc * 32 + half * 16, v);
        if (q >= nq) return;
        const bf16* xq = x + (size_t)q * CIN + half * 16;
        float* d = a.dx + (size_t)q * CIN + half * 16;
#pragma unroll
        for (int j = 0; j < 16; j++) d[j] = __bfloat162float(xq[j]) > 0.0f ? v[j] : 0.0f;
    };
    int it = 0, prev = -1;
    for (int c = blockIdx.x; c < nchunks && ok; c += gridDim.x, it++) {
        const int buf = it & 1;
        stage(c, buf);
        fenceAsyncShared();
        tcFenceBefore();
        ok = __syncthreads_and(ok);
        if (!ok) break;
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t A = smemAddr(sm + buf * Sh::A_BYTES), B = smemAddr(Bm);
            for (int s = 0; s < Sh::KG / 2; s++)
                tcMma(tbase + buf * 32, tcDesc(A + (uint32_t)(2 * s * 128), 128, Sh::KG * 128),
                      tcDesc(B + (uint32_t)(2 * s * 128), 128, Sh::KG * 128), idesc, s > 0 ? 1u : 0u);
            tcCommit(&bars[buf]);
        }
        if (prev >= 0) {   // the previous chunk's epilogue overlaps this chunk's MMAs
            ok = waitPhase(&bars[buf ^ 1], ph[buf ^ 1]) && ok;
            tcFenceAfter();
            if (ok) epi(prev, buf ^ 1);
        }
        prev = c;
    }
    if (prev >= 0 && ok) {
        const int buf = (it - 1) & 1;
        ok = waitPhase(&bars[buf], ph[buf]) && ok;
        tcFenceAfter();
        if (ok) epi(prev, buf);
    }
    if (!ok) {
        if (tid == 0 && err) atomicOr(err, kErrSeedNet);
        for (int b = 0; b < 2; b++) mbarWait(&bars[b], ph[b], kBwdWaitNs);
    }
    tcFenceBefore();
    __syncthreads();
    if (warp == 0) {
        tcFenceAfter();
        tmemFree(tbase, 64);
    }
}

namespace {

template <int CIN, int COUT, int S>
cudaError_t dwLaunch(const SnBackArgs& a, unsigned int* err, cudaStream_t s) {
    using Sh = DwShape<CIN, COUT>;
    static_assert(Sh::SMEM <= 227 * 1024, "shared memory");
    const int npix = a.B * a.Ho * a.Wo;
    const int nchunks = (npix + kDwK - 1) / kDwK;
    const int ctas = std::min(nchunks, a.partCtas);
    const int per = (nchunks + ctas - 1) / ctas;
    const int grid = (nchunks + per - 1) / per;
    k_sn_dw_tc<CIN, COUT, S><<<grid, kBwdThreads, Sh::SMEM, s>>>(a, per, err);
    k_sn_dw_sum<CIN, COUT><<<divUp((9 * CIN + 1) * COUT, 256), 256, 0, s>>>(a, grid);
    return cudaGetLastError();
}

template <int COUT, int S>
cudaError_t dxLaunch(const SnBackArgs& a, unsigned int* err, cudaStream_t s) {
    using Sh = DxShape<32, COUT>;
    const int nchunks = (a.B * a.H * a.W + 127) / 128;
    k_sn_dx_tc<32, COUT, S><<<std::min(nchunks, 2 * smCount()), kBwdThreads, Sh::SMEM, s>>>(a, err);
    return cudaGetLastError();
}

template <class K>
cudaError_t setSmem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

cudaError_t prepareSeedNetBackward() {
    cudaError_t e = setSmem(k_sn_dw_tc<2, 32, 2>, DwShape<2, 32>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dw_tc<32, 32, 2>, DwShape<32, 32>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dw_tc<32, 32, 1>, DwShape<32, 32>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dw_tc<32, kSnOut, 1>, DwShape<32, kSnOut>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dx_tc<32, 32, 2>, DxShape<32, 32>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dx_tc<32, 32, 1>, DxShape<32, 32>::SMEM);
    if (e == cudaSuccess) e = setSmem(k_sn_dx_tc<32, kSnOut, 1>, DxShape<32, kSnOut>::SMEM);
    return e;
}

cudaError_t launchSnBackwardTc(int layer, const SnBackArgs& a, bool needDx, unsigned int* err, cudaStream_t s) {
    cudaError_t e;
    switch (layer) {
        case 0: return dwLaunch<2, 32, 2>(a, err, s);
        case 1:
        case 2:
            e = dwLaunch<32, 32, 2>(a, err, s);
            return e == cudaSuccess && needDx ? dxLaunch<32, 2>(a, err, s) : e;
        case 3:
        case 4:
            e = dwLaunch<32, 32, 1>(a, err, s);
            return e == cudaSuccess && needDx ? dxLaunch<32, 1>(a, err, s) : e;
        case 5:
            e = dwLaunch<32, kSnOut, 1>(a, err, s);
            return e == cudaSuccess && needDx ? dxLaunch<kSnOut, 1>(a, err, s) : e;
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace fgk
