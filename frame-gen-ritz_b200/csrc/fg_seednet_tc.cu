// The seed proposer's forward pass for the Interpolator, fused into two kernels on the fifth-generation tensor cores
// (tcgen05: bf16 operands in shared memory, f32 accumulators in tensor memory). Same net and arithmetic as the
// per-layer forward in fg_seednet.cu (3x3 convolutions, zero padding 1, ReLU, bf16 activations rounded to nearest,
// f32 accumulation and biases); only the accumulation order inside a dot product differs.
//
//   k_sn_enc  layers 1-3 (the three stride-2 layers): one CTA per tile of 7 x 9 output cells of layer 3 (the level's
//             8x8 block grid). It loads the 79 x 63 luma region the tile depends on, and computes layer 1 on the
//             39 x 31 region of layer 1 that layer 2 needs, layer 2 on 19 x 15, layer 3 on the tile; the layer
//             outputs stay in shared memory, only layer 3's goes to global memory (bf16, NHWC).
//   k_sn_head layers 4-6 (stride 1, on the block grid): one CTA per tile of 10 x 8 cells; loads the 16 x 14 cells of
//             layer 3 around it, computes layer 4 on 14 x 12, layer 5 on 12 x 10, layer 6 on the tile (float out).
// For training the same two kernels also store layers 1, 2, 4 and 5 (the backward's inputs): each CTA the part of
// every layer that its tile owns (the tiles partition the block grid, so their footprints partition every layer),
// and may read the packed bf16 input instead of the float luma.
//
// Each layer is an implicit GEMM: M = output pixels (chunks of 128 rows), N = 32 output channels (layer 6: 16, of
// which 8 are the net's outputs), K = 9 taps x 32 input channels, issued as 18 MMAs of K = 16.
// The A operand is never gathered: the activations sit in shared memory as planes [8-channel group][pixel][8 x bf16],
// so the 8 consecutive pixels of a core matrix are 16 bytes apart, and a tap is a shift of the start address.
//   - Rows are output pixels in a padded raster: output (y, x) is row y * P + x, where P is the pitch of the plane the
//     layer reads; columns x beyond the region are computed and thrown away. A stride-1 tap (ky, kx) then reads
//     plane row m + ky * P + kx for output row m.
//   - A stride-2 layer reads its input split into four phase planes (even / odd row x even / odd column), each of
//     pitch P: tap (ky, kx) reads phase (ky & 1, kx & 1) at row m + (ky >> 1) * P + (kx >> 1).
//   - The epilogue of each layer (tensor memory -> registers -> bias, ReLU, bf16) writes straight into the layout the
//     next layer reads, and writes 0 for positions outside the layer's image (the next layer's zero padding).
// Layer 1 has 2 input channels, so its A operand (K = 18, padded to 32) is built per chunk from the luma region
// (im2col into a double buffer) while the previous chunk's MMAs run.
//
// Synchronisation: one thread issues a chunk's MMAs and commits them to an mbarrier; every thread waits on it (a
// bounded wait: after 100 ms the kernel records kErrSeedNet, waits once more for what it issued and frees its tensor
// memory), then reads its rows and columns of the accumulator (warp w reads lanes 32 (w % 4) .. + 31). Two
// accumulators in tensor memory alternate, so chunk c's MMAs overlap chunk c-1's epilogue.
#include <cuda_bf16.h>

#include <cstdint>

#include "fg_device.h"
#include "fg_params.h"
#include "fg_seednet.h"
#include "fg_tc.h"

namespace fgk {
namespace {

using bf16 = __nv_bfloat16;

constexpr uint64_t kWaitNs = 100000000ull;   // 100 ms: far beyond any chunk's MMAs

// offsets of every layer's weights and biases in the flat parameter array
__device__ constexpr int kW[kSnLayers] = {snWeightOff(0), snWeightOff(1), snWeightOff(2), snWeightOff(3),
                                          snWeightOff(4), snWeightOff(5)};
__device__ constexpr int kB[kSnLayers] = {snBiasOff(0), snBiasOff(1), snBiasOff(2), snBiasOff(3), snBiasOff(4),
                                          snBiasOff(5)};

// ---- encoder tile geometry (region sizes in each layer's own grid)
constexpr int kEncTX = 7, kEncTY = 9;                        // layer-3 cells per tile
constexpr int kP3 = kEncTX + 1;                              // layer-3 rows' pitch = its phase planes' pitch
constexpr int kM3 = kEncTY * kP3;                            // 72 rows: one 128-row chunk
constexpr int kR2y = 2 * kEncTY + 1, kR2x = 2 * kEncTX + 1;  // 19 x 15 layer-2 outputs
constexpr int kP2 = kR2x + 1;                                // 16
constexpr int kM2 = kR2y * kP2;                              // 304 rows: chunks at 0, 128, 176
constexpr int kR1y = 2 * kR2y + 1, kR1x = 2 * kR2x + 1;      // 39 x 31 layer-1 outputs
constexpr int kP1 = kR1x + 1;                                // 32
constexpr int kM1 = kR1y * kP1;                              // 1248 rows: 10 chunks
constexpr int kR0y = 2 * kR1y + 1, kR0x = 2 * kR1x + 1;      // 79 x 63 luma
constexpr int kP0 = kR0x + 1;                                // 64
constexpr int kNC1 = (kM1 + 127) / 128, kNC2 = (kM2 + 127) / 128;
// phase-plane lengths: what the region writes, and at least the last row a 128-row chunk reads + 1
constexpr int kPl2 = ((kR1y + 1) / 2) * kP2 + 1;             // 321
constexpr int kPl3 = 127 + kP3 + 1 + 1;                      // 137
static_assert(kPl2 >= kM2 + kP2 + 1 && kPl2 >= ((kR1y + 1) / 2) * kP2, "layer-2 phase planes");
static_assert(kPl3 >= 128 + kP3 + 1 && kPl3 >= ((kR2y + 1) / 2) * kP3, "layer-3 phase planes");
static_assert(kM3 <= 128 && kM2 >= 128 && kM1 >= 128, "chunking");
static_assert(2 * (kR1x - 1) + 2 < kR0x, "im2col reads stay inside the luma region");

// shared-memory carve-up of k_sn_enc (bytes, 128-aligned)
constexpr int kEncThreads = 512;
constexpr size_t kOffLuma = 0;                                          // uint32 (bf16 prev, bf16 curr) kR0y x kP0
constexpr size_t kOffCol = kOffLuma + (size_t)kR0y * kP0 * 4;           // 2 x [4][128] x 16 B
constexpr size_t kOffPl2 = kOffCol + 2 * 4 * 128 * 16;                  // [4 phase][4 c8][kPl2] x 16 B
constexpr size_t kOffPl3 = kOffPl2 + (size_t)16 * kPl2 * 16;            // [4 phase][4 c8][kPl3] x 16 B
constexpr size_t kOffW1 = kOffPl3 + (size_t)16 * kPl3 * 16;             // [4 kc][32 n] x 16 B
constexpr size_t kOffW2 = kOffW1 + 4 * 32 * 16;                         // [36 kc][32 n] x 16 B
constexpr size_t kOffW3 = kOffW2 + 36 * 32 * 16;
constexpr size_t kOffB = kOffW3 + 36 * 32 * 16;                         // 3 x 32 float
constexpr size_t kOffBar = kOffB + 3 * 32 * 4;                          // 2 mbarriers + the tensor-memory address
constexpr size_t kEncSmem = kOffBar + 32;
static_assert(kOffCol % 128 == 0 && kOffPl2 % 128 == 0 && kOffPl3 % 128 == 0 && kOffW1 % 128 == 0 &&
              kOffW2 % 128 == 0 && kOffW3 % 128 == 0 && kOffBar % 8 == 0, "alignment");
static_assert(kEncSmem <= 227 * 1024, "shared memory");

// ---- head tile geometry (all on the block grid)
constexpr int kHTX = 10, kHTY = 8;
constexpr int kHP = kHTX + 6;                                // 16: the pitch of every plane
constexpr int kM4 = (kHTY + 4) * kHP, kM5 = (kHTY + 2) * kHP, kM6 = kHTY * kHP;   // 192, 160, 128
constexpr int kPin = kM4 - 1 + 2 * kHP + 2 + 1;              // 226
constexpr int kPl4 = kM5 - 1 + 2 * kHP + 2 + 1;              // 194
constexpr int kPl5 = kM6 - 1 + 2 * kHP + 2 + 1;              // 162
static_assert(kPin >= (kHTY + 6) * kHP && kPl4 >= kM4 && kPl5 >= kM5 && kM6 == 128, "head planes");
constexpr int kHeadThreads = 256;
constexpr size_t kHOffIn = 0;
constexpr size_t kHOffP4 = kHOffIn + (size_t)4 * kPin * 16;
constexpr size_t kHOffP5 = kHOffP4 + (size_t)4 * kPl4 * 16;
constexpr size_t kHOffW4 = kHOffP5 + (size_t)4 * kPl5 * 16;
constexpr size_t kHOffW5 = kHOffW4 + 36 * 32 * 16;
constexpr size_t kHOffW6 = kHOffW5 + 36 * 32 * 16;                      // [36 kc][16 n] x 16 B
constexpr size_t kHOffB = kHOffW6 + 36 * 16 * 16;                       // 32 + 32 + 8 float (+ padding)
constexpr size_t kHOffBar = kHOffB + 80 * 4;
constexpr size_t kHeadSmem = kHOffBar + 32;
static_assert(kHOffP4 % 128 == 0 && kHOffP5 % 128 == 0 && kHOffW4 % 128 == 0 && kHOffW5 % 128 == 0 &&
              kHOffW6 % 128 == 0 && kHOffBar % 8 == 0, "alignment");

__device__ __forceinline__ uint32_t packBf2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// 8 channels: bias, ReLU (or 0 outside the image), bf16
__device__ __forceinline__ uint4 actPack(const float v[8], const float* b, bool in) {
    float r[8];
#pragma unroll
    for (int i = 0; i < 8; i++) r[i] = in ? fmaxf(__fadd_rn(v[i], b[i]), 0.0f) : 0.0f;
    return make_uint4(packBf2(r[0], r[1]), packBf2(r[2], r[3]), packBf2(r[4], r[5]), packBf2(r[6], r[7]));
}

// a 32 -> N layer's bf16 weights [n][9][32] (global) into the canonical K-major layout [kc = k / 8][n][8]; rows
// n >= nValid are zero
template <int N, int kThreads>
__device__ __forceinline__ void stageW32(const bf16* __restrict__ w, int nValid, uint4* dst, int tid) {
    constexpr int kIt = (36 * N + kThreads - 1) / kThreads;
    uint4 v[kIt];
#pragma unroll
    for (int j = 0; j < kIt; j++) {   // all loads in flight before the first store
        const int i = tid + j * kThreads, kc = i / N, n = i % N;
        v[j] = i < 36 * N && n < nValid ? __ldg(reinterpret_cast<const uint4*>(w + (size_t)n * 288 + kc * 8)) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int j = 0; j < kIt; j++)
        if (tid + j * kThreads < 36 * N) dst[tid + j * kThreads] = v[j];
}

// chunk schedule: 128-row chunks covering [0, M), the last one moved back to end at M (rows recomputed, not read past)
__device__ __forceinline__ int chunkStart(int c, int M) { return min(c * 128, M - 128); }

// the chunk loop shared by every layer: issue(c, acc) by thread 0, then epilogue(c - 1) overlapping chunk c's MMAs,
// then prep(c + 1) (layer 1's im2col). Returns false (uniformly) when a wait gave up.
template <class Issue, class Epi, class Prep>
__device__ __forceinline__ bool chunkLoop(int n, uint64_t* bars, uint32_t* phase, Issue issue, Epi epi, Prep prep) {
    bool ok = true;
    for (int c = 0; c <= n; c++) {
        if (c < n) {
            fenceAsyncShared();
            tcFenceBefore();
            ok = __syncthreads_and(ok);
            if (!ok) return false;
            if (threadIdx.x == 0) {
                tcFenceAfter();
                issue(c, c & 1);
                tcCommit(&bars[c & 1]);
            }
        }
        if (c >= 1) {
            const int b = (c - 1) & 1;
            ok = mbarWait(&bars[b], phase[b], kWaitNs) && ok;
            phase[b] ^= 1u;
            tcFenceAfter();
            if (ok) epi(c - 1, b);
        }
        if (c + 1 < n) prep(c + 1, (c + 1) & 1);
    }
    return __syncthreads_and(ok);
}

}  // namespace

__global__ void __launch_bounds__(kEncThreads, 1) k_sn_enc(const SnFusedArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    uint32_t* luma = reinterpret_cast<uint32_t*>(sm + kOffLuma);
    uint4* col = reinterpret_cast<uint4*>(sm + kOffCol);
    uint4* pl2 = reinterpret_cast<uint4*>(sm + kOffPl2);
    uint4* pl3 = reinterpret_cast<uint4*>(sm + kOffPl3);
    bf16* w1 = reinterpret_cast<bf16*>(sm + kOffW1);
    float* bias = reinterpret_cast<float*>(sm + kOffB);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kOffBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kOffBar + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bz = blockIdx.z;
    const int cx0 = blockIdx.x * kEncTX, cy0 = blockIdx.y * kEncTY;

    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (warp == 0) tmemAlloc(tslot, 64);
    if (tid == 0) {
        mbarInit(&bars[0], 1);
        mbarInit(&bars[1], 1);
    }
    // weights and biases (not produced by the preceding kernels)
    {
        const bf16* __restrict__ wg = reinterpret_cast<const bf16*>(a.wb);
        bf16 v1[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {   // layer 1: K = 18 (tap * 2 + ci), padded to 32; 4 x 32 x 8 = 2 x 512 entries
            const int i = tid + j * kEncThreads, kc = i >> 8, n = (i >> 3) & 31, e = i & 7, k = kc * 8 + e;
            v1[j] = k < 18 ? wg[kW[0] + n * 18 + k] : __float2bfloat16(0.0f);
        }
        const float bv = tid < 96 ? a.p[(tid < 32 ? kB[0] : tid < 64 ? kB[1] : kB[2]) + (tid & 31)] : 0.0f;
        stageW32<32, kEncThreads>(wg + kW[1], 32, reinterpret_cast<uint4*>(sm + kOffW2), tid);
        stageW32<32, kEncThreads>(wg + kW[2], 32, reinterpret_cast<uint4*>(sm + kOffW3), tid);
        w1[tid] = v1[0];
        w1[tid + kEncThreads] = v1[1];
        if (tid < 96) bias[tid] = bv;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // the luma region, normalised ((v - 128) / 64, bf16), zero outside the level
    {
        const int ly0 = 8 * cy0 - 7, lx0 = 8 * cx0 - 7;
        const float* __restrict__ la = a.xp ? nullptr : a.la + (size_t)bz * a.h * a.w;
        const float* __restrict__ lc = a.xp ? nullptr : a.lc + (size_t)bz * a.h * a.w;
        constexpr int kIt = (kR0y * kP0 + kEncThreads - 1) / kEncThreads;
        float va[kIt], vc[kIt];
        uint32_t vx[kIt];
#pragma unroll
        for (int j = 0; j < kIt; j++) {   // every load first, then the conversions and stores
            const int i = tid + j * kEncThreads, y = i / kP0, x = i % kP0, gy = ly0 + y, gx = lx0 + x;
            const bool in = i < kR0y * kP0 && x < kR0x && gy >= 0 && gy < a.h && gx >= 0 && gx < a.w;
            const size_t o = in ? (size_t)gy * a.w + gx : 0;
            vx[j] = 0u;
            va[j] = vc[j] = 128.0f;   // (v - 128) / 64 = 0 outside the level
            if (in) {
                if (a.xp) vx[j] = __ldg(a.xp + (size_t)bz * a.h * a.w + o);
                else {
                    va[j] = __ldg(la + o);
                    vc[j] = __ldg(lc + o);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kIt; j++) {
            const int i = tid + j * kEncThreads;
            if (i < kR0y * kP0)
                luma[i] = a.xp ? vx[j]
                               : packBf2(__fmul_rn(__fsub_rn(va[j], 128.0f), 1.0f / 64.0f),
                                         __fmul_rn(__fsub_rn(vc[j], 128.0f), 1.0f / 64.0f));
        }
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tbase = *tslot;
    uint32_t phase[2] = {0u, 0u};
    const int q = warp & 3, part = warp >> 2;          // lanes 32 q .. + 31, columns 8 part .. + 7
    const int row = 32 * q + lane;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;
    const uint32_t idesc = tcIdescBf16(128, 32);

    // layer 1: im2col of chunk c (row r = tid & 127, k-chunk tid >> 7: taps 4 kc .. 4 kc + 3, 2 channels each)
    auto prep1 = [&](int c, int buf) {
        const int r = tid & 127, kc = tid >> 7;
        const int m = chunkStart(c, kM1) + r, oy = m / kP1, ox = m % kP1;
        uint32_t v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int tap = kc * 4 + j;
            v[j] = (tap < 9 && ox < kR1x) ? luma[(2 * oy + tap / 3) * kP0 + 2 * ox + tap % 3] : 0u;
        }
        col[(buf * 4 + kc) * 128 + r] = make_uint4(v[0], v[1], v[2], v[3]);
    };
    auto issue1 = [&](int c, int acc) {
        const uint32_t cb = smemAddr(col + (size_t)(c & 1) * 4 * 128), wb = smemAddr(w1);
        for (int j = 0; j < 2; j++)
            tcMma(tbase + 32 * acc, tcDesc(cb + j * 2 * 2048, 2048, 128), tcDesc(wb + j * 2 * 512, 512, 128), idesc, j);
    };
    auto epi1 = [&](int c, int acc) {
        float v[8];
        tmemLd8(tbase + tlane + 32 * acc + 8 * part, v);
        const int m = chunkStart(c, kM1) + row, oy = m / kP1, ox = m % kP1;
        if (ox < kR1x) {
            const int gy = 4 * cy0 - 3 + oy, gx = 4 * cx0 - 3 + ox;
            const bool in = gy >= 0 && gy < a.h1 && gx >= 0 && gx < a.w1;
            const int ph = ((oy & 1) << 1) | (ox & 1);
            const uint4 val = actPack(v, bias + 8 * part, in);
            pl2[(ph * 4 + part) * kPl2 + (oy >> 1) * kP2 + (ox >> 1)] = val;
            if (a.act[0] && in && gy >= 4 * cy0 && gy < 4 * (cy0 + kEncTY) && gx >= 4 * cx0 && gx < 4 * (cx0 + kEncTX))
                reinterpret_cast<uint4*>(a.act[0])[(((size_t)bz * a.h1 + gy) * a.w1 + gx) * 4 + part] = val;
        }
    };
    prep1(0, 0);
    bool ok = chunkLoop(kNC1, bars, phase, issue1, epi1, prep1);

    // layers 2 and 3: stride 2 over phase planes
    auto issueS2 = [&](const uint4* planes, int plLen, int P, const uint4* w, int m0, int acc) {
        const uint32_t pb = smemAddr(planes), wb = smemAddr(w);
        for (int t = 0; t < 9; t++) {
            const int ky = t / 3, kx = t % 3, ph = ((ky & 1) << 1) | (kx & 1), off = (ky >> 1) * P + (kx >> 1);
            for (int j = 0; j < 2; j++) {
                const uint32_t aa = pb + (uint32_t)(((ph * 4 + 2 * j) * plLen + m0 + off) * 16);
                tcMma(tbase + 32 * acc, tcDesc(aa, (uint32_t)plLen * 16, 128), tcDesc(wb + (t * 4 + 2 * j) * 512, 512, 128),
                      idesc, (t | j) != 0);
            }
        }
    };
    auto issue2 = [&](int c, int acc) {
        issueS2(pl2, kPl2, kP2, reinterpret_cast<const uint4*>(sm + kOffW2), chunkStart(c, kM2), acc);
    };
    auto epi2 = [&](int c, int acc) {
        float v[8];
        tmemLd8(tbase + tlane + 32 * acc + 8 * part, v);
        const int m = chunkStart(c, kM2) + row, oy = m / kP2, ox = m % kP2;
        if (ox < kR2x) {
            const int gy = 2 * cy0 - 1 + oy, gx = 2 * cx0 - 1 + ox;
            const bool in = gy >= 0 && gy < a.h2 && gx >= 0 && gx < a.w2;
            const int ph = ((oy & 1) << 1) | (ox & 1);
            const uint4 val = actPack(v, bias + 32 + 8 * part, in);
            pl3[(ph * 4 + part) * kPl3 + (oy >> 1) * kP3 + (ox >> 1)] = val;
            if (a.act[1] && in && gy >= 2 * cy0 && gy < 2 * (cy0 + kEncTY) && gx >= 2 * cx0 && gx < 2 * (cx0 + kEncTX))
                reinterpret_cast<uint4*>(a.act[1])[(((size_t)bz * a.h2 + gy) * a.w2 + gx) * 4 + part] = val;
        }
    };
    auto none = [&](int, int) {};
    if (ok) ok = chunkLoop(kNC2, bars, phase, issue2, epi2, none);

    auto issue3 = [&](int, int acc) { issueS2(pl3, kPl3, kP3, reinterpret_cast<const uint4*>(sm + kOffW3), 0, acc); };
    auto epi3 = [&](int, int acc) {
        float v[8];
        tmemLd8(tbase + tlane + 32 * acc + 8 * part, v);
        const int oy = row / kP3, ox = row % kP3, cy = cy0 + oy, cx = cx0 + ox;
        if (row < kM3 && ox < kEncTX && cy < a.h3 && cx < a.w3)
            reinterpret_cast<uint4*>(a.y3)[(((size_t)bz * a.h3 + cy) * a.w3 + cx) * 4 + part] = actPack(v, bias + 64 + 8 * part, true);
    };
    if (ok) ok = chunkLoop(1, bars, phase, issue3, epi3, none);

    if (!ok) {   // a wait gave up: record it, give the MMAs issued so far one more bounded wait, then free
        if (tid == 0) atomicOr(a.err, kErrSeedNet);
        for (int b = 0; b < 2; b++) mbarWait(&bars[b], phase[b], kWaitNs);
    }
    tcFenceBefore();
    __syncthreads();
    if (warp == 0) {
        tcFenceAfter();
        tmemFree(tbase, 64);
    }
}

__global__ void __launch_bounds__(kHeadThreads) k_sn_head(const SnFusedArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    uint4* pin = reinterpret_cast<uint4*>(sm + kHOffIn);
    uint4* p4 = reinterpret_cast<uint4*>(sm + kHOffP4);
    uint4* p5 = reinterpret_cast<uint4*>(sm + kHOffP5);
    float* bias = reinterpret_cast<float*>(sm + kHOffB);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kHOffBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kHOffBar + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bz = blockIdx.z;
    const int cx0 = blockIdx.x * kHTX, cy0 = blockIdx.y * kHTY;

    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (warp == 0) tmemAlloc(tslot, 64);
    if (tid == 0) {
        mbarInit(&bars[0], 1);
        mbarInit(&bars[1], 1);
    }
    {
        const bf16* __restrict__ wg = reinterpret_cast<const bf16*>(a.wb);
        const float bv = tid < 64 ? a.p[(tid < 32 ? kB[3] : kB[4]) + (tid & 31)] : tid < 64 + kSnOut ? a.p[kB[5] + tid - 64] : 0.0f;
        stageW32<32, kHeadThreads>(wg + kW[3], 32, reinterpret_cast<uint4*>(sm + kHOffW4), tid);
        stageW32<32, kHeadThreads>(wg + kW[4], 32, reinterpret_cast<uint4*>(sm + kHOffW5), tid);
        stageW32<16, kHeadThreads>(wg + kW[5], kSnOut, reinterpret_cast<uint4*>(sm + kHOffW6), tid);
        if (tid < 64 + kSnOut) bias[tid] = bv;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // layer 3's cells around the tile
    {
        const uint4* __restrict__ y3 = reinterpret_cast<const uint4*>(a.y3);
        constexpr int kN = (kHTY + 6) * kHP * 4, kIt = (kN + kHeadThreads - 1) / kHeadThreads;
        uint4 v[kIt];
#pragma unroll
        for (int j = 0; j < kIt; j++) {   // every load first, then the stores
            const int i = tid + j * kHeadThreads, c8 = i & 3, pix = i >> 2, y = pix / kHP, x = pix % kHP;
            const int gy = cy0 - 3 + y, gx = cx0 - 3 + x;
            v[j] = make_uint4(0, 0, 0, 0);
            if (i < kN && gy >= 0 && gy < a.h3 && gx >= 0 && gx < a.w3) v[j] = y3[(((size_t)bz * a.h3 + gy) * a.w3 + gx) * 4 + c8];
        }
#pragma unroll
        for (int j = 0; j < kIt; j++) {
            const int i = tid + j * kHeadThreads;
            if (i < kN) pin[(i & 3) * kPin + (i >> 2)] = v[j];
        }
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tbase = *tslot;
    uint32_t phase[2] = {0u, 0u};
    const int q = warp & 3, part = warp >> 2;          // lanes 32 q .. + 31, columns 16 part .. + 15 (layer 6: 8)
    const int row = 32 * q + lane;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;

    auto issueS1 = [&](const uint4* planes, int plLen, const uint4* w, int N, int m0, int acc) {
        const uint32_t pb = smemAddr(planes), wb = smemAddr(w), idesc = tcIdescBf16(128, N);
        for (int t = 0; t < 9; t++) {
            const int off = (t / 3) * kHP + t % 3;
            for (int j = 0; j < 2; j++)
                tcMma(tbase + 32 * acc, tcDesc(pb + (uint32_t)(((2 * j) * plLen + m0 + off) * 16), (uint32_t)plLen * 16, 128),
                      tcDesc(wb + (t * 4 + 2 * j) * N * 16, (uint32_t)N * 16, 128), idesc, (t | j) != 0);
        }
    };
    // layers 4, 5: the layer's region starts d cells before the tile; columns >= validX are the padded raster's
    auto epiS1 = [&](uint4* dst, int plLen, int M, int d, int validX, const float* b, void* act, int c, int acc) {
        float v[16];
        tmemLd16(tbase + tlane + 32 * acc + 16 * part, v);
        const int m = chunkStart(c, M) + row, oy = m / kHP, ox = m % kHP;
        const int gy = cy0 - d + oy, gx = cx0 - d + ox;
        const bool in = ox < validX && gy >= 0 && gy < a.h3 && gx >= 0 && gx < a.w3;
        const uint4 v0 = actPack(v, b + 16 * part, in), v1 = actPack(v + 8, b + 16 * part + 8, in);
        dst[(2 * part) * plLen + m] = v0;
        dst[(2 * part + 1) * plLen + m] = v1;
        if (act && in && gy >= cy0 && gy < cy0 + kHTY && gx >= cx0 && gx < cx0 + kHTX) {
            uint4* o = reinterpret_cast<uint4*>(act) + (((size_t)bz * a.h3 + gy) * a.w3 + gx) * 4 + 2 * part;
            o[0] = v0;
            o[1] = v1;
        }
    };
    auto none = [&](int, int) {};
    auto issue4 = [&](int c, int acc) { issueS1(pin, kPin, reinterpret_cast<const uint4*>(sm + kHOffW4), 32, chunkStart(c, kM4), acc); };
    auto epi4 = [&](int c, int acc) { epiS1(p4, kPl4, kM4, 2, kHP - 2, bias, a.act[3], c, acc); };
    bool ok = chunkLoop((kM4 + 127) / 128, bars, phase, issue4, epi4, none);
    auto issue5 = [&](int c, int acc) { issueS1(p4, kPl4, reinterpret_cast<const uint4*>(sm + kHOffW5), 32, chunkStart(c, kM5), acc); };
    auto epi5 = [&](int c, int acc) { epiS1(p5, kPl5, kM5, 1, kHP - 4, bias + 32, a.act[4], c, acc); };
    if (ok) ok = chunkLoop((kM5 + 127) / 128, bars, phase, issue5, epi5, none);
    auto issue6 = [&](int, int acc) { issueS1(p5, kPl5, reinterpret_cast<const uint4*>(sm + kHOffW6), 16, 0, acc); };
    auto epi6 = [&](int, int acc) {
        if (part != 0) return;   // columns 8..15 are the zero padding of N = 16
        float v[8];
        tmemLd8(tbase + tlane + 32 * acc, v);
        const int oy = row / kHP, ox = row % kHP, cy = cy0 + oy, cx = cx0 + ox;
        if (ox < kHTX && cy < a.h3 && cx < a.w3) {
            float4* o = reinterpret_cast<float4*>(a.out + (((size_t)bz * a.h3 + cy) * a.w3 + cx) * kSnOut);
            o[0] = make_float4(__fadd_rn(v[0], bias[64]), __fadd_rn(v[1], bias[65]), __fadd_rn(v[2], bias[66]), __fadd_rn(v[3], bias[67]));
            o[1] = make_float4(__fadd_rn(v[4], bias[68]), __fadd_rn(v[5], bias[69]), __fadd_rn(v[6], bias[70]), __fadd_rn(v[7], bias[71]));
        }
    };
    if (ok) ok = chunkLoop(1, bars, phase, issue6, epi6, none);

    if (!ok) {
        if (tid == 0) atomicOr(a.err, kErrSeedNet);
        for (int b = 0; b < 2; b++) mbarWait(&bars[b], phase[b], kWaitNs);
    }
    tcFenceBefore();
    __syncthreads();
    if (warp == 0) {
        tcFenceAfter();
        tmemFree(tbase, 64);
    }
}

cudaError_t prepareSeedNetFused() {
    cudaError_t e = cudaFuncSetAttribute(k_sn_enc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEncSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sn_head, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHeadSmem);
    return e;
}

cudaError_t launchSnFused(const SnFusedArgs& a, cudaStream_t s) {
    const dim3 ge((a.w3 + kEncTX - 1) / kEncTX, (a.h3 + kEncTY - 1) / kEncTY, a.B);
    cudaError_t e = launchPdl(k_sn_enc, ge, dim3(kEncThreads), kEncSmem, s, a);
    if (e != cudaSuccess) return e;
    const dim3 gh((a.w3 + kHTX - 1) / kHTX, (a.h3 + kHTY - 1) / kHTY, a.B);
    return launchPdl(k_sn_head, gh, dim3(kHeadThreads), kHeadSmem, s, a);
}

}  // namespace fgk
