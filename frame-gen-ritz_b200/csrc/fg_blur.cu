// fg_blur.cu -- the blend of recordSynthBlur's stored sub-frames (8-bit RGBA / BGRA).
//
// Motion blur (gpu/framegen.h:553-573, gpu/shaders/blur_resolve.comp) averages the frames recordSynth(t_k) gives at
// the sample times t_k. On this path each synthesized sample is written to its own sub-frame by the synthesis kernel
// itself (k_synth / k_synth_ui, full occupancy, counting the sample's untrusted pixels), and one HBM-bound pass here
// forms out = (sum_k q_k frame_k + 2^15) >> 16 per byte, the weights q_k integers summing to 2^16. frame_k is the
// sample's sub-frame, or its nearer real frame where the sample is a real instant (t_k <= 0 or >= 1) or flicked (more
// than globalFallback of its pixels untrusted, interp.py:238-239): the flick test is made here, from the counters, so
// the syntheses need no fallback pass. The alpha byte of every frame_k is its nearer frame's, so the output's is the
// weighted mean of prev's and curr's. The bytes equal those of the fused kernel k_synth_blur_t, which keeps every
// sample in registers instead (used when the sub-frames would not fit their memory cap).
#include <algorithm>

#include "fg_blur.h"
#include "fg_device.h"

namespace fgk {

constexpr int kBlendThreads = 256;

// kPx consecutive pixels of a row: one 16-byte access for 4 (the row 16-byte aligned, x a multiple of 4), else one word
template <int kPx>
__device__ __forceinline__ void loadPx(const uint8_t* row, int x, uint32_t (&v)[kPx]) {
    if constexpr (kPx == 4) {
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(row) + (x >> 2));
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
    } else {
        v[0] = __ldg(reinterpret_cast<const uint32_t*>(row) + x);
    }
}
template <int kPx>
__device__ __forceinline__ void storePx(uint8_t* row, int x, const uint32_t (&v)[kPx]) {
    if constexpr (kPx == 4) reinterpret_cast<uint4*>(row)[x >> 2] = make_uint4(v[0], v[1], v[2], v[3]);
    else reinterpret_cast<uint32_t*>(row)[x] = v[0];
}

// kPx pixels per thread (4: every row involved 16-byte aligned and W a multiple of 4, so each thread's 4 pixels are
// inside the row; 1 otherwise)
template <int kPx>
__global__ void __launch_bounds__(kBlendThreads) k_blur_blend(const __grid_constant__ BlurBlendParams p) {
    pdlEnter();   // the syntheses' sub-frames and counters are complete
    __shared__ const uint8_t* src[kBlurMax + 2];
    __shared__ size_t srcPitch[kBlurMax + 2];
    __shared__ uint32_t srcQ[kBlurMax + 2];
    __shared__ int nSrc;
    if (threadIdx.x < 32) {   // the source list: the kept sub-frames, then prev and curr with the replaced weights
        const int k = threadIdx.x;
        const bool live = k < p.n;
        const uint32_t q = live ? p.q[k] : 0u;
        bool repl = false, nc = false;
        if (live) {
            const int mode = p.mode[k];
            repl = mode != 0;
            nc = mode == 2 || (mode == 0 && p.nearC[k] != 0);
            if (!repl && (double)p.cnt[k] / ((double)p.W * (double)p.H) > p.frac) repl = true;
        }
        const unsigned int keep = __ballot_sync(~0u, live && !repl);
        const uint32_t wp = __reduce_add_sync(~0u, live && repl && !nc ? q : 0u);
        const uint32_t wc = __reduce_add_sync(~0u, live && repl && nc ? q : 0u);
        if (live && !repl) {
            const int j = __popc(keep & ((1u << k) - 1u));
            src[j] = p.sub + (size_t)p.slot[k] * p.subStride;
            srcPitch[j] = p.subPitch;
            srcQ[j] = q;
        }
        if (k == 0) {
            int j = __popc(keep);
            if (wp) { src[j] = p.a; srcPitch[j] = p.pitch; srcQ[j] = wp; j++; }
            if (wc) { src[j] = p.c; srcPitch[j] = p.pitch; srcQ[j] = wc; j++; }
            nSrc = j;
        }
    }
    __syncthreads();
    const int n = nSrc;
    const int x = (blockIdx.x * kBlendThreads + threadIdx.x) * kPx;   // this thread's first pixel
    if (x >= p.W) return;
    for (int y = blockIdx.y; y < p.H; y += gridDim.y) {
        // per byte: sum q_k v_k + 2^15 <= 255 * 2^16 + 2^15 < 2^24
        uint32_t sum[kPx][4];
#pragma unroll
        for (int i = 0; i < kPx; i++) sum[i][0] = sum[i][1] = sum[i][2] = sum[i][3] = 32768u;
#pragma unroll 4
        for (int k = 0; k < n; k++) {
            uint32_t v[kPx];
            loadPx<kPx>(src[k] + (size_t)y * srcPitch[k], x, v);
            const uint32_t q = srcQ[k];
#pragma unroll
            for (int i = 0; i < kPx; i++) {
                sum[i][0] += q * (v[i] & 255u);
                sum[i][1] += q * ((v[i] >> 8) & 255u);
                sum[i][2] += q * ((v[i] >> 16) & 255u);
                sum[i][3] += q * (v[i] >> 24);
            }
        }
        uint32_t o[kPx];
#pragma unroll
        for (int i = 0; i < kPx; i++)
            o[i] = (sum[i][0] >> 16) | ((sum[i][1] >> 16) << 8) | ((sum[i][2] >> 16) << 16) | ((sum[i][3] >> 16) << 24);
        storePx<kPx>(p.out + (size_t)y * p.outPitch, x, o);
    }
}

static bool aligned16(const void* ptr, size_t pitch) { return ((uintptr_t)ptr & 15u) == 0 && pitch % 16 == 0; }

cudaError_t launchBlurBlend(const BlurBlendParams& p, cudaStream_t s) {
    // a row segment of 256 threads per CTA, rows dealt out so that about 8 CTAs per SM cover the frame
    const bool vec = p.W % 4 == 0 && aligned16(p.a, p.pitch) && aligned16(p.c, p.pitch) &&
                     aligned16(p.sub, p.subPitch) && p.subStride % 16 == 0 && aligned16(p.out, p.outPitch);
    const int px = vec ? 4 : 1;
    const unsigned int gx = divUp(p.W / px + (p.W % px != 0), kBlendThreads);
    const unsigned int gy = (unsigned int)std::max(1, std::min(p.H, (int)std::max(1u, (unsigned int)smCount() * 8u / gx)));
    if (vec) return launchPdl(k_blur_blend<4>, dim3(gx, gy), dim3(kBlendThreads), 0, s, p);
    return launchPdl(k_blur_blend<1>, dim3(gx, gy), dim3(kBlendThreads), 0, s, p);
}

}  // namespace fgk
