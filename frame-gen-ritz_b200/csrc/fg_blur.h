// Motion blur from stored sub-frames (8-bit RGBA / BGRA): the parameters and launcher of the blend that closes
// recordSynthBlur when each sample's synthesis was written to a sub-frame by the ordinary synthesis kernel.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fg_params.h"

namespace fgk {

struct BlurBlendParams {
    const uint8_t* a; const uint8_t* c; size_t pitch;   // prev, curr
    const uint8_t* sub; size_t subPitch, subStride;     // the sub-frame of slot j starts at sub + j * subStride
    uint8_t* out; size_t outPitch;
    int W, H, n;
    int mode[kBlurMax];      // 0: synthesized into sub-frame slot[k]; 1: the real frame prev (t_k <= 0); 2: curr
    int nearC[kBlurMax];     // mode 0: the sample's nearer frame is curr (t_k > 0.5)
    int slot[kBlurMax];
    uint32_t q[kBlurMax];    // weights, units of 2^-16, summing to 2^16
    double frac;             // globalFallback: a synthesized sample past it is its nearer real frame
    const unsigned int* cnt; // per sample, its synthesis' untrusted pixels
};

// out = (sum_k q_k frame_k + 2^15) >> 16 per byte; returns the launch's cudaError_t
cudaError_t launchBlurBlend(const BlurBlendParams& p, cudaStream_t s);

}  // namespace fgk
