// fg_seednet.h -- the seed proposer's parameter layout and kernel arguments (fg_seednet.cu), shared with the host
// code (fg_seednet_host.cpp, framegen.cpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct fg_seednet;   // the C ABI's handle (framegen_c.h)

namespace fgk {

constexpr int kSnLayers = 6;
constexpr int kSnOut = 8;                   // per block: c1x, c1y, c2x, c2y, confidence logit, 3 unused
constexpr int kSnTargets = 6;               // per block: truth (2), search vector (2), weight, unused
constexpr int kSnCin[kSnLayers] = {2, 32, 32, 32, 32, 32};
constexpr int kSnCout[kSnLayers] = {32, 32, 32, 32, 32, kSnOut};
constexpr int kSnStride[kSnLayers] = {2, 2, 2, 1, 1, 1};

// the flat parameter array: per layer, weights [cout][9][cin] then biases [cout]
constexpr int snWeightOff(int l) { return l == 0 ? 0 : snWeightOff(l - 1) + kSnCout[l - 1] * (9 * kSnCin[l - 1] + 1); }
constexpr int snBiasOff(int l) { return snWeightOff(l) + kSnCout[l] * 9 * kSnCin[l]; }
constexpr int kSnParams = snWeightOff(kSnLayers);   // 39,912

struct SnConvArgs {
    const void* x;     // layer input, NHWC bf16 [B][H][W][cin]
    const void* w;     // bf16 [cout][9][cin]
    const float* b;    // float [cout]
    void* y;           // layer output, NHWC bf16 (ReLU layers)
    float* yf;         // last layer: float [B][Ho][Wo][8]
    int B, H, W, Ho, Wo;
    const float* la;   // layer 1 only, optional: read the float luma planes (prev, curr) instead of x
    const float* lc;
};

struct SnBackArgs {
    const void* x;     // layer input (bf16), the previous layer's ReLU output (its mask for dx)
    const void* w;     // bf16 weights of this layer
    const float* dy;   // gradient at this layer's pre-activation, float [B][Ho][Wo][cout]
    float* dx;         // gradient at the previous layer's pre-activation, float [B][H][W][cin]
    float* dw;         // += dL/dW, float [cout][9][cin]
    float* db;         // += dL/db, float [cout]
    int B, H, W, Ho, Wo;
    float* part;       // the weight gradient's per-CTA partial sums (kSnPartFloats per CTA, up to partCtas CTAs)
    int partCtas;
};
constexpr int kSnPartFloats = (9 * 32 + 1) * 32;   // rows (tap, ci) + the bias row, times cout, of the widest layer

struct SnAdamArgs {
    float* p; float* m; float* v; float* grad;   // float32 master parameters, moments, gradients (zeroed here)
    void* wb;                                    // bf16 copy of p (the forward's weights)
    int n;
    float lr, b1, b2, eps, c1, c2;               // c1 = 1 / (1 - b1^t), c2 = 1 / (1 - b2^t)
    float gscale;                                // the gradient is read as grad * gscale (1 / ranks after a sum)
};

// the fused forward (fg_seednet_tc.cu, tensor cores): B images of h x w float luma (prev, curr) -> per block 8 floats
struct SnFusedArgs {
    const float* la; const float* lc;   // [B][h][w] each
    const uint32_t* xp;                 // or (when set) the packed input [B][h][w] (bf16 prev | bf16 curr << 16)
    void* act[5];                       // optional (training): layers 1-5's bf16 outputs [B][h_l][w_l][32]
    const void* wb;                     // bf16 parameters (the flat array)
    const float* p;                     // float parameters (the biases)
    void* y3;                           // layer 3's output, bf16 [B][h3][w3][32]
    float* out;                         // [B][h3][w3][kSnOut]
    int B, h, w, h1, w1, h2, w2, h3, w3;
    unsigned int* err;                  // kErrSeedNet is or-ed in when a tensor-core wait gave up
};
cudaError_t prepareSeedNetFused();
cudaError_t launchSnFused(const SnFusedArgs& a, cudaStream_t s);

cudaError_t launchSnPack(const float* la, const float* lc, int n, void* x, cudaStream_t s);
cudaError_t launchSnConv(int layer, const SnConvArgs& a, cudaStream_t s);
// the forward of a net (fg_seednet_host.cpp) for the Interpolator: one image of h x w from its float luma planes, on
// the fused tensor-core kernels; kErrSeedNet is or-ed into *err if a tensor-core wait gave up; *why = the failure's
// message
bool seedNetForwardLuma(::fg_seednet* n, cudaStream_t s, const float* la, const float* lc, int h, int w, float* out,
                        unsigned int* err, const char** why);
// one layer's weight / bias gradient (and its input gradient when needDx) on the tensor cores (fg_seednet_bwd.cu);
// kErrSeedNet into *err if a tensor-core wait gave up
cudaError_t prepareSeedNetBackward();
cudaError_t launchSnBackwardTc(int layer, const SnBackArgs& a, bool needDx, unsigned int* err, cudaStream_t s);
cudaError_t launchSnLoss(const float* out, const float* tgt, int n, float* dout, float* loss, float scale, cudaStream_t s);
cudaError_t launchSnAdam(const SnAdamArgs& a, cudaStream_t s);

}  // namespace fgk
