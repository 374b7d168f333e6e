// Host side of the seed proposer (fg_seednet.cu): its parameters, workspace, forward pass, training step (loss,
// backward, Adam) behind the C ABI of include/framegen_c.h (fg_seednet_*). No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fg_seednet.h"
#include "framegen_c.h"

namespace {

using namespace fgk;

inline int ceilHalf(int v) { return (v + 1) / 2; }

// the output grid of every layer for an input of h x w
struct SnDims {
    int h[kSnLayers + 1], w[kSnLayers + 1];
    SnDims(int H, int W) {
        h[0] = H; w[0] = W;
        for (int l = 0; l < kSnLayers; l++) {
            h[l + 1] = kSnStride[l] == 2 ? ceilHalf(h[l]) : h[l];
            w[l + 1] = kSnStride[l] == 2 ? ceilHalf(w[l]) : w[l];
        }
    }
};

uint16_t toBf16(float f) {   // round to nearest even (finite inputs)
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

struct DevScope {   // makes `dev` current for the scope
    int old = -1;
    explicit DevScope(int dev) {
        if (cudaGetDevice(&old) == cudaSuccess && old != dev) cudaSetDevice(dev);
        else old = -1;
    }
    ~DevScope() {
        if (old >= 0) cudaSetDevice(old);
    }
};

}  // namespace

struct fg_seednet {
    int device = 0;
    int maxB = 0, maxH = 0, maxW = 0;
    char* mem = nullptr;
    float* p = nullptr;       // float32 master parameters
    uint16_t* wb = nullptr;   // their bfloat16 copy
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    float* loss = nullptr;
    void* act[kSnLayers - 1] = {};   // bf16 outputs of layers 1..5
    unsigned int* errFlags = nullptr;   // the fused forward's sticky error bits (kErrSeedNet) when no other is given
    float* part = nullptr;              // the weight gradient's per-CTA partial sums
    int partCtas = 0;
    float* out = nullptr;            // last layer (float)
    float* dA = nullptr;             // gradient ping-pong buffers (float)
    float* dB = nullptr;
    int step = 0;
    const char* err = nullptr;
    char errBuf[160] = {};

    bool ok(cudaError_t e, const char* where = nullptr, int layer = -1) {
        if (e == cudaSuccess) return true;
        cudaGetLastError();
        if (where) {
            std::snprintf(errBuf, sizeof(errBuf), "%s (%s, layer %d)", cudaGetErrorString(e), where, layer + 1);
            err = errBuf;
        } else {
            err = cudaGetErrorString(e);
        }
        return false;
    }
    bool fits(int B, int H, int W) const { return B >= 1 && H >= 1 && W >= 1 && B <= maxB && H <= maxH && W <= maxW; }

    // the arguments of every layer. x: the packed input, or null with la / lc: the float luma planes read by the
    // first layer directly
    void layerArgs(SnConvArgs* args, const void* x, int B, int H, int W, float* dst, const float* la, const float* lc) {
        const SnDims d(H, W);
        const void* in = x;
        for (int l = 0; l < kSnLayers; l++) {
            SnConvArgs& a = args[l];
            a = SnConvArgs{};
            a.x = in;
            if (l == 0) { a.la = la; a.lc = lc; }
            a.w = wb + snWeightOff(l);
            a.b = p + snBiasOff(l);
            a.y = l < kSnLayers - 1 ? act[l] : nullptr;
            a.yf = l == kSnLayers - 1 ? dst : nullptr;
            a.B = B; a.H = d.h[l]; a.W = d.w[l]; a.Ho = d.h[l + 1]; a.Wo = d.w[l + 1];
            if (l < kSnLayers - 1) in = act[l];
        }
    }

    // one launch per layer (PDL-chained)
    bool forward(cudaStream_t s, const void* x, int B, int H, int W, float* dst, const float* la = nullptr,
                 const float* lc = nullptr) {
        SnConvArgs args[kSnLayers];
        layerArgs(args, x, B, H, W, dst, la, lc);
        for (int l = 0; l < kSnLayers; l++)
            if (!ok(launchSnConv(l, args[l], s), "forward", l)) return false;
        return true;
    }

    // the fused forward on the tensor cores (two launches, fg_seednet_tc.cu) from the float luma planes or (xp) the
    // packed input; keep: also store layers 1-5's outputs (the backward's inputs)
    bool forwardFused(cudaStream_t s, int B, int H, int W, float* dst, const float* la, const float* lc,
                      unsigned int* errOut, const void* xp = nullptr, bool keep = false) {
        const SnDims d(H, W);
        SnFusedArgs a{};
        a.la = la; a.lc = lc; a.wb = wb; a.p = p; a.y3 = act[2]; a.out = dst;
        a.xp = static_cast<const uint32_t*>(xp);
        if (keep)
            for (int l = 0; l < kSnLayers - 1; l++) a.act[l] = act[l];
        a.B = B; a.h = H; a.w = W;
        a.h1 = d.h[1]; a.w1 = d.w[1]; a.h2 = d.h[2]; a.w2 = d.w[2]; a.h3 = d.h[3]; a.w3 = d.w[3];
        a.err = errOut ? errOut : errFlags;
        return ok(launchSnFused(a, s), "fused forward");
    }

    bool backward(cudaStream_t s, const void* x, int B, int H, int W, const float* targets) {
        const SnDims d(H, W);
        const int nb = B * d.h[kSnLayers] * d.w[kSnLayers];
        if (!forwardFused(s, B, H, W, out, nullptr, nullptr, nullptr, x, true)) return false;   // keeps layers 1-5
        if (!ok(cudaMemsetAsync(loss, 0, sizeof(float), s))) return false;
        float* dy = dA;
        if (!ok(launchSnLoss(out, targets, nb, dy, loss, 1.0f / (float)nb, s), "loss")) return false;
        for (int l = kSnLayers - 1; l >= 0; l--) {
            SnBackArgs a{};
            a.x = l == 0 ? x : act[l - 1];
            a.w = wb + snWeightOff(l);
            a.dy = dy;
            a.dx = dy == dA ? dB : dA;
            a.dw = grad + snWeightOff(l);
            a.db = grad + snBiasOff(l);
            a.B = B; a.H = d.h[l]; a.W = d.w[l]; a.Ho = d.h[l + 1]; a.Wo = d.w[l + 1];
            a.part = part; a.partCtas = partCtas;
            if (!ok(launchSnBackwardTc(l, a, l > 0, errFlags, s), "backward", l)) return false;
            dy = a.dx;
        }
        return true;
    }
};

namespace fgk {
bool seedNetForwardLuma(::fg_seednet* n, cudaStream_t s, const float* la, const float* lc, int h, int w, float* out,
                        unsigned int* err, const char** why) {
    if (!n || !n->fits(1, h, w)) { *why = "seed net workspace too small"; return false; }
    DevScope g(n->device);
    if (n->forwardFused(s, 1, h, w, out, la, lc, err)) return true;
    *why = n->err;
    return false;
}
}  // namespace fgk

extern "C" {

uint32_t fg_seednet_param_count(void) { return (uint32_t)kSnParams; }

fg_seednet* fg_seednet_create(int device, int max_batch, int max_h, int max_w) {
    if (max_batch < 1 || max_h < 1 || max_w < 1) return nullptr;
    int old = -1;
    if (cudaGetDevice(&old) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    fg_seednet* n = new fg_seednet();
    n->device = device >= 0 ? device : old;
    n->maxB = max_batch; n->maxH = max_h; n->maxW = max_w;
    const SnDims d(max_h, max_w);
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) / 256 * 256; return o; };
    const size_t P = kSnParams;
    const size_t oP = take(P * 4), oW = take(P * 2), oM = take(P * 4), oV = take(P * 4), oG = take(P * 4), oL = take(4);
    size_t oAct[kSnLayers - 1];
    size_t maxGrad = (size_t)max_batch * d.h[kSnLayers] * d.w[kSnLayers] * kSnOut;
    for (int l = 0; l < kSnLayers - 1; l++) {
        const size_t e = (size_t)max_batch * d.h[l + 1] * d.w[l + 1] * kSnCout[l];
        oAct[l] = take(e * 2);
        maxGrad = std::max(maxGrad, e);
    }
    const size_t oOut = take((size_t)max_batch * d.h[kSnLayers] * d.w[kSnLayers] * kSnOut * 4);
    const size_t oErr = take(4);
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device) != cudaSuccess) { cudaGetLastError(); sms = 148; }
    n->partCtas = 2 * sms;
    const size_t oPart = take((size_t)n->partCtas * kSnPartFloats * 4);
    const size_t oDA = take(maxGrad * 4), oDB = take(maxGrad * 4);
    if (cudaMalloc(&n->mem, off) != cudaSuccess) {
        cudaGetLastError();
        delete n;
        cudaSetDevice(old);
        return nullptr;
    }
    cudaMemset(n->mem, 0, off);
    n->p = (float*)(n->mem + oP); n->wb = (uint16_t*)(n->mem + oW); n->m = (float*)(n->mem + oM);
    n->v = (float*)(n->mem + oV); n->grad = (float*)(n->mem + oG); n->loss = (float*)(n->mem + oL);
    for (int l = 0; l < kSnLayers - 1; l++) n->act[l] = n->mem + oAct[l];
    n->out = (float*)(n->mem + oOut);
    n->errFlags = (unsigned int*)(n->mem + oErr);
    n->part = (float*)(n->mem + oPart);
    if (prepareSeedNetFused() != cudaSuccess || prepareSeedNetBackward() != cudaSuccess) {   // shared-memory limits
        cudaGetLastError();
        cudaFree(n->mem);
        delete n;
        cudaSetDevice(old);
        return nullptr;
    }
    n->dA = (float*)(n->mem + oDA); n->dB = (float*)(n->mem + oDB);
    cudaDeviceSynchronize();
    cudaSetDevice(old);
    return n;
}

void fg_seednet_destroy(fg_seednet* n) {
    if (!n) return;
    int old = -1;
    cudaGetDevice(&old);
    cudaSetDevice(n->device);
    cudaFree(n->mem);
    cudaSetDevice(old);
    delete n;
}

const char* fg_seednet_error(const fg_seednet* n) { return n ? n->err : "no net"; }

int fg_seednet_set_params(fg_seednet* n, const float* host) {
    if (!n || !host) return 0;
    std::vector<uint16_t> b(kSnParams);
    for (int i = 0; i < kSnParams; i++) b[i] = toBf16(host[i]);
    int old = -1;
    cudaGetDevice(&old);
    cudaSetDevice(n->device);
    const bool r = n->ok(cudaMemcpy(n->p, host, (size_t)kSnParams * 4, cudaMemcpyHostToDevice)) &&
                   n->ok(cudaMemcpy(n->wb, b.data(), (size_t)kSnParams * 2, cudaMemcpyHostToDevice)) &&
                   n->ok(cudaMemset(n->m, 0, (size_t)kSnParams * 4)) && n->ok(cudaMemset(n->v, 0, (size_t)kSnParams * 4)) &&
                   n->ok(cudaMemset(n->grad, 0, (size_t)kSnParams * 4));
    n->step = 0;
    cudaSetDevice(old);
    return r;
}

int fg_seednet_get_params(fg_seednet* n, float* host) {
    if (!n || !host) return 0;
    DevScope g(n->device);
    return n->ok(cudaMemcpy(host, n->p, (size_t)kSnParams * 4, cudaMemcpyDeviceToHost));
}

int fg_seednet_get_grads(fg_seednet* n, float* host) {
    if (!n || !host) return 0;
    DevScope g(n->device);
    return n->ok(cudaMemcpy(host, n->grad, (size_t)kSnParams * 4, cudaMemcpyDeviceToHost));
}

int fg_seednet_pack(void* stream, const float* luma_prev, const float* luma_curr, int n, void* x) {
    if (!luma_prev || !luma_curr || !x || n < 1) return 0;
    return launchSnPack(luma_prev, luma_curr, n, x, (cudaStream_t)stream) == cudaSuccess;
}

int fg_seednet_forward(fg_seednet* n, void* stream, const void* x, int batch, int h, int w, float* out) {
    if (!n || !x || !out || !n->fits(batch, h, w)) return 0;
    DevScope g(n->device);
    return n->forward((cudaStream_t)stream, x, batch, h, w, out);
}

int fg_seednet_forward_luma(fg_seednet* n, void* stream, const float* luma_prev, const float* luma_curr, int batch, int h,
                           int w, float* out) {
    if (!n || !luma_prev || !luma_curr || !out || !n->fits(batch, h, w)) return 0;
    DevScope g(n->device);
    return n->forward((cudaStream_t)stream, nullptr, batch, h, w, out, luma_prev, luma_curr);
}

int fg_seednet_forward_fused(fg_seednet* n, void* stream, const float* luma_prev, const float* luma_curr, int batch,
                            int h, int w, float* out) {
    if (!n || !luma_prev || !luma_curr || !out || !n->fits(batch, h, w)) return 0;
    DevScope g(n->device);
    return n->forwardFused((cudaStream_t)stream, batch, h, w, out, luma_prev, luma_curr, nullptr);
}

uint32_t fg_seednet_fused_errors(fg_seednet* n) {
    if (!n) return UINT32_MAX;
    DevScope g(n->device);
    uint32_t v = 0;
    if (!n->ok(cudaMemcpy(&v, n->errFlags, 4, cudaMemcpyDeviceToHost))) return UINT32_MAX;
    return v;
}

int fg_seednet_backward(fg_seednet* n, void* stream, const void* x, int batch, int h, int w, const float* targets,
                        float* loss) {
    if (!n || !x || !targets || !n->fits(batch, h, w)) return 0;
    DevScope g(n->device);
    if (!n->backward((cudaStream_t)stream, x, batch, h, w, targets)) return 0;
    if (loss) return n->ok(cudaMemcpyAsync(loss, n->loss, 4, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return 1;
}

int fg_seednet_zero_grads(fg_seednet* n, void* stream) {
    if (!n) return 0;
    DevScope g(n->device);
    return n->ok(cudaMemsetAsync(n->grad, 0, (size_t)kSnParams * 4, (cudaStream_t)stream));
}

float* fg_seednet_grad_buffer(fg_seednet* n) { return n ? n->grad : nullptr; }

int fg_seednet_adam(fg_seednet* n, void* stream, float lr) { return fg_seednet_adam_scaled(n, stream, lr, 1.0f); }

int fg_seednet_adam_scaled(fg_seednet* n, void* stream, float lr, float grad_scale) {
    if (!n) return 0;
    DevScope g(n->device);
    n->step++;
    SnAdamArgs a{};
    a.p = n->p; a.m = n->m; a.v = n->v; a.grad = n->grad; a.wb = n->wb; a.n = kSnParams;
    a.lr = lr; a.b1 = 0.9f; a.b2 = 0.999f; a.eps = 1e-8f; a.gscale = grad_scale;
    a.c1 = (float)(1.0 / (1.0 - std::pow(0.9, n->step)));
    a.c2 = (float)(1.0 / (1.0 - std::pow(0.999, n->step)));
    return n->ok(launchSnAdam(a, (cudaStream_t)stream));
}

}  // extern "C"
