// fg_record_synth_noalloc: the synthesis of one generated frame for callers that cannot allocate device memory.
//
// Some hosts of a frame generator may not call cudaMalloc at the point where they generate frames: a compositor or
// game overlay that runs inside another program's frame callback with a fixed memory budget owned by that program, a
// real-time presentation thread that must not block (cudaMalloc and cudaFree can synchronise the whole device and take
// milliseconds), or a plugin sandbox that hands the plugin device buffers but no allocator. Such a caller still owns its
// frames, the per-pixel half-vector field of the pair and the output, and passes them in; everything else this path
// needs lives in one statically sized device array that the library declares below.
//
// The scratch array (g_fgNoAllocScratch): a DevState (the scene-cut flag and the untrusted-pixel counters) and the
// per-pixel field looked up at time t, for at most kNoAllocMaxFlowPixels flow pixels (3,145,728: 3840x2160 at
// flowScale 2 needs 2,073,600). About 24 MiB on every GPU where it has been placed, held until the process exits.
// The driver places it when this file's module is first used on a device: with CUDA's default lazy module loading
// that is the first call's cudaGetSymbolAddress, so the first call on a device is where the 24 MiB are taken, and it
// can fail there for lack of device memory. Hosts with a fixed memory budget make that first call at set-up time.
// All calls share the array and it keeps the last call's contents: the counters are cleared by each call's first
// kernel, the field is rewritten in full. Calls that overlap on the GPU (two streams, or two threads) race on it.
//
// Host code does not use the array's name as an address (in host code it is only a stand-in for the symbol): the first
// call on a device, with that device current, looks the address up with cudaGetSymbolAddress and keeps it for that
// device (under a lock, so two host threads may make their first calls at once). That first call therefore does a
// little set-up work on the host and should come before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "fg_params.h"
#include "framegen.h"
#include "framegen_c.h"

namespace {

constexpr size_t kNoAllocMaxFlowPixels = size_t(3) << 20;
constexpr size_t kNoAllocStateBytes = 256;   // the DevState, padded to the field's alignment
static_assert(sizeof(fgk::DevState) <= kNoAllocStateBytes, "DevState fits its slot");

static __device__ __align__(256) unsigned char g_fgNoAllocScratch[kNoAllocStateBytes + kNoAllocMaxFlowPixels * 8];

constexpr int kMaxDevices = 64;
// device address of g_fgNoAllocScratch per device (null: not set up yet); written once, under g_setupLock
std::atomic<unsigned char*> g_scratchOfDevice[kMaxDevices];
std::mutex g_setupLock;

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// cv2.remap INTER_LINEAR / BORDER_REPLICATE of the 2-channel float field at (x, y), rounded exactly as OpenCV does:
// coordinates to 1/32 px (half even), ((p00 w00 + p01 w01) + p10 w10) + p11 w11 per channel in float32
__device__ float2 remapField(const float2* __restrict__ F, int w, int h, float x, float y) {
    const int X = __float2int_rn(__fmul_rn(x, 32.0f)), Y = __float2int_rn(__fmul_rn(y, 32.0f));
    const int ix = X >> 5, iy = Y >> 5;
    const float fx = (float)(X & 31) * (1.0f / 32.0f), fy = (float)(Y & 31) * (1.0f / 32.0f);
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    const float w00 = __fmul_rn(gy, gx), w01 = __fmul_rn(gy, fx), w10 = __fmul_rn(fy, gx), w11 = __fmul_rn(fy, fx);
    const int x0 = clampi(ix, 0, w - 1), x1 = clampi(ix + 1, 0, w - 1);
    const size_t r0 = (size_t)clampi(iy, 0, h - 1) * w, r1 = (size_t)clampi(iy + 1, 0, h - 1) * w;
    const float2 p00 = F[r0 + x0], p01 = F[r0 + x1], p10 = F[r1 + x0], p11 = F[r1 + x1];
    float2 r;
    r.x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.x, w00), __fmul_rn(p01.x, w01)), __fmul_rn(p10.x, w10)), __fmul_rn(p11.x, w11));
    r.y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p00.y, w00), __fmul_rn(p01.y, w01)), __fmul_rn(p10.y, w10)), __fmul_rn(p11.y, w11));
    return r;
}

// The field at time t into the scratch (interp.field_at: g <- pf(q - s g), twice, from g = pf(q); s = 0: the field
// itself), and the call's flags: the scene-cut decision, both untrusted counters cleared.
__global__ void __launch_bounds__(256) k_noalloc_prepare(const float2* __restrict__ pf, int fw, int fh, float s, int lookup,
                                                         int cut, unsigned char* scratch) {
    fgk::DevState* st = reinterpret_cast<fgk::DevState*>(scratch);
    float2* g = reinterpret_cast<float2*>(scratch + kNoAllocStateBytes);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->cut = cut ? 1u : 0u;
        st->untrusted[0] = 0;
        st->untrusted[1] = 0;
    }
    const int n = fw * fh;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const int qx = i % fw, qy = i / fw;
        float2 v = pf[i];
        if (lookup) {
            const float fx = (float)qx, fy = (float)qy;
            for (int it = 0; it < 2; it++)
                v = remapField(pf, fw, fh, __fsub_rn(fx, __fmul_rn(s, v.x)), __fsub_rn(fy, __fmul_rn(s, v.y)));
        }
        g[i] = v;
    }
}

}  // namespace

extern "C" int fg_record_synth_noalloc(void* stream, uint32_t view_format, uint32_t width, uint32_t height,
                                       const fg_frame* prev, const fg_frame* curr, const fg_frame* out, const float* field,
                                       int cut, float t, const fg_settings* settings, const char** error) {
    const char* dummy;
    const char** err = error ? error : &dummy;
    *err = nullptr;
    framegen::Settings set;
    if (settings) {
        const fg_settings& c = *settings;   // the V1 fields only (a caller's struct may end after pyramidMinSide)
        set.trustLow = c.trustLow; set.trustHigh = c.trustHigh; set.globalFallback = c.globalFallback;
        set.sceneCutSad = c.sceneCutSad; set.hudBonus = c.hudBonus; set.smoothBonus = c.smoothBonus;
        set.searchPenalty = c.searchPenalty; set.searchRadius = c.searchRadius; set.searchRadiusTop = c.searchRadiusTop;
        set.subpixel = c.subpixel != 0; set.uiProtection = (framegen::UiProtection)c.uiProtection;
        set.blurSamples = c.blurSamples; set.blurWeights = (framegen::BlurWeights)c.blurWeights;
        set.motionVersion = (framegen::MotionVersion)c.motionVersion; set.flowScale = c.flowScale;
        set.pyramidMinSide = c.pyramidMinSide;
    }
    if (const char* e = framegen::Interpolator::settingsError(set, framegen::Format::Rgba8)) { *err = e; return 0; }
    if (view_format != framegen::kVkFormatR8G8B8A8Unorm && view_format != framegen::kVkFormatB8G8R8A8Unorm) {
        *err = "fg_record_synth_noalloc takes the 8-bit RGBA / BGRA view formats only";
        return 0;
    }
    if (width < framegen::Interpolator::kMinSize || height < framegen::Interpolator::kMinSize) {
        *err = "the frame size is below Interpolator::kMinSize (16 pixels) in width or height";
        return 0;
    }
    if (!(t > 0.0f && t < 1.0f)) { *err = "t is outside (0, 1)"; return 0; }
    const int fs = (int)set.flowScale;
    const int fw = (int)std::nearbyint(width * (1.0 / fs)), fh = (int)std::nearbyint(height * (1.0 / fs));
    if ((size_t)fw * (size_t)fh > kNoAllocMaxFlowPixels) {
        *err = "the frame's per-pixel field exceeds the no-allocation scratch (at most 3,145,728 flow pixels, "
               "e.g. 3840x2160 at flowScale 2); use the Interpolator path";
        return 0;
    }
    auto ok = [&](const fg_frame* f) {
        return f && f->data && f->pitch >= (uint64_t)width * 4 && f->pitch % 4 == 0 && ((uintptr_t)f->data & 3) == 0 &&
               f->pitch <= fgk::kMaxPlaneSpan && (uint64_t)(height - 1) * f->pitch + (uint64_t)width * 4 <= fgk::kMaxPlaneSpan;
    };
    if (!ok(prev) || !ok(curr) || !ok(out) || prev->pitch != curr->pitch) {
        *err = "a frame is missing, misaligned, narrower than the width or spans more than 2^34 bytes";
        return 0;
    }
    if (!field) {
        *err = "the per-pixel field is null";
        return 0;
    }
    if (((uintptr_t)field & 7) != 0) {   // read as (x, y) pairs of floats
        *err = "the per-pixel field is not 8-byte aligned";
        return 0;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        *err = "no usable CUDA device";
        return 0;
    }
    unsigned char* scratch = g_scratchOfDevice[dev].load(std::memory_order_acquire);
    if (!scratch) {   // set-up, once per device (with that device current)
        std::lock_guard<std::mutex> lock(g_setupLock);
        scratch = g_scratchOfDevice[dev].load(std::memory_order_acquire);
        if (!scratch) {
            void* ptr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&ptr, g_fgNoAllocScratch);
            if (e != cudaSuccess || !ptr) {
                cudaGetLastError();
                *err = "cudaGetSymbolAddress of the no-allocation scratch failed (the first call on a device places "
                       "its 24 MiB array; is the device out of memory?)";
                return 0;
            }
            if (fgk::prepareKernels() != cudaSuccess) {
                cudaGetLastError();
                *err = "the kernels' shared-memory limits could not be set";
                return 0;
            }
            fgk::smCount();   // cached per device here, so later calls make no attribute query
            scratch = static_cast<unsigned char*>(ptr);
            g_scratchOfDevice[dev].store(scratch, std::memory_order_release);
        }
    }
    fgk::DevState* st = reinterpret_cast<fgk::DevState*>(scratch);
    float2* g = reinterpret_cast<float2*>(scratch + kNoAllocStateBytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double td = t;
    const float sv = (float)(2.0 * td - 1.0);
    const int lookup = sv != 0.0f;
    const int n = fw * fh;
    k_noalloc_prepare<<<(unsigned)std::min(fgk::smCount() * 8, (n + 255) / 256), 256, 0, s>>>(
        reinterpret_cast<const float2*>(field), fw, fh, sv, lookup, cut, scratch);
    cudaError_t e = cudaGetLastError();
    const bool rgba = view_format == framegen::kVkFormatR8G8B8A8Unorm;
    fgk::SynthParams sp{};
    sp.a = (const uint8_t*)prev->data; sp.c = (const uint8_t*)curr->data; sp.pitch = prev->pitch;
    sp.out = (uint8_t*)out->data; sp.outPitch = out->pitch;
    sp.W = (int)width; sp.H = (int)height; sp.fs = fs; sp.fw = fw; sp.fh = fh;
    sp.ri = rgba ? 0 : 2; sp.gi = 1; sp.bi = rgba ? 2 : 0;
    sp.pf = g;
    sp.lookup = 0;   // the field at t is already in the scratch
    sp.mid = t == 0.5f;
    sp.s = sv;
    sp.nearC = t > 0.5f;
    sp.ka = (float)(2.0 * td);
    sp.kc = (float)(2.0 * (1.0 - td));
    sp.wA = (float)(1.0 - td);
    sp.wC = t;
    sp.trust0 = set.trustLow;
    sp.trustSpan = (float)((double)set.trustHigh - (double)set.trustLow);
    fgk::trustShortcuts(set.trustLow, set.trustHigh, sp.sZero, sp.sOne);
    sp.st = st;
    sp.untrusted = &st->untrusted[0];
    sp.emap = nullptr;
    if (e == cudaSuccess) e = fgk::launchSynth(sp, s);
    fgk::FallbackParams fp{};
    fp.a = sp.a; fp.c = sp.c; fp.pitch = sp.pitch; fp.out = sp.out; fp.outPitch = sp.outPitch;
    fp.W = sp.W; fp.H = sp.H; fp.nearC = sp.nearC;
    fp.frac = (double)set.globalFallback;
    fp.untrusted = &st->untrusted[0];
    fp.untrustedNext = &st->untrusted[1];
    if (e == cudaSuccess) e = fgk::launchFallback(fp, s);
    if (e != cudaSuccess) {
        *err = cudaGetErrorString(e);
        return 0;
    }
    return 1;
}
