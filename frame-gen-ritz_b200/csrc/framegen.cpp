// Host side of the B200 framegen library: framegen::Interpolator (include/framegen.h) and the C ABI
// (include/framegen_c.h). It owns the device buffers of one frame size, turns Settings into kernel parameters and
// records the V1 passes as kernel launches on the caller's stream (fg_kernels.cu). Nothing here allocates, copies
// to the host or synchronises while recording.
//
// The control flow mirrors gpu/framegen.cpp: sizeLayout :658-685, validate :1679-1700, settingsError :1702-1711,
// setSettings / reconfigure :1723-1760, recordEstimate :2866-2940 + :3090-3154, recordSynth :3467-3532, record :3636.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "fg_blur.h"
#include "fg_params.h"
#include "fg_seednet.h"
#include "framegen.h"
#include "framegen_c.h"

namespace framegen {

namespace {

int rintHalfEven(double v) { return (int)std::nearbyint(v); }   // == cv2 saturate_cast<int>(double)

struct Level {
    int w = 0, h = 0, bw = 0, bh = 0;
    size_t lumaA = 0, lumaC = 0;   // float offsets into the luma buffer
    size_t fS = 0, fM = 0;         // float2 offsets into the field buffer: search output, median3 output
};

// gpu/framegen.cpp:658-685 (interp.flow / interp.pyramid sizes). The luma and field buffers are laid out level by
// level, finest first: luma a | c; field search | median3; then the two sub-pixel steps.
struct SizeLayout {
    int fw = 0, fh = 0;
    std::vector<Level> lv;
    size_t lumaFloats = 0, fieldF2 = 0, sub0 = 0, sub1 = 0;
};

SizeLayout sizeLayout(uint32_t W, uint32_t H, uint32_t flowScale, uint32_t minSide) {
    SizeLayout L;
    L.fw = rintHalfEven(W * (1.0 / flowScale));
    L.fh = rintHalfEven(H * (1.0 / flowScale));
    int w = L.fw, h = L.fh;
    size_t lo = 0, fo = 0;
    for (;;) {
        Level l;
        l.w = w; l.h = h;
        l.bw = (w + 7) / 8; l.bh = (h + 7) / 8;   // pad_to_block
        l.lumaA = lo; l.lumaC = lo + (size_t)w * h;
        lo += 2 * (size_t)w * h;
        l.fS = fo; l.fM = fo + (size_t)l.bw * l.bh;
        fo += 2 * (size_t)l.bw * l.bh;
        L.lv.push_back(l);
        if ((uint32_t)(std::min(w, h) / 2) < minSide || L.lv.size() >= (size_t)fgk::kMaxLevels) break;
        w = rintHalfEven(w * 0.5);
        h = rintHalfEven(h * 0.5);
    }
    L.sub0 = fo;
    fo += (size_t)L.lv[0].bw * L.lv[0].bh;
    L.sub1 = fo;
    fo += (size_t)L.lv[0].bw * L.lv[0].bh;
    L.lumaFloats = lo;
    L.fieldF2 = fo;
    return L;
}

// gpu/framegen.cpp:430-433: the longest integer half-vector the search can reach at level j of an n-level pyramid
int64_t reachBound(int n, int j, int R, int Rt) {
    const int64_t a = (int64_t)1 << (n - 1 - j);
    return Rt * a + (int64_t)R * (a - 1);
}

// numpy's pairwise summation tree over N elements (leaves of <= 128 elements, splits at n/2 rounded down to a
// multiple of 8), with the inner nodes ordered by height so each height is one parallel step.
struct CutPlanHost {
    std::vector<int2> leaves, inner;
    std::vector<int> depthStart;
    int root = 0, nSteps = 0;
};
CutPlanHost buildCutPlan(int N) {
    struct TNode { bool leaf; int idx, height; };
    std::vector<int2> leaves;
    std::vector<std::array<TNode, 2>> kids;
    std::vector<int> heights;
    std::vector<std::array<int, 3>> stack;   // explicit recursion: (start, n, state)
    // recursive lambda (depth <= log2(N / 64) + 1)
    struct B {
        std::vector<int2>& leaves;
        std::vector<std::array<TNode, 2>>& kids;
        std::vector<int>& heights;
        TNode go(int start, int n) {
            if (n <= 128) {
                leaves.push_back(make_int2(start, n));
                return {true, (int)leaves.size() - 1, 0};
            }
            int n2 = n / 2;
            n2 -= n2 % 8;
            TNode l = go(start, n2), r = go(start + n2, n - n2);
            kids.push_back({l, r});
            heights.push_back(1 + std::max(l.height, r.height));
            return {false, (int)kids.size() - 1, heights.back()};
        }
    } b{leaves, kids, heights};
    TNode root = b.go(0, N);
    CutPlanHost P;
    P.leaves = leaves;
    const int nL = (int)leaves.size(), nI = (int)kids.size();
    std::vector<int> order(nI);
    for (int i = 0; i < nI; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return heights[x] < heights[y]; });
    std::vector<int> slot(nI);
    for (int r = 0; r < nI; r++) slot[order[r]] = nL + r;
    auto slotOf = [&](const TNode& t) { return t.leaf ? t.idx : slot[t.idx]; };
    int maxH = 0;
    for (int r = 0; r < nI; r++) {
        const auto& k = kids[order[r]];
        P.inner.push_back(make_int2(slotOf(k[0]), slotOf(k[1])));
        maxH = std::max(maxH, heights[order[r]]);
    }
    P.nSteps = maxH;
    P.depthStart.assign(maxH + 1, nI);
    for (int h = maxH; h >= 1; h--)
        for (int r = nI - 1; r >= 0; r--)
            if (heights[order[r]] == h) P.depthStart[h - 1] = r;
    P.depthStart[maxH] = nI;
    for (int h = maxH - 1; h >= 0; h--) P.depthStart[h] = std::min(P.depthStart[h], P.depthStart[h + 1]);
    P.root = slotOf(root);
    (void)stack;
    return P;
}

size_t alignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }

// the most device memory recordSynthBlur's stored sub-frames may take (16 samples of a 3840x2160 frame are 531 MB);
// past it the blur runs as the fused kernel, which stores none
constexpr size_t kBlurSubMaxBytes = (size_t)1 << 30;

const char* kErrSettings = "invalid settings: a field is out of range or not finite (see Interpolator::validate)";
const char* kErrVersion = "this library runs MotionVersion::V1 only (V2, Learned and V3 are not built into it)";
const char* kErrUi = "static-UI protection: only CrosshairV2 is built into this library (Crosshair and WholeScreen are not)";
const char* kErrUiFormat = "static-UI protection (CrosshairV2): unknown frame format";
const char* kErrNoFormat = "unsupported viewFormat (see framegen::Format)";
const char* kErrYuvMatrix = "yuvMatrix must be Bt601, Bt709 or Bt2020";
const char* kErrNits = "linearWhiteNits must be in (0, 10000]";
const char* kErrMinSize = "the frame size is below Interpolator::kMinSize (16 pixels) in width or height";
const char* kErrMaxSize = "the frame size exceeds 2^30 pixels (32-bit indexing of the library's buffers)";
const char* kErrDevice = "CUDA device not available";
const char* kErrAlloc = "CUDA device memory allocation failed";

// the per-format constants of the kernels (gpu/framegen.cpp:1508-1539 for YUV; fg_formats.cu for their use)
fgk::FmtConst makeFmtConst(Format fmt, uint32_t viewFormat, const InitInfo& ii) {
    fgk::FmtConst c{};
    c.format = (int)fmt;
    c.rHigh = viewFormat == kVkFormatA2R10G10B10UnormPack32;
    c.linear = ii.transfer == Transfer::Linear;
    c.kWhite = ii.linearWhiteNits / 10000.0f;
    c.k10 = (float)(255.0 / 1023.0);
    c.k10i = (float)(1023.0 / 255.0);
    double kr = 0.2126, kb = 0.0722;   // BT.709
    if (ii.yuvMatrix == YuvMatrix::Bt601) { kr = 0.299; kb = 0.114; }
    if (ii.yuvMatrix == YuvMatrix::Bt2020) { kr = 0.2627; kb = 0.0593; }
    const double kg = 1.0 - kr - kb;
    const double sY = ii.yuvFullRange ? 1.0 : 255.0 / 219.0, sC = ii.yuvFullRange ? 1.0 : 255.0 / 224.0;
    c.black = ii.yuvFullRange ? 0.0f : 16.0f;
    c.ys = (float)sY;
    c.rcr = (float)(sC * 2.0 * (1.0 - kr));
    c.bcb = (float)(sC * 2.0 * (1.0 - kb));
    c.gcb = (float)(-sC * 2.0 * (1.0 - kb) * kb / kg);
    c.gcr = (float)(-sC * 2.0 * (1.0 - kr) * kr / kg);
    return c;
}

// bytes per pixel of plane 0 and per texel of the CbCr plane (0: none)
int planeBytes(Format f) { return f == Format::RgbaF16 ? 8 : (f == Format::Nv12 ? 1 : (f == Format::P010 ? 2 : 4)); }
int chromaBytes(Format f) { return f == Format::Nv12 ? 2 : (f == Format::P010 ? 4 : 0); }

struct DeviceGuard {   // makes `dev` current for the scope, restores the caller's device after
    int old = -1;
    bool changed = false;
    explicit DeviceGuard(int dev) {
        if (dev >= 0 && cudaGetDevice(&old) == cudaSuccess && old != dev) changed = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(old);
    }
};

}  // namespace

bool formatOf(uint32_t vf, Format* out) {
    Format f;
    switch (vf) {
        case kVkFormatR8G8B8A8Unorm:
        case kVkFormatB8G8R8A8Unorm: f = Format::Rgba8; break;
        case kVkFormatA2R10G10B10UnormPack32:
        case kVkFormatA2B10G10R10UnormPack32: f = Format::Rgb10; break;
        case kVkFormatR16G16B16A16Sfloat: f = Format::RgbaF16; break;
        case kVkFormatR8Unorm: f = Format::Nv12; break;
        case kVkFormatR16Unorm: f = Format::P010; break;
        default: return false;
    }
    if (out) *out = f;
    return true;
}

struct Interpolator::Impl {
    int device = 0;
    Format fmt = Format::Rgba8;
    uint32_t viewFormat = kVkFormatB8G8R8A8Unorm;
    int ri = 2, gi = 1, bi = 0;
    fgk::FmtConst fc{};
    InitInfo info{};
    Settings set{};
    uint32_t W = 0, H = 0;
    SizeLayout L;
    // device memory (one allocation)
    char* arena = nullptr;
    size_t arenaBytes = 0;
    float* luma = nullptr;
    float* pqTab = nullptr;   // linear RgbaF16: the PQ level of every half value (the luma pass looks them up)
    float2* field = nullptr;
    float* sads = nullptr;
    float2* pf = nullptr;
    unsigned int* hist = nullptr;
    int histB = 0;
    fgk::DevState* st = nullptr;
    unsigned int* blurCnt = nullptr;   // recordSynthBlur: per sample, its untrusted pixels (kBlurMax)
    // recordSynthBlur's sub-frames (8-bit RGBA): blurSubCap frames of blurSubPitch x H bytes, or none
    uint8_t* blurSub = nullptr;
    size_t blurSubPitch = 0;
    uint32_t blurSubCap = 0;
    uint8_t* emap = nullptr;
    fgk::CutPlan plan{};
    // trust-ramp shortcuts of the current settings
    int sZero = 0, sOne = 0;
    // record state
    bool haveEst = false;
    const void* estPrev = nullptr;
    const void* estCurr = nullptr;
    uint32_t estSets = 0, synthSets = 0;
    unsigned int parity = 0, lastParity = 0;
    bool capture = false;
    const char* lastErr = nullptr;
    // the seed net (setSeedNet): its parameters, the requested level, the level of this size, its buffers
    std::vector<float> snParams;
    int snLevelReq = -1, snK = -1;
    fg_seednet* snet = nullptr;
    float* snOut = nullptr;    // its output, bw x bh x kSeedNetOut floats
    // static-UI protection, CrosshairV2 (recordObserve / recordTrack): the box and work rectangle of this size and
    // settings, the per-pixel state of the work rectangle, and the kept frames' masks (LRU by observe order)
    struct UiEntry {
        const void* key = nullptr;    // the frame (device pointer); null = free
        uint32_t* mask = nullptr;     // header + bytes (fg_params.h UiV2Params)
        uint64_t stamp = 0;           // observe order
    };
    std::vector<UiEntry> uiE;
    uint32_t* uiState = nullptr;
    int32_t uiBox[4] = {}, uiWork[4] = {};
    int uiStride = 0;
    bool uiReset = true, uiExplicit = false;
    const void* uiLast = nullptr;
    uint64_t uiClock = 0;
    bool estUi = false;
    const uint32_t* fillMask[2] = {nullptr, nullptr};   // the estimate fill's masks of the pair being estimated
    int estEnt[2] = {-1, -1};
    uint64_t estStamp[2] = {0, 0};
    // profiling
    bool profiling = false;
    std::vector<cudaEvent_t> events;
    std::vector<const char*> evNames;
    size_t evCount = 0;
    uint32_t profileNo = 0, profileRead = 0, costSeq = 0;   // readCosts: profiles started, the last one read

    ~Impl() { freeAll(); }

    void freeSeedNet() {
        if (snet) fg_seednet_destroy(snet);
        if (snOut) cudaFree(snOut);
        snet = nullptr;
        snOut = nullptr;
        snK = -1;
    }

    // the seed net's buffers for the current size (after allocSize; outside any capture)
    const char* setupSeedNet() {
        DeviceGuard g(device);
        freeSeedNet();
        if (snLevelReq < 0 || !W) return nullptr;
        snK = std::min(snLevelReq, (int)L.lv.size() - 1);
        const Level& lk = L.lv[snK];
        snet = fg_seednet_create(device, 1, lk.h, lk.w);
        if (!snet || !fg_seednet_set_params(snet, snParams.data()) ||
            cudaMalloc((void**)&snOut, (size_t)lk.bw * lk.bh * fgk::kSeedNetOut * 4) != cudaSuccess) {
            cudaGetLastError();
            freeSeedNet();
            return kErrAlloc;
        }
        return nullptr;
    }

    bool uiOn() const { return set.uiProtection == UiProtection::CrosshairV2; }

    void uiFree() {
        DeviceGuard g(device);
        for (UiEntry& e : uiE)
            if (e.mask) cudaFree(e.mask);
        uiE.clear();
        if (uiState) cudaFree(uiState);
        uiState = nullptr;
        uiWork[2] = uiWork[3] = 0;
        uiReset = true;
        uiLast = nullptr;
        estUi = false;
    }

    // the protection's buffers for the current size and settings (outside any capture; only ever allocates, except
    // when the work rectangle changes): the state of the work rectangle, uiHistory masks. A new rectangle (size or box
    // change) or `restart` (protection switched on) starts the state afresh and forgets every kept frame.
    const char* uiSetup(bool restart) {
        if (!uiOn() || !W) return nullptr;
        int32_t box[4], work[4];
        Interpolator::boxRect(set, W, H, box);
        Interpolator::workRect(set, W, H, work);
        const bool same = uiState && std::equal(work, work + 4, uiWork) && std::equal(box, box + 4, uiBox);
        DeviceGuard g(device);
        if (!same) {
            uiFree();
            std::copy(box, box + 4, uiBox);
            std::copy(work, work + 4, uiWork);
            uiStride = (work[2] + 3) / 4;
            if (cudaMalloc((void**)&uiState, (size_t)work[2] * work[3] * 16) != cudaSuccess) {
                cudaGetLastError();
                uiState = nullptr;
                uiWork[2] = uiWork[3] = 0;
                return kErrAlloc;
            }
            restart = true;
        }
        if (restart) {
            uiReset = true;
            uiLast = nullptr;
            for (UiEntry& e : uiE) e.key = nullptr;
            estUi = false;
        }
        const size_t words = (size_t)fgk::kUiMaskHeader + (size_t)uiStride * uiWork[3];
        while (uiE.size() < set.uiHistory) {
            UiEntry e;
            if (cudaMalloc((void**)&e.mask, words * 4) != cudaSuccess) {
                cudaGetLastError();
                return kErrAlloc;
            }
            uiE.push_back(e);
        }
        uiEvict(set.uiHistory);
        return nullptr;
    }

    int uiCount() const {
        int n = 0;
        for (const UiEntry& e : uiE) n += e.key != nullptr;
        return n;
    }
    // forget the least recently observed frames until at most `keep` are kept
    void uiEvict(uint32_t keep) {
        while ((uint32_t)uiCount() > keep) {
            UiEntry* old = nullptr;
            for (UiEntry& e : uiE)
                if (e.key && (!old || e.stamp < old->stamp)) old = &e;
            old->key = nullptr;
        }
    }
    int uiFind(const void* key) const {
        for (size_t i = 0; i < uiE.size(); i++)
            if (uiE[i].key == key) return (int)i;
        return -1;
    }

    // one observed (track = false) or tracked frame: the state update, then (observe) the frame's mask in its entry
    bool uiObserve(cudaStream_t s, const Frame& f, bool track) {
        fgk::UiV2Params p{};
        p.frame = (const uint8_t*)f.data; p.pitch = f.pitch;
        p.W = (int)W; p.H = (int)H; p.ri = ri; p.gi = gi; p.bi = bi;
        p.f = fc;
        p.pq = pqTab;
        p.frameC = (const uint8_t*)f.chroma; p.cpitch = f.chromaPitch;
        p.bx = uiBox[0]; p.by = uiBox[1]; p.bw = uiBox[2]; p.bh = uiBox[3];
        p.wx = uiWork[0]; p.wy = uiWork[1]; p.ww = uiWork[2]; p.wh = uiWork[3];
        p.st = uiState;
        p.reset = uiReset;
        p.thr = set.uiStillThreshold; p.cthr = set.uiContrastThreshold;
        p.still = (int)set.uiStillFrames; p.leave = (int)set.uiLeaveFrames; p.reentry = (int)set.uiReentryFrames;
        p.maskStride = uiStride;
        int slot = uiFind(f.data);
        if (track) {
            if (slot >= 0) uiE[slot].key = nullptr;   // the frame holds new pixels: its kept mask is stale
        } else if (slot < 0) {
            uiEvict(set.uiHistory - 1);
            slot = uiFind(nullptr);
        }
        p.mask = track ? nullptr : uiE[slot].mask;
        if (!check(fgk::launchUiV2Update(p, s))) return false;
        if (!track) {
            if (!check(fgk::launchUiV2Mask(p, s))) return false;
            uiE[slot].key = f.data;
            uiE[slot].stamp = ++uiClock;
            uiLast = f.data;
        }
        uiReset = false;
        stamp(s, track ? "ui track" : "ui observe");
        return true;
    }

    // the kept masks the latest estimate's pair uses, if they are still the same entries (else a synthesis refuses)
    bool uiPairMasks(const uint32_t*& ma, const uint32_t*& mc) const {
        ma = mc = nullptr;
        if (!uiOn() || !estUi) return true;
        for (int k = 0; k < 2; k++) {
            if (estEnt[k] < 0 || estEnt[k] >= (int)uiE.size()) return false;
            const UiEntry& e = uiE[estEnt[k]];
            if (e.key != (k ? estCurr : estPrev) || e.stamp != estStamp[k]) return false;
        }
        ma = uiE[estEnt[0]].mask;
        mc = uiE[estEnt[1]].mask;
        return true;
    }

    bool uiPatch(cudaStream_t s, const Frame& curr, const Frame& out, const uint32_t* mc) {
        fgk::UiPatchParams pp{(const uint8_t*)curr.data, curr.pitch, (uint8_t*)out.data, out.pitch, mc, fc.format,
                              (const uint8_t*)curr.chroma, curr.chromaPitch, (uint8_t*)out.chroma, out.chromaPitch};
        if (!check(fgk::launchUiPatch(pp, uiWork[0], uiWork[1], uiWork[2], uiWork[3], s))) return false;
        stamp(s, "ui patch");
        return true;
    }

    void blurFree() {
        DeviceGuard g(device);
        if (blurSub) cudaFree(blurSub);
        blurSub = nullptr;
        blurSubPitch = 0;
        blurSubCap = 0;
    }

    // the sub-frames of the current size and settings (after allocSize and on a settings change; outside any capture).
    // 8-bit RGBA with blur on keeps one frame per sample while they fit kBlurSubMaxBytes; otherwise, or when the
    // allocation fails, recordSynthBlur runs the fused kernel, which stores none (not an error)
    void blurSetup() {
        const uint32_t need = fmt == Format::Rgba8 && W && set.blurSamples >= 2
                                  ? std::min<uint32_t>(set.blurSamples, Interpolator::kBlurMaxSamples) : 0u;
        const size_t pitch = alignUp((size_t)W * 4, 256);
        if (!need || (size_t)need * pitch * H > kBlurSubMaxBytes) { blurFree(); return; }
        if (blurSubCap >= need && blurSubPitch == pitch) return;
        blurFree();
        DeviceGuard g(device);
        if (cudaMalloc((void**)&blurSub, (size_t)need * pitch * H) != cudaSuccess) {
            cudaGetLastError();
            blurSub = nullptr;
            return;
        }
        blurSubPitch = pitch;
        blurSubCap = need;
    }

    void freeAll() {
        DeviceGuard g(device);
        uiFree();
        blurFree();
        freeSeedNet();
        if (arena) cudaFree(arena);
        arena = nullptr;
        pqTab = nullptr;
        arenaBytes = 0;
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        events.clear();
        W = H = 0;
        haveEst = false;
    }

    void updateTrust() { fgk::trustShortcuts(set.trustLow, set.trustHigh, sZero, sOne); }

    // buffers of one size (createSizeDependent, gpu/framegen.cpp:994-1014)
    const char* allocSize(uint32_t w, uint32_t h) {
        freeAll();
        DeviceGuard g(device);
        L = sizeLayout(w, h, set.flowScale, set.pyramidMinSide);
        const int n = (int)L.lv.size();
        // the median histograms hold any parent vector the largest radii (12, 12) can reach, so a runtime change
        // of the radii (setSettings) never needs new buffers
        int64_t B = n > 1 ? reachBound(n, 1, 12, 12) : 0;
        if (snLevelReq >= 1 && n > 1) {   // seed-net candidates (clamped to +-256) can start anywhere at its level
            const int k = std::min(snLevelReq, n - 1);
            const int64_t a = (int64_t)1 << (k - 1);
            B = std::max<int64_t>(B, (256 + 12) * a + 12 * (a - 1));
        }
        histB = (int)B;
        const int nb0 = L.lv[0].bw * L.lv[0].bh;
        CutPlanHost P = buildCutPlan(nb0);
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t o = off; off = alignUp(off + bytes, 256); return o; };
        const size_t oLuma = take(L.lumaFloats * 4), oField = take(L.fieldF2 * 8), oSads = take((size_t)nb0 * 4);
        const size_t oPf = take((size_t)L.fw * L.fh * 8), oHist = take((size_t)2 * (2 * histB + 1) * 4);
        const size_t oSt = take(sizeof(fgk::DevState)), oEmap = take((size_t)((w + 3) & ~3u) * h);
        const size_t oBlur = take((size_t)fgk::kBlurMax * 4);
        const size_t oLeaves = take(P.leaves.size() * 8), oInner = take(std::max<size_t>(P.inner.size(), 1) * 8);
        const size_t oDepth = take(P.depthStart.size() * 4 + 4);
        const size_t oVals = take((P.leaves.size() + P.inner.size()) * 4);
        const size_t oLeafOf = take((size_t)nb0 * 4), oLeafCnt = take(P.leaves.size() * 4), oLeafS = take(P.leaves.size() * 4);
        const bool pqLuma = fmt == Format::RgbaF16 && fc.linear;
        const size_t oPq = take(pqLuma ? (size_t)65536 * 4 : 0);
        if (cudaMalloc(&arena, off) != cudaSuccess) { arena = nullptr; cudaGetLastError(); return kErrAlloc; }
        arenaBytes = off;
        cudaMemset(arena, 0, off);
        luma = (float*)(arena + oLuma);
        field = (float2*)(arena + oField);
        sads = (float*)(arena + oSads);
        pf = (float2*)(arena + oPf);
        hist = (unsigned int*)(arena + oHist);
        st = (fgk::DevState*)(arena + oSt);
        blurCnt = (unsigned int*)(arena + oBlur);
        emap = (uint8_t*)(arena + oEmap);
        pqTab = pqLuma ? (float*)(arena + oPq) : nullptr;
        if (pqTab) fgk::launchPqTable(pqTab, fc.kWhite, 0);
        cudaMemcpy(arena + oLeaves, P.leaves.data(), P.leaves.size() * 8, cudaMemcpyHostToDevice);
        if (!P.inner.empty()) cudaMemcpy(arena + oInner, P.inner.data(), P.inner.size() * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(arena + oDepth, P.depthStart.data(), P.depthStart.size() * 4, cudaMemcpyHostToDevice);
        {
            std::vector<int> leafOf((size_t)nb0);
            for (size_t i = 0; i < P.leaves.size(); i++)
                for (int k = 0; k < P.leaves[i].y; k++) leafOf[(size_t)P.leaves[i].x + k] = (int)i;
            cudaMemcpy(arena + oLeafOf, leafOf.data(), (size_t)nb0 * 4, cudaMemcpyHostToDevice);
        }
        if (cudaDeviceSynchronize() != cudaSuccess) { cudaGetLastError(); freeAll(); return kErrAlloc; }
        plan.leaves = (const int2*)(arena + oLeaves);
        plan.inner = (const int2*)(arena + oInner);
        plan.depthStart = (const int*)(arena + oDepth);
        plan.nLeaves = (int)P.leaves.size();
        plan.nInner = (int)P.inner.size();
        plan.nSteps = P.nSteps;
        plan.root = P.root;
        plan.gvals = (float*)(arena + oVals);
        plan.leafOf = (const int*)(arena + oLeafOf);
        plan.leafCnt = (unsigned int*)(arena + oLeafCnt);
        plan.leafS256 = (unsigned int*)(arena + oLeafS);
        W = w;
        H = h;
        haveEst = false;
        if (const char* e = setupSeedNet()) return e;
        blurSetup();
        return uiSetup(true);
    }

    // a frame the kernels can address: plane 0 (and the CbCr plane of YUV) aligned to its sample size, rows wide enough,
    // plane 0 within fgk::kMaxPlaneSpan bytes
    bool frameOk(const Frame& f) const {
        const size_t bpp = (size_t)planeBytes(fmt), cb = (size_t)chromaBytes(fmt);
        const size_t al = fmt == Format::Nv12 ? 1 : bpp;
        if (!f.data || f.pitch < (size_t)W * bpp || f.pitch % al || ((uintptr_t)f.data % al)) return false;
        if (f.pitch > fgk::kMaxPlaneSpan || (size_t)(H - 1) * f.pitch + (size_t)W * bpp > fgk::kMaxPlaneSpan) return false;
        if (!cb) return true;
        return f.chroma && f.chromaPitch >= (size_t)((W + 1) / 2) * cb && f.chromaPitch % cb == 0 &&
               (uintptr_t)f.chroma % cb == 0;
    }
    bool samePitch(const Frame& a, const Frame& b) const {
        return a.pitch == b.pitch && (!chromaBytes(fmt) || a.chromaPitch == b.chromaPitch);
    }

    // --- profiling (gpu/framegen.cpp Rec::stamp)
    void stamp(cudaStream_t s, const char* name) {
        if (!profiling) return;
        if (evCount >= 64) return;
        while (events.size() <= evCount) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
            events.push_back(e);
        }
        cudaEventRecord(events[evCount], s);
        if (evNames.size() <= evCount) evNames.resize(evCount + 1);
        evNames[evCount++] = name;
    }

    bool check(cudaError_t e) {
        if (e != cudaSuccess) { lastErr = cudaGetErrorString(e); return false; }
        return true;
    }

    // Every pass of one estimate, its parameters resolved (the luma, the pyramid levels beyond the luma kernel's tower,
    // per level from the coarsest searched down: search and median3, then the sub-pixel refinement or the scene-cut
    // mean, then the pixel field). fill: CrosshairV2's estimate fill rebuilds levels >= 1 from the filled level 0.
    struct EstPlan {
        fgk::LumaPyrParams luma{};
        std::vector<fgk::DownParams> down;
        int top = 0;                                 // the coarsest level searched
        std::vector<fgk::SearchParams> search;       // by level
        std::vector<fgk::Median3Params> med;         // by level
        fgk::SubpixParams sub{};
        fgk::CutMeanParams cut{};
        fgk::PixfieldParams pix{};
    };
    void planEstimate(const Frame& prev, const Frame& curr, bool fill, EstPlan& e) const {
        const int n = (int)L.lv.size();
        const float lam = set.searchPenalty;
        // 1-2. luma + pyramid
        fgk::LumaPyrParams& lp = e.luma;
        lp = fgk::LumaPyrParams{};
        lp.a = (const uint8_t*)prev.data; lp.c = (const uint8_t*)curr.data; lp.pitch = prev.pitch;
        lp.W = (int)W; lp.H = (int)H; lp.fs = (int)set.flowScale;
        lp.ri = ri; lp.gi = gi; lp.bi = bi;
        e.top = snK >= 0 ? snK : n - 1;
        lp.nlev = std::min(e.top + 1, fgk::kPyrInKernel);
        lp.f = fc;
        lp.pq = pqTab;
        lp.vec16 = fmt == Format::Rgba8 && set.flowScale == 2 && prev.pitch % 16 == 0 && ((uintptr_t)prev.data & 15) == 0 && ((uintptr_t)curr.data & 15) == 0 &&
                   W % 4 == 0 && H % 2 == 0;   // complete 2x2 cells in every full tile, 8-byte aligned level-0 rows
        for (int l = 0; l < lp.nlev; l++) {
            lp.lw[l] = L.lv[l].w; lp.lh[l] = L.lv[l].h;
            lp.la[l] = luma + L.lv[l].lumaA; lp.lc[l] = luma + L.lv[l].lumaC;
        }
        e.down.clear();
        for (int l = fill ? 1 : fgk::kPyrInKernel; l <= e.top; l++)
            e.down.push_back(fgk::DownParams{luma + L.lv[l - 1].lumaA, luma + L.lv[l - 1].lumaC, L.lv[l - 1].w, L.lv[l - 1].h,
                                             luma + L.lv[l].lumaA, luma + L.lv[l].lumaC, L.lv[l].w, L.lv[l].h, fmt != Format::Rgba8});
        // 3-5. per level, coarse -> fine
        e.search.assign(n, fgk::SearchParams{});
        e.med.assign(n, fgk::Median3Params{});
        for (int i = e.top; i >= 0; i--) {
            const Level& l = L.lv[i];
            fgk::SearchParams& sp = e.search[i];
            sp.la = luma + l.lumaA; sp.lc = luma + l.lumaC;
            sp.w = l.w; sp.h = l.h; sp.bw = l.bw; sp.bh = l.bh;
            sp.top = i == n - 1 && snK < 0;
            sp.cnn = i == snK ? snOut : nullptr;
            sp.R = (int)(sp.top ? set.searchRadiusTop : set.searchRadius);
            if (!sp.top && !sp.cnn) {
                const Level& pl = L.lv[i + 1];
                sp.parent = field + pl.fM; sp.pw = pl.bw; sp.ph = pl.bh;
                sp.med = st->med[i];
            }
            sp.lambda = lam;
            for (int k = 0; k <= 2 * sp.R; k++) sp.pen[k] = (float)((double)lam * 1.0 * (double)k);
            sp.out = field + l.fS;
            sp.sadOut = (i == 0 && !set.subpixel) ? sads : nullptr;
            fgk::Median3Params& mp = e.med[i];
            mp.in = field + l.fS; mp.out = field + l.fM; mp.bw = l.bw; mp.bh = l.bh;
            mp.doHist = i > 0;
            if (i > 0) {
                mp.fbw = L.lv[i - 1].bw; mp.fbh = L.lv[i - 1].bh; mp.B = histB;
                mp.hist = hist; mp.done = &st->medDone[i]; mp.medOut = st->med[i - 1];
            }
            mp.err = &st->err;
        }
        // 6. sub-pixel refinement + the scene-cut mean
        const Level& l0 = L.lv[0];
        const float2* vfin = field + l0.fM;
        if (set.subpixel) {
            fgk::SubpixParams& sp = e.sub;
            sp = fgk::SubpixParams{};
            sp.la = luma + l0.lumaA; sp.lc = luma + l0.lumaC;
            sp.w = l0.w; sp.h = l0.h; sp.bw = l0.bw; sp.bh = l0.bh;
            sp.in = field + l0.fM; sp.out = field + L.sub1; sp.out0 = field + L.sub0; sp.sads = sads;
            const float steps[2] = {0.5f, 0.25f};
            for (int p = 0; p < 2; p++)
                for (int k = 0; k < 3; k++) sp.pen[p][k] = (float)((double)lam * (double)steps[p] * (double)k);
            sp.plan = plan; sp.cutSad = set.sceneCutSad; sp.st = st;
            vfin = field + L.sub1;
        } else {
            e.cut = fgk::CutMeanParams{sads, l0.bw * l0.bh, plan, set.sceneCutSad, st};
        }
        // 8. per-pixel vector choice
        e.pix = fgk::PixfieldParams{luma + l0.lumaA, luma + l0.lumaC, l0.w, l0.h, vfin, l0.bw, l0.bh, set.smoothBonus,
                                    set.hudBonus, pf};
    }

    bool estimate(cudaStream_t s, const Frame& prev, const Frame& curr) {
        if (prev.pitch != curr.pitch) return false;
        if (profiling) { evCount = 0; profileNo++; stamp(s, "start"); }
        const bool fill = fillMask[0] && fillMask[1];
        EstPlan e;
        planEstimate(prev, curr, fill, e);
        const fgk::LumaPyrParams& lp = e.luma;
        if (!check(fmt == Format::Rgba8 ? fgk::launchLumaPyr(lp, s) : fgk::launchLumaFmt(lp, s))) return false;
        stamp(s, "luma");
        if (fill) {   // CrosshairV2's estimate fill of level 0; the pyramid is then rebuilt from the filled level 0
            fgk::UiFillParams fp{};
            fp.a = lp.a; fp.c = lp.c; fp.pitch = lp.pitch;
            fp.W = (int)W; fp.H = (int)H; fp.ri = ri; fp.gi = gi; fp.bi = bi; fp.fs = (int)set.flowScale;
            fp.fw = L.lv[0].w; fp.fh = L.lv[0].h;
            fp.ma = fillMask[0]; fp.mc = fillMask[1];
            fp.la = luma + L.lv[0].lumaA; fp.lc = luma + L.lv[0].lumaC;
            fp.cx0 = uiWork[0] / fp.fs; fp.cy0 = uiWork[1] / fp.fs;
            fp.ncx = (uiWork[0] + uiWork[2] - 1) / fp.fs - fp.cx0 + 1;
            fp.ncy = (uiWork[1] + uiWork[3] - 1) / fp.fs - fp.cy0 + 1;
            fp.f = fc;
            fp.pq = pqTab;
            if (!check(fmt == Format::Rgba8 ? fgk::launchUiFill(fp, s) : fgk::launchUiFillFmt(fp, s))) return false;
            stamp(s, "ui fill");
        }
        for (const fgk::DownParams& dp : e.down)
            if (!check(fgk::launchDown(dp, s))) return false;
        stamp(s, "pyramid");
        if (snK >= 0) {   // the seed net on level snK
            const Level& lk = L.lv[snK];
            if (!fgk::seedNetForwardLuma(snet, s, luma + lk.lumaA, luma + lk.lumaC, lk.h, lk.w, snOut, &st->err, &lastErr))
                return false;
            stamp(s, "seed net");
        }
        static const char* names[] = {"level 0 (finest)", "level 1", "level 2", "level 3", "level 4", "level 5",
                                      "level 6", "level 7"};
        for (int i = e.top; i >= 0; i--) {
            if (!check(fgk::launchSearch(e.search[i], s))) return false;
            if (!check(fgk::launchMedian3(e.med[i], s))) return false;
            stamp(s, names[std::min(i, 7)]);
        }
        if (!check(set.subpixel ? fgk::launchSubpix(e.sub, s) : fgk::launchCutMean(e.cut, s))) return false;
        stamp(s, "subpixel");
        if (!check(fgk::launchPixfield(e.pix, s))) return false;
        stamp(s, "pixel field");
        return true;
    }

    // the parameters of one synthesis (interp.synth's t constants, this size's buffers); untrusted: its counter
    fgk::SynthParams synthParams(const Frame& prev, const Frame& curr, const Frame& out, float t, unsigned int* untrusted) const {
        const double td = t;
        fgk::SynthParams sp{};
        sp.a = (const uint8_t*)prev.data; sp.c = (const uint8_t*)curr.data; sp.pitch = prev.pitch;
        sp.out = (uint8_t*)out.data; sp.outPitch = out.pitch;
        sp.W = (int)W; sp.H = (int)H; sp.fs = (int)set.flowScale; sp.fw = L.fw; sp.fh = L.fh;
        sp.ri = ri; sp.gi = gi; sp.bi = bi;
        sp.pf = pf;
        sp.mid = t == 0.5f;
        sp.s = (float)(2.0 * td - 1.0);
        sp.lookup = sp.s != 0.0f;
        sp.nearC = t > 0.5f;
        sp.ka = (float)(2.0 * td);
        sp.kc = (float)(2.0 * (1.0 - td));
        sp.wA = (float)(1.0 - td);
        sp.wC = t;
        sp.trust0 = set.trustLow;
        sp.trustSpan = (float)((double)set.trustHigh - (double)set.trustLow);
        sp.sZero = sZero; sp.sOne = sOne;
        sp.st = st;
        sp.untrusted = untrusted;
        sp.emap = capture ? emap : nullptr;
        sp.f = fc;
        sp.ac = (const uint8_t*)prev.chroma; sp.cc = (const uint8_t*)curr.chroma; sp.cpitch = prev.chromaPitch;
        sp.outc = (uint8_t*)out.chroma; sp.outCPitch = out.chromaPitch;
        return sp;
    }

    // the parameters of its whole-frame fallback (interp.py:238-239); next: the counter to clear (may be null)
    fgk::FallbackParams fallbackParams(const fgk::SynthParams& sp, unsigned int* next) const {
        fgk::FallbackParams fp{};
        fp.a = sp.a; fp.c = sp.c; fp.pitch = sp.pitch; fp.out = sp.out; fp.outPitch = sp.outPitch;
        fp.W = sp.W; fp.H = sp.H; fp.nearC = sp.nearC;
        fp.frac = (double)set.globalFallback;
        fp.untrusted = sp.untrusted;
        fp.untrustedNext = next;
        fp.rowBytes = (size_t)W * planeBytes(fmt);
        if (chromaBytes(fmt)) {
            fp.cbytes = (size_t)((W + 1) / 2) * chromaBytes(fmt);
            fp.ch = (int)(H + 1) / 2;
            fp.ac = sp.ac; fp.cc = sp.cc; fp.cpitch = sp.cpitch; fp.outc = sp.outc; fp.outCPitch = sp.outCPitch;
        }
        return fp;
    }

    // recordSynthBlur (gpu/framegen.cpp:3534-3630): every sample's synthesis parameters as recordSynth(t_k) builds
    // them, the per-sample counters zeroed, then the blur's main and fix-up passes
    bool blur(cudaStream_t s, const Frame& prev, const Frame& curr, const Frame& out, float t0, float t1,
              const uint32_t* ma, const uint32_t* mc) {
        float tk[Interpolator::kBlurMaxSamples];
        uint32_t q[Interpolator::kBlurMaxSamples];
        const int n = (int)Interpolator::blurPlan(set.blurSamples, set.blurWeights, t0, t1, tk, q);
        if (n < 1) return false;
        fgk::BlurParams bp{};
        bp.base = synthParams(prev, curr, out, 0.5f, nullptr);
        bp.base.emap = nullptr;
        bp.base.uiA = ma;
        bp.base.uiC = mc;
        for (int k = 0; k < n; k++) {
            fgk::BlurSample& m = bp.smp[k];
            m.q = q[k];
            if (tk[k] <= 0.0f || tk[k] >= 1.0f) {
                m.mode = tk[k] <= 0.0f ? 1 : 2;
                continue;
            }
            const fgk::SynthParams sp = synthParams(prev, curr, out, tk[k], nullptr);
            m.lookup = sp.lookup; m.mid = sp.mid; m.nearC = sp.nearC;
            m.s = sp.s; m.ka = sp.ka; m.kc = sp.kc; m.wA = sp.wA; m.wC = sp.wC;
        }
        bp.n = n;
        bp.frac = (double)set.globalFallback;
        bp.cnt = blurCnt;
        if (!check(cudaMemsetAsync(blurCnt, 0, (size_t)fgk::kBlurMax * 4, s))) return false;
        const bool rgba8 = fmt == Format::Rgba8;
        int nSynth = 0;
        for (int k = 0; k < n; k++) nSynth += bp.smp[k].mode == 0;
        if (rgba8 && blurSub && (uint32_t)nSynth <= blurSubCap) {
            // each synthesized sample to its own sub-frame by the synthesis kernel, counting into blurCnt[k]; then
            // one blend of the sub-frames and the real frames (the flick test from the counters)
            fgk::BlurBlendParams bb{};
            bb.a = bp.base.a; bb.c = bp.base.c; bb.pitch = bp.base.pitch;
            bb.sub = blurSub; bb.subPitch = blurSubPitch; bb.subStride = blurSubPitch * H;
            bb.out = (uint8_t*)out.data; bb.outPitch = out.pitch;
            bb.W = (int)W; bb.H = (int)H; bb.n = n;
            bb.frac = bp.frac;
            bb.cnt = blurCnt;
            int slot = 0;
            for (int k = 0; k < n; k++) {
                const fgk::BlurSample& m = bp.smp[k];
                bb.mode[k] = m.mode;
                bb.nearC[k] = m.nearC;
                bb.q[k] = m.q;
                if (m.mode != 0) continue;
                bb.slot[k] = slot;
                fgk::SynthParams sp = synthParams(prev, curr, out, tk[k], blurCnt + k);
                sp.out = blurSub + (size_t)slot * bb.subStride;
                sp.outPitch = blurSubPitch;
                sp.emap = nullptr;
                sp.uiA = ma;
                sp.uiC = mc;
                if (!check(fgk::launchSynth(sp, s))) return false;
                slot++;
            }
            stamp(s, "blur samples");
            if (!check(fgk::launchBlurBlend(bb, s))) return false;
            stamp(s, "blur blend");
            return !mc || uiPatch(s, curr, out, mc);
        }
        if (!check(rgba8 ? fgk::launchSynthBlur(bp, 0, s) : fgk::launchSynthBlurFmt(bp, 0, s))) return false;
        stamp(s, "blur resolve");
        if (!check(rgba8 ? fgk::launchSynthBlur(bp, 1, s) : fgk::launchSynthBlurFmt(bp, 1, s))) return false;
        stamp(s, "blur fixup");
        return !mc || uiPatch(s, curr, out, mc);
    }

    // ma / mc: the pair's UI masks (CrosshairV2) or null: the tap rejection in the synthesis, then curr's UI pixels
    // pasted back over the finished frame
    bool synth(cudaStream_t s, const Frame& prev, const Frame& curr, const Frame& out, float t, const uint32_t* ma,
               const uint32_t* mc) {
        fgk::SynthParams sp = synthParams(prev, curr, out, t, &st->untrusted[parity]);
        sp.uiA = ma;
        sp.uiC = mc;
        if (!check(fmt == Format::Rgba8 ? fgk::launchSynth(sp, s) : fgk::launchSynthFmt(sp, s))) return false;
        stamp(s, "synth");
        const fgk::FallbackParams fp = fallbackParams(sp, &st->untrusted[parity ^ 1u]);
        if (!check(fmt == Format::Rgba8 ? fgk::launchFallback(fp, s) : fgk::launchFallbackFmt(fp, s))) return false;
        stamp(s, "fallback");
        lastParity = parity;
        parity ^= 1u;
        return !mc || uiPatch(s, curr, out, mc);
    }
};

Interpolator::~Interpolator() { destroy(); }

bool Interpolator::validate(const Settings& s) {
    auto in = [](float v, float lo, float hi) { return std::isfinite(v) && v >= lo && v <= hi; };
    return in(s.trustLow, 0.0f, 255.0f) && in(s.trustHigh, 0.0f, 255.0f) && s.trustHigh - s.trustLow >= 1.0f &&
           in(s.globalFallback, 0.0f, 1.0f) && s.globalFallback > 0.0f && in(s.sceneCutSad, 0.0f, 255.0f) &&
           s.sceneCutSad > 0.0f && in(s.hudBonus, 0.0f, 255.0f) && in(s.smoothBonus, 0.0f, 255.0f) &&
           in(s.searchPenalty, 0.0f, 255.0f) && s.searchRadius >= 1 && s.searchRadius <= 12 && s.searchRadiusTop >= 1 &&
           s.searchRadiusTop <= 12 && (s.flowScale == 1 || s.flowScale == 2 || s.flowScale == 4) &&
           s.pyramidMinSide >= 16 && s.pyramidMinSide <= 256 &&
           (uint32_t)s.uiProtection <= (uint32_t)UiProtection::CrosshairV2 &&
           (uint32_t)s.motionVersion <= (uint32_t)MotionVersion::V3 && s.blurSamples <= kBlurMaxSamples &&
           (uint32_t)s.blurWeights <= (uint32_t)BlurWeights::Gaussian &&
           // the other versions' and UI protection's fields, with the reference's ranges (gpu/framegen.cpp:1688-1699)
           (uint32_t)s.v2Mode <= (uint32_t)V2Mode::Performance && (uint32_t)s.v3Guard <= (uint32_t)V3Guard::V2Motion &&
           (uint32_t)s.learnedNet < kLearnedNets && in(s.v3Smear, 0.0f, 1.0f) && in(s.v3OcclSoft, 0.25f, 4.0f) &&
           in(s.v3Unsure, 0.25f, 4.0f) && in(s.v3SceneCut, 0.0f, 4.0f) && in(s.uiCrosshairArea, 0.0f, 1.0f) &&
           s.uiCrosshairArea > 0.0f && in(s.uiBoxHeightFrac, 0.0f, 1.0f) && s.uiBoxWidth <= 16384 &&
           s.uiBoxHeight <= 16384 && s.uiBoxOffsetX >= -16384 && s.uiBoxOffsetX <= 16384 && s.uiBoxOffsetY >= -16384 &&
           s.uiBoxOffsetY <= 16384 && s.uiStillFrames >= 1 && s.uiStillFrames <= 255 &&
           in(s.uiStillThreshold, 0.0f, 255.0f) && s.uiInpaintReach >= 1 && s.uiInpaintReach <= 16 &&
           in(s.uiMaxStillFraction, 0.0f, 1.0f) && s.uiMaxStillFraction > 0.0f && in(s.uiContrastThreshold, 0.0f, 255.0f) &&
           s.uiLeaveFrames >= 1 && s.uiLeaveFrames <= 255 && s.uiReentryFrames <= 255 && s.uiHistory >= 3 &&
           s.uiHistory <= 65;
}

const char* Interpolator::settingsError(const Settings& s, Format f) {
    if (!validate(s)) return kErrSettings;
    if (s.motionVersion != MotionVersion::V1) return kErrVersion;
    if (s.uiProtection != UiProtection::Off && s.uiProtection != UiProtection::CrosshairV2) return kErrUi;
    if (s.uiProtection == UiProtection::CrosshairV2 && (uint32_t)f > (uint32_t)Format::P010) return kErrUiFormat;
    return nullptr;
}

const char* Interpolator::settingsError(const Settings& s) const {
    if (const char* e = settingsError(s, m ? m->fmt : Format::Rgba8)) return e;
    return m && m->W ? sizeError(m->W, m->H) : nullptr;
}

const char* Interpolator::sizeError(uint32_t w, uint32_t h) const {
    if (!m) return "not initialised";
    if (w < kMinSize || h < kMinSize) return kErrMinSize;
    if ((uint64_t)w * h > (1ull << 30)) return kErrMaxSize;
    return nullptr;
}

bool Interpolator::init(const InitInfo& ii) {
    destroy();
    err_ = nullptr;
    Format fmt;
    if (!validate(ii.settings)) { err_ = "missing device, or invalid settings"; return false; }
    if (!formatOf(ii.viewFormat, &fmt)) { err_ = kErrNoFormat; return false; }
    if (const char* e = settingsError(ii.settings, fmt)) { err_ = e; return false; }
    if (fmt == Format::RgbaF16 && ii.transfer == Transfer::Linear && !(ii.linearWhiteNits > 0.0f && ii.linearWhiteNits <= 10000.0f)) {
        err_ = kErrNits;
        return false;
    }
    if ((fmt == Format::Nv12 || fmt == Format::P010) && (uint32_t)ii.yuvMatrix > (uint32_t)YuvMatrix::Bt2020) {
        err_ = kErrYuvMatrix;
        return false;
    }
    if (ii.width < kMinSize || ii.height < kMinSize) { err_ = kErrMinSize; return false; }
    if ((uint64_t)ii.width * ii.height > (1ull << 30)) { err_ = kErrMaxSize; return false; }
    int dev = ii.device, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); err_ = kErrDevice; return false; }
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); err_ = kErrDevice; return false; }
    if (dev >= ndev) { err_ = kErrDevice; return false; }
    {
        DeviceGuard g(dev);
        if (fgk::prepareKernels() != cudaSuccess || fgk::prepareFormatKernels() != cudaSuccess) {
            cudaGetLastError();
            err_ = kErrDevice;
            return false;
        }
    }
    m = new Impl();
    m->device = dev;
    m->info = ii;
    m->fmt = fmt;
    m->viewFormat = ii.viewFormat;
    m->set = ii.settings;
    m->ri = ii.viewFormat == kVkFormatR8G8B8A8Unorm ? 0 : 2;
    m->gi = 1;
    m->bi = ii.viewFormat == kVkFormatR8G8B8A8Unorm ? 2 : 0;
    m->fc = makeFmtConst(fmt, ii.viewFormat, ii);
    m->updateTrust();
    if (const char* e = m->allocSize(ii.width, ii.height)) {
        err_ = e;
        delete m;
        m = nullptr;
        return false;
    }
    return true;
}

Format Interpolator::format() const { return m ? m->fmt : Format::Rgba8; }

void Interpolator::destroy() {
    delete m;
    m = nullptr;
}

bool Interpolator::resize(uint32_t w, uint32_t h, uint32_t viewFormat) {
    if (!m) return false;
    Format f;
    if (!formatOf(viewFormat, &f) || f != m->fmt) return false;
    if (sizeError(w, h)) return false;
    m->viewFormat = viewFormat;
    m->ri = viewFormat == kVkFormatR8G8B8A8Unorm ? 0 : 2;
    m->bi = viewFormat == kVkFormatR8G8B8A8Unorm ? 2 : 0;
    m->fc = makeFmtConst(m->fmt, viewFormat, m->info);
    return m->allocSize(w, h) == nullptr;
}

// A change of static-UI protection's mode or box restarts its state and drops the current estimate (gpu/framegen.h:590-592)
static bool uiGeometryChanged(const Settings& a, const Settings& b) {
    return a.uiProtection != b.uiProtection || a.uiBoxHeightFrac != b.uiBoxHeightFrac || a.uiBoxWidth != b.uiBoxWidth ||
           a.uiBoxHeight != b.uiBoxHeight || a.uiCrosshairArea != b.uiCrosshairArea || a.uiBoxOffsetX != b.uiBoxOffsetX ||
           a.uiBoxOffsetY != b.uiBoxOffsetY;
}

bool Interpolator::setSettings(const Settings& s) {
    if (!m || settingsError(s) || s.flowScale != m->set.flowScale || s.pyramidMinSide != m->set.pyramidMinSide) return false;
    const Settings old = m->set;
    const bool restart = uiGeometryChanged(old, s);
    m->set = s;
    if (m->uiSetup(restart)) {   // the allocation failed: nothing changed
        m->set = old;
        return false;
    }
    if (restart) m->haveEst = m->estUi = false;
    m->updateTrust();
    m->blurSetup();
    return true;
}

bool Interpolator::reconfigure(const Settings& s) {
    if (!m || settingsError(s)) return false;
    const Settings old = m->set;
    const bool structural = s.flowScale != old.flowScale || s.pyramidMinSide != old.pyramidMinSide;
    m->set = s;
    m->updateTrust();
    if (structural && m->W) {
        if (m->allocSize(m->W, m->H)) { m->set = old; m->updateTrust(); m->allocSize(m->W, m->H); return false; }
    } else if (m->W) {
        const bool restart = uiGeometryChanged(old, s);
        if (m->uiSetup(restart)) { m->set = old; m->updateTrust(); return false; }
        if (restart) m->haveEst = m->estUi = false;
        m->blurSetup();
    }
    return true;
}

Settings Interpolator::settings() const { return m ? m->set : Settings{}; }

void Interpolator::beginFrame() {
    if (m) m->estSets = m->synthSets = 0;
}

void Interpolator::releaseUnusedUi() {
    if (!m) return;
    DeviceGuard g(m->device);
    if (!m->uiOn()) {
        m->uiFree();
        return;
    }
    // free the masks beyond uiHistory (uiEvict already keeps at most uiHistory frames): the forgotten entries go
    for (size_t i = m->uiE.size(); i-- > 0 && m->uiE.size() > m->set.uiHistory;) {
        if (m->uiE[i].key) continue;
        if (m->uiE[i].mask) cudaFree(m->uiE[i].mask);
        m->uiE.erase(m->uiE.begin() + (long)i);
    }
    if (m->estUi) {   // the kept entries moved: the estimate's pair by key (same stamps, or the synthesis refuses)
        m->estEnt[0] = m->uiFind(m->estPrev);
        m->estEnt[1] = m->uiFind(m->estCurr);
        m->estUi = m->estEnt[0] >= 0 && m->estEnt[1] >= 0;
    }
}
void Interpolator::releaseUnusedMotion() {}   // V1 is the only motion version

bool Interpolator::recordEstimate(cudaStream_t stream, Frame prev, Frame curr) {
    if (!m || !m->W) return false;
    if (!m->frameOk(prev) || !m->frameOk(curr) || !m->samePitch(prev, curr)) return false;
    if (m->estSets >= kSetRing) return false;
    DeviceGuard g(m->device);
    m->estSets++;
    m->haveEst = false;
    m->estUi = false;
    if (m->uiOn() && !m->uiExplicit && m->uiState) {   // the implicit observe (gpu/framegen.h:602-609)
        if (m->profiling && m->evCount == 0) m->stamp(stream, "start");
        if (m->uiFind(prev.data) < 0 && !m->uiObserve(stream, prev, false)) return false;
        if (m->uiLast != curr.data && !m->uiObserve(stream, curr, false)) return false;
    }
    bool ui = false;
    int ep = -1, ec = -1;
    if (m->uiOn()) {   // the pair is protected if both frames are kept
        ep = m->uiFind(prev.data);
        ec = m->uiFind(curr.data);
        ui = ep >= 0 && ec >= 0;
    }
    m->fillMask[0] = ui && m->set.uiEstimateFill ? m->uiE[ep].mask : nullptr;
    m->fillMask[1] = ui && m->set.uiEstimateFill ? m->uiE[ec].mask : nullptr;
    const bool ok = m->estimate(stream, prev, curr);
    m->fillMask[0] = m->fillMask[1] = nullptr;
    if (!ok) return false;
    m->haveEst = true;
    m->estPrev = prev.data;
    m->estCurr = curr.data;
    m->estUi = ui;
    if (ui) {
        m->estEnt[0] = ep;
        m->estEnt[1] = ec;
        m->estStamp[0] = m->uiE[ep].stamp;
        m->estStamp[1] = m->uiE[ec].stamp;
    }
    return true;
}

bool Interpolator::recordObserve(cudaStream_t stream, Frame frame) {
    if (!m || !m->W) return false;
    if (!m->uiOn()) return true;
    if (!m->frameOk(frame) || !m->uiState) return false;
    DeviceGuard g(m->device);
    m->uiExplicit = true;
    if (m->profiling && m->evCount == 0) m->stamp(stream, "start");
    return m->uiObserve(stream, frame, false);
}

bool Interpolator::recordTrack(cudaStream_t stream, Frame frame) {
    if (!m || !m->W) return false;
    if (!m->uiOn()) return true;
    if (!m->frameOk(frame) || !m->uiState) return false;
    DeviceGuard g(m->device);
    if (m->profiling && m->evCount == 0) m->stamp(stream, "start");
    return m->uiObserve(stream, frame, true);
}

size_t Interpolator::uiTraceBytes() const {
    if (!m || !m->uiOn() || !m->uiState) return 0;
    return (size_t)m->uiWork[2] * m->uiWork[3] * 16 + ((size_t)fgk::kUiMaskHeader + (size_t)m->uiStride * m->uiWork[3]) * 4;
}

bool Interpolator::uiTrace(cudaStream_t stream, const void* frame, void* dst) {
    const size_t total = uiTraceBytes();
    if (!total || !dst) return false;
    DeviceGuard g(m->device);
    const size_t sb = (size_t)m->uiWork[2] * m->uiWork[3] * 16;
    char* d = static_cast<char*>(dst);
    if (!m->check(cudaMemcpyAsync(d, m->uiState, sb, cudaMemcpyDeviceToDevice, stream))) return false;
    const int k = frame ? m->uiFind(frame) : -1;
    return m->check(k >= 0 ? cudaMemcpyAsync(d + sb, m->uiE[k].mask, total - sb, cudaMemcpyDeviceToDevice, stream)
                           : cudaMemsetAsync(d + sb, 0, total - sb, stream));
}

void Interpolator::boxSize(const Settings& set, uint32_t w, uint32_t h, uint32_t* boxW, uint32_t* boxH) {
    const int fw = (int)w, fh = (int)h;
    int side;
    if (set.uiBoxHeightFrac > 0.0f)
        side = std::min(std::max((int)std::lround((double)h * set.uiBoxHeightFrac), 8), std::min(fw, fh));
    else   // the legacy area fraction
        side = std::min(std::max((int)std::lround(std::sqrt((double)set.uiCrosshairArea * fw * fh)), 32), std::min(fw, fh));
    *boxW = set.uiBoxWidth ? (uint32_t)std::min(std::max((int)set.uiBoxWidth, 4), fw) : (uint32_t)side;
    *boxH = set.uiBoxHeight ? (uint32_t)std::min(std::max((int)set.uiBoxHeight, 4), fh) : (uint32_t)side;
}

void Interpolator::boxRect(const Settings& set, uint32_t w, uint32_t h, int32_t r[4]) {
    uint32_t bw, bh;
    boxSize(set, w, h, &bw, &bh);
    r[2] = (int32_t)bw;
    r[3] = (int32_t)bh;
    r[0] = std::min(std::max(((int)w - r[2]) / 2 + set.uiBoxOffsetX, 0), (int)w - r[2]);
    r[1] = std::min(std::max(((int)h - r[3]) / 2 + set.uiBoxOffsetY, 0), (int)h - r[3]);
}

uint32_t Interpolator::boxMargin(const Settings& set) {
    return set.uiProtection == UiProtection::Crosshair ? 2u : set.uiProtection == UiProtection::CrosshairV2 ? 1u : 0u;
}

void Interpolator::workRect(const Settings& set, uint32_t w, uint32_t h, int32_t r[4]) {
    boxRect(set, w, h, r);
    const int mg = (int)boxMargin(set);
    const int x0 = std::max(r[0] - mg, 0), y0 = std::max(r[1] - mg, 0);
    const int x1 = std::min(r[0] + r[2] + mg, (int)w), y1 = std::min(r[1] + r[3] + mg, (int)h);
    r[0] = x0; r[1] = y0; r[2] = x1 - x0; r[3] = y1 - y0;
}

bool Interpolator::recordSynth(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t) {
    if (!m || !m->W || !(t > 0.0f && t < 1.0f)) return false;
    if (!m->haveEst || prev.data != m->estPrev || curr.data != m->estCurr) return false;
    if (!m->frameOk(prev) || !m->frameOk(curr) || !m->frameOk(out) || !m->samePitch(prev, curr)) return false;
    if (m->synthSets >= kSetRing) return false;
    const uint32_t *ma, *mc;
    if (!m->uiPairMasks(ma, mc)) return false;   // an entry the estimate used was evicted or replaced since
    DeviceGuard g(m->device);
    m->synthSets++;
    if (m->profiling && m->evCount == 0) m->stamp(stream, "start");
    return m->synth(stream, prev, curr, out, t, ma, mc);
}

uint32_t Interpolator::blurPlan(uint32_t samples, BlurWeights weights, float t0, float t1, float* times, uint32_t* q) {
    if (!(t0 >= 0.0f && t1 <= 1.0f && t0 <= t1) || !times || !q) return 0;   // (also false for NaN)
    const bool on = samples >= 2 && t0 < t1;
    const int n = on ? (int)std::min(samples, kBlurMaxSamples) : 1;
    double w[kBlurMaxSamples], frac[kBlurMaxSamples], sum = 0.0;
    for (int k = 0; k < n; k++) {
        // the midpoints of n equal slices of [t0, t1] (gpu/framegen.cpp:3552-3557); one instant t1 without blur
        const double t = on ? t0 + ((double)t1 - (double)t0) * (k + 0.5) / n : (double)t1;
        times[k] = std::min(std::max((float)t, t0), t1);
        const double x = (2.0 * k + 1.0 - n) / n;   // the slice centre; the window ends are x = -+1
        w[k] = weights == BlurWeights::Gaussian ? std::exp(-2.0 * x * x) : 1.0;
        sum += w[k];
    }
    // the normalised weights in units of 2^-16: floors, then the remaining units to the largest remainders (ties to
    // the lower sample), so that they sum to exactly 2^16
    int64_t tot = 0;
    for (int k = 0; k < n; k++) {
        const double r = w[k] / sum * 65536.0;
        q[k] = (uint32_t)std::floor(r);
        frac[k] = r - (double)q[k];
        tot += q[k];
    }
    while (tot != 65536) {
        int best = 0;
        for (int k = 1; k < n; k++)
            if (tot < 65536 ? frac[k] > frac[best] : frac[k] < frac[best]) best = k;
        if (tot < 65536) { q[best]++; frac[best] -= 1.0; tot++; }
        else { q[best]--; frac[best] += 1.0; tot--; }
    }
    return (uint32_t)n;
}

bool Interpolator::recordSynthBlur(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t0, float t1) {
    if (!m || !m->W || !(t0 >= 0.0f && t1 <= 1.0f && t0 <= t1)) return false;   // (also false for NaN)
    const bool blur = m->set.blurSamples >= 2 && t0 < t1;
    if (!blur && t1 > 0.0f && t1 < 1.0f) return recordSynth(stream, prev, curr, out, t1);   // one interior instant
    if (!m->haveEst || prev.data != m->estPrev || curr.data != m->estCurr) return false;
    if (!m->frameOk(prev) || !m->frameOk(curr) || !m->frameOk(out) || !m->samePitch(prev, curr)) return false;
    if (m->synthSets >= kSetRing) return false;
    const uint32_t *ma, *mc;
    if (!m->uiPairMasks(ma, mc)) return false;
    DeviceGuard g(m->device);
    m->synthSets++;
    if (m->profiling && m->evCount == 0) m->stamp(stream, "start");
    return m->blur(stream, prev, curr, out, t0, t1, ma, mc);
}

bool Interpolator::record(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t) {
    if (!m || !m->W || !(t > 0.0f && t < 1.0f)) return false;
    if (!m->frameOk(out) || m->estSets >= kSetRing || m->synthSets >= kSetRing) return false;
    return recordEstimate(stream, prev, curr) && recordSynth(stream, prev, curr, out, t);
}

const char* Interpolator::lastCudaError() const { return m ? m->lastErr : nullptr; }

bool Interpolator::setSeedNet(const float* params, uint32_t level) {
    if (!m) return false;
    if (params) {
        m->snParams.assign(params, params + fgk::kSnParams);
        m->snLevelReq = (int)std::min<uint32_t>(level, fgk::kMaxLevels - 1);
    } else {
        m->snParams.clear();
        m->snLevelReq = -1;
    }
    if (!m->W) return true;
    return m->allocSize(m->W, m->H) == nullptr;   // the histogram bound and the net's buffers depend on the level
}

uint32_t Interpolator::seedNetLevel() const { return m && m->snK >= 0 ? (uint32_t)m->snK : UINT32_MAX; }

bool Interpolator::setProfiling(bool on) {
    if (!m) return false;
    m->profiling = on;
    m->evCount = 0;
    return true;
}

bool Interpolator::readTimings(std::vector<const char*>& names, std::vector<uint64_t>& ticks) {
    names.clear();
    ticks.clear();
    if (!m || !m->profiling || m->evCount < 2) return false;
    DeviceGuard g(m->device);
    if (cudaEventSynchronize(m->events[m->evCount - 1]) != cudaSuccess) { cudaGetLastError(); return false; }
    for (size_t i = 1; i < m->evCount; i++) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, m->events[i - 1], m->events[i]) != cudaSuccess) { cudaGetLastError(); return false; }
        names.push_back(m->evNames[i]);
        ticks.push_back((uint64_t)std::llround((double)ms * 1e6));
    }
    return true;
}

bool Interpolator::readCosts(CostTimings& c) {
    c = CostTimings{};
    std::vector<const char*> names;
    std::vector<uint64_t> ns;
    if (!readTimings(names, ns)) return false;
    static const char* const kEstimate[] = {"luma", "pyramid", "seed net", "subpixel", "pixel field"};
    static const char* const kSynth[] = {"synth", "fallback", "blur resolve", "blur fixup", "blur samples", "blur blend"};
    auto in = [](const char* n, const auto& set) {
        for (const char* s : set)
            if (std::strcmp(n, s) == 0) return true;
        return false;
    };
    uint64_t est = 0, syn = 0;
    bool haveEst = false;
    for (size_t i = 0; i < names.size(); i++) {
        const char* n = names[i];
        if (in(n, kEstimate) || std::strncmp(n, "level ", 6) == 0) { est += ns[i]; haveEst = true; }
        else if (in(n, kSynth)) {
            syn += ns[i];
            if (std::strcmp(n, "synth") == 0 || std::strcmp(n, "blur resolve") == 0 || std::strcmp(n, "blur samples") == 0)
                c.synths++;
        }
    }
    if (haveEst) c.estimateMs = (float)((double)est * 1e-6);
    if (c.synths) c.synthMs = (float)((double)syn * 1e-6 / c.synths);
    if (m->profileRead != m->profileNo || m->costSeq == 0) { m->costSeq++; m->profileRead = m->profileNo; }
    c.seq = m->costSeq;
    return true;
}

bool Interpolator::recordDebugCounters(cudaStream_t stream, void* dst) {
    if (!m || !m->W || !dst) return false;
    DeviceGuard g(m->device);
    return cudaMemcpyAsync(dst, &m->st->untrusted[m->lastParity], 4, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
           cudaMemcpyAsync((char*)dst + 4, &m->st->sadSum256, 4, cudaMemcpyDeviceToDevice, stream) == cudaSuccess;
}

uint32_t Interpolator::debugSadBlocks() const { return m && m->W ? (uint32_t)(m->L.lv[0].bw * m->L.lv[0].bh) : 0; }

bool Interpolator::debugMapLayout(DebugMapLayout& l) const {
    if (!m || !m->W) return false;
    l.W = m->W; l.H = m->H; l.fw = m->L.fw; l.fh = m->L.fh;
    l.bw = m->L.lv[0].bw; l.bh = m->L.lv[0].bh; l.fscale = m->set.flowScale; l.eStride = (m->W + 3) / 4;
    // contiguous, as gpu/framegen.cpp:2096-2099 lays it out: the bytes after an fgmaps header (gpu/fgtest.cpp:777-789)
    l.blockOff = 0;
    l.pixOff = (uint64_t)l.bw * l.bh * 8;
    l.eOff = l.pixOff + (uint64_t)l.fw * l.fh * 8;
    l.size = l.eOff + (uint64_t)l.eStride * 4 * l.H;
    return true;
}

bool Interpolator::recordDebugMaps(cudaStream_t stream, void* dst) {
    DebugMapLayout l;
    if (!debugMapLayout(l) || !dst) return false;
    DeviceGuard g(m->device);
    char* d = (char*)dst;
    const float2* blk = m->field + (m->set.subpixel ? m->L.sub1 : m->L.lv[0].fM);
    return cudaMemcpyAsync(d + l.blockOff, blk, (size_t)l.bw * l.bh * 8, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
           cudaMemcpyAsync(d + l.pixOff, m->pf, (size_t)l.fw * l.fh * 8, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
           cudaMemcpyAsync(d + l.eOff, m->emap, (size_t)l.eStride * 4 * l.H, cudaMemcpyDeviceToDevice, stream) == cudaSuccess;
}

bool Interpolator::setDebugCapture(bool on) {
    if (!m) return false;
    m->capture = on;
    return true;
}

bool Interpolator::traceLayout(TraceLayout& l) const {
    if (!m || !m->W) return false;
    std::memset(&l, 0, sizeof(l));
    const SizeLayout& L = m->L;
    l.nLevels = (uint32_t)L.lv.size(); l.fw = L.fw; l.fh = L.fh;
    for (size_t i = 0; i < L.lv.size(); i++) {
        l.lw[i] = L.lv[i].w; l.lh[i] = L.lv[i].h; l.bw[i] = L.lv[i].bw; l.bh[i] = L.lv[i].bh;
    }
    uint64_t o = 0;
    l.lumaOff = o; l.lumaBytes = L.lumaFloats * 4; o = alignUp(o + l.lumaBytes, 256);
    l.fieldOff = o; l.fieldBytes = L.fieldF2 * 8; o = alignUp(o + l.fieldBytes, 256);
    l.medOff = o; o = alignUp(o + (uint64_t)L.lv.size() * 8, 256);
    l.sadOff = o; o = alignUp(o + (uint64_t)L.lv[0].bw * L.lv[0].bh * 4, 256);
    l.pfOff = o; o = alignUp(o + (uint64_t)L.fw * L.fh * 8, 256);
    l.stateOff = o; o = alignUp(o + 16, 256);
    l.seedLevel = m->snK >= 0 ? (uint32_t)m->snK : UINT32_MAX;
    l.seedOff = o;
    if (m->snK >= 0) o += (uint64_t)L.lv[m->snK].bw * L.lv[m->snK].bh * fgk::kSeedNetOut * 4;
    l.size = o;
    return true;
}

bool Interpolator::recordTrace(cudaStream_t stream, void* dst) {
    TraceLayout l;
    if (!traceLayout(l) || !dst) return false;
    DeviceGuard g(m->device);
    char* d = (char*)dst;
    const auto D2D = cudaMemcpyDeviceToDevice;
    bool ok = cudaMemcpyAsync(d + l.lumaOff, m->luma, l.lumaBytes, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.fieldOff, m->field, l.fieldBytes, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.medOff, m->st->med, (size_t)l.nLevels * 8, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.sadOff, m->sads, (size_t)l.bw[0] * l.bh[0] * 4, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.pfOff, m->pf, (size_t)l.fw * l.fh * 8, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.stateOff, &m->st->cut, 4, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.stateOff + 4, &m->st->sadMean, 4, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.stateOff + 8, &m->st->sadSum256, 4, D2D, stream) == cudaSuccess &&
              cudaMemcpyAsync(d + l.stateOff + 12, &m->st->err, 4, D2D, stream) == cudaSuccess;
    if (ok && m->snK >= 0)
        ok = cudaMemcpyAsync(d + l.seedOff, m->snOut, (size_t)l.bw[m->snK] * l.bh[m->snK] * fgk::kSeedNetOut * 4, D2D,
                             stream) == cudaSuccess;
    return ok;
}


// ================================================================================================== batches
struct Batch::Impl {
    static constexpr int kRing = 8;   // pinned upload buffers: at most this many records in flight
    static constexpr int kFormats = 5;   // persistent synthesis launches: at most one per frame format
    std::vector<std::unique_ptr<Interpolator>> slots;
    std::vector<uint32_t> mult;
    Shape shape;
    const char* err = nullptr;
    int device = -1, sms = 0;
    int maxItems = 0;
    // the work list on the device, one blob: items, fallbacks, tile starts, tiles across; then the counters
    char* dev = nullptr;
    unsigned int* counters = nullptr;   // maxItems per-item untrusted counters + a work counter per format
    size_t oFall = 0, oStart = 0, oTx = 0, blobBytes = 0;
    char* host = nullptr;               // kRing x blobBytes, pinned
    int ring = 0;
    // the fork / join pool of the slots' estimates
    static constexpr int kMaxStreams = 8;
    bool mergeable() const;   // no slot needs a per-slot estimate pass (UI protection, the seed net, profiling)
    bool mergedEstimates(cudaStream_t s, const Frame* prev, const Frame* curr, const std::vector<int>& idx);
    cudaStream_t pool[kMaxStreams] = {};
    cudaEvent_t fork = nullptr, join[kMaxStreams] = {};

    ~Impl() {
        release();
        DeviceGuard g(device);
        for (int i = 0; i < kMaxStreams; i++) {
            if (pool[i]) cudaStreamDestroy(pool[i]);
            if (join[i]) cudaEventDestroy(join[i]);
        }
        if (fork) cudaEventDestroy(fork);
    }
    bool makePool() {
        if (fork) return true;
        DeviceGuard g(device);
        bool ok = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess;
        for (int i = 0; ok && i < kMaxStreams; i++)
            ok = cudaStreamCreateWithFlags(&pool[i], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) cudaGetLastError();
        return ok;
    }
    void release() {
        DeviceGuard g(device);
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
        dev = nullptr;
        host = nullptr;
        counters = nullptr;
    }
    bool grow() {   // the work-list buffers for the current slots (called by add, outside any capture)
        DeviceGuard g(device);
        release();
        maxItems = 0;
        for (uint32_t v : mult) maxItems += (int)v - 1;
        const size_t n = (size_t)std::max(maxItems, 1);
        oFall = alignUp(n * sizeof(fgk::SynthParams), 256);
        oStart = alignUp(oFall + n * sizeof(fgk::FallbackParams), 256);
        oTx = alignUp(oStart + (n + 1) * 4, 256);
        blobBytes = alignUp(oTx + n * 4, 256);
        if (cudaMalloc(&dev, blobBytes + (n + kFormats) * 4) != cudaSuccess ||
            cudaMallocHost(&host, blobBytes * kRing) != cudaSuccess) {
            cudaGetLastError();
            release();
            return false;
        }
        counters = (unsigned int*)(dev + blobBytes);
        return true;
    }
};

Batch::Batch() : m(new Impl()) {}
Batch::~Batch() { delete m; }
const char* Batch::error() const { return m->err; }
uint32_t Batch::slots() const { return (uint32_t)m->slots.size(); }
uint32_t Batch::synthsOf(uint32_t i) const { return i < m->mult.size() ? m->mult[i] - 1 : 0; }
Interpolator* Batch::slot(uint32_t i) { return i < m->slots.size() ? m->slots[i].get() : nullptr; }
Batch::Shape Batch::shape() const { return m->shape; }
bool Batch::setShape(const Shape& s) {
    if (s.ctasPerSm > 4 || s.order > 1 || s.streams < 1 || s.streams > (uint32_t)Impl::kMaxStreams || s.mergeEstimates > 8)
        return false;
    m->shape = s;
    return true;
}

int Batch::add(const InitInfo& ii, uint32_t multiplier) {
    m->err = nullptr;
    if (multiplier < 2 || multiplier > 8) { m->err = "the multiplier must be 2 .. 8"; return -1; }
    int dev = ii.device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); m->err = kErrDevice; return -1; }
    if (m->device >= 0 && dev != m->device) { m->err = "every slot of a batch must be on the batch's device"; return -1; }
    std::unique_ptr<Interpolator> I(new Interpolator());
    InitInfo j = ii;
    j.device = dev;
    if (!I->init(j)) { m->err = I->initError(); return -1; }
    m->device = dev;
    if (!m->sms && cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        m->err = kErrDevice;
        return -1;
    }
    m->slots.push_back(std::move(I));
    m->mult.push_back(multiplier);
    if (!m->makePool() || !m->grow()) {
        m->slots.pop_back();
        m->mult.pop_back();
        m->grow();
        m->err = kErrAlloc;
        return -1;
    }
    return (int)m->slots.size() - 1;
}

// Items of one estimate pass grouped by key (the kernel variant they take) and launched merged, at most kMergeMax
// per launch; launch(merged, key)
template <class P, class Launch>
static cudaError_t launchMergedGroups(const std::vector<P>& items, const std::vector<int>& keys, Launch launch) {
    if (items.empty()) return cudaSuccess;
    std::vector<int> idx(items.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    std::unique_ptr<fgk::Merged<P>> mg(new fgk::Merged<P>());
    size_t i = 0;
    while (i < idx.size()) {
        const int key = keys[idx[i]];
        mg->n = 0;
        while (i < idx.size() && keys[idx[i]] == key && mg->n < fgk::kMergeMax) mg->item[mg->n++] = items[idx[i++]];
        const cudaError_t e = launch(*mg, key);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Merged estimates need every slot's estimate to be the plain pass sequence
bool Batch::Impl::mergeable() const {
    for (const auto& I : slots) {
        const Interpolator::Impl& im = *I->m;
        if (im.uiOn() || im.snK >= 0 || im.profiling) return false;
    }
    return true;
}

// The estimates of the slots idx (Shape::mergeEstimates): one launch per pass for all of them on the caller's stream,
// in the order an estimate runs its passes (luma, levels from the coarsest down to level 0 with the finest levels
// aligned, so level l of every slot that has one is searched in the same launch, sub-pixel, pixel field). The same
// kernels' work per slot as recordEstimate; only the launches are shared.
bool Batch::Impl::mergedEstimates(cudaStream_t s, const Frame* prev, const Frame* curr, const std::vector<int>& idx) {
    const int ns = (int)idx.size();
    for (int j = 0; j < ns; j++) {
        const int i = idx[j];
        slots[i]->beginFrame();
        const Interpolator::Impl& im = *slots[i]->m;
        if (!im.W || !im.frameOk(prev[i]) || !im.frameOk(curr[i]) || !im.samePitch(prev[i], curr[i])) {
            err = "a slot's estimate was refused (frames?)";
            return false;
        }
    }
    std::vector<Interpolator::Impl::EstPlan> plans(ns);
    int maxTop = 0;
    for (int j = 0; j < ns; j++) {
        const int i = idx[j];
        Interpolator::Impl& im = *slots[i]->m;
        im.estSets++;
        im.haveEst = im.estUi = false;
        im.planEstimate(prev[i], curr[i], false, plans[j]);
        maxTop = std::max(maxTop, plans[j].top);
    }
    auto fail = [&](cudaError_t e) {
        if (e == cudaSuccess) return false;
        cudaGetLastError();
        err = cudaGetErrorString(e);
        return true;
    };
    std::vector<fgk::LumaPyrParams> luma;
    std::vector<int> fmts;
    for (int j = 0; j < ns; j++) {
        const int i = idx[j];
        luma.push_back(plans[j].luma);
        fmts.push_back((int)slots[i]->m->fmt);
    }
    if (fail(launchMergedGroups(luma, fmts, [&](fgk::Merged<fgk::LumaPyrParams>& mg, int f) {
            return f == (int)Format::Rgba8 ? fgk::launchLumaPyrMerged(mg, s) : fgk::launchLumaFmtMerged(mg, mg.item[0].f.format, s);
        })))
        return false;
    for (int j = 0; j < ns; j++)
        for (const fgk::DownParams& dp : plans[j].down)
            if (fail(fgk::launchDown(dp, s))) return false;
    for (int l = maxTop; l >= 0; l--) {
        std::vector<fgk::SearchParams> se;
        std::vector<fgk::Median3Params> me;
        std::vector<int> sk, mk;
        for (int j = 0; j < ns; j++)
            if (l <= plans[j].top) {
                se.push_back(plans[j].search[l]);
                sk.push_back(fgk::searchVariant(se.back()));
                me.push_back(plans[j].med[l]);
                mk.push_back(fgk::median3Variant(me.back()));
            }
        if (fail(launchMergedGroups(se, sk, [&](fgk::Merged<fgk::SearchParams>& mg, int) { return fgk::launchSearchMerged(mg, s); })) ||
            fail(launchMergedGroups(me, mk, [&](fgk::Merged<fgk::Median3Params>& mg, int) { return fgk::launchMedian3Merged(mg, s); })))
            return false;
    }
    std::vector<fgk::SubpixParams> sub;
    std::vector<fgk::PixfieldParams> pix;
    for (int j = 0; j < ns; j++) {
        const int i = idx[j];
        if (slots[i]->m->set.subpixel) sub.push_back(plans[j].sub);
        else if (fail(fgk::launchCutMean(plans[j].cut, s))) return false;
        pix.push_back(plans[j].pix);
    }
    if (fail(launchMergedGroups(sub, std::vector<int>(sub.size(), 0),
                                [&](fgk::Merged<fgk::SubpixParams>& mg, int) { return fgk::launchSubpixMerged(mg, s); })) ||
        fail(launchMergedGroups(pix, std::vector<int>(pix.size(), 0),
                                [&](fgk::Merged<fgk::PixfieldParams>& mg, int) { return fgk::launchPixfieldMerged(mg, s); })))
        return false;
    for (int j = 0; j < ns; j++) {
        const int i = idx[j];
        Interpolator::Impl& im = *slots[i]->m;
        im.haveEst = true;
        im.estPrev = prev[i].data;
        im.estCurr = curr[i].data;
    }
    return true;
}

bool Batch::record(cudaStream_t s, const Frame* prev, const Frame* curr, const Frame* outs) {
    m->err = nullptr;
    const int ns = (int)m->slots.size();
    if (!ns || !prev || !curr || !outs || !m->dev) { m->err = "empty batch or missing frames"; return false; }
    DeviceGuard g(m->device);
    std::vector<int> first(ns);   // each slot's first output frame in outs
    for (int i = 0, o = 0; i < ns; i++) { first[i] = o; o += (int)m->mult[i] - 1; }
    const bool batched = m->shape.ctasPerSm > 0;
    // 0. mergeEstimates = G: the slots' estimates as merged launches on s, in G groups (slots dealt by decreasing pair
    //    size); each group's syntheses are forked off as soon as its estimates are recorded, so they overlap the next
    //    group's estimates (merged only when no slot needs a per-slot estimate pass)
    const bool merged = m->shape.mergeEstimates && m->mergeable();
    std::vector<std::vector<int>> groups(merged ? std::min<int>((int)m->shape.mergeEstimates, ns) : 1);
    {
        std::vector<int> order(ns);
        std::iota(order.begin(), order.end(), 0);
        if (merged)
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                return (size_t)m->slots[a]->m->W * m->slots[a]->m->H > (size_t)m->slots[b]->m->W * m->slots[b]->m->H;
            });
        for (int j = 0; j < ns; j++) groups[j % groups.size()].push_back(order[j]);
    }
    // 1. every slot's estimate (merged, or per slot on its pool stream) and, for the slots outside the persistent launch,
    //    its syntheses, forked over the pool: slot i on stream i % streams, joined back into s before the persistent
    //    launch
    const int nst = (int)std::min<uint32_t>(m->shape.streams, (uint32_t)Impl::kMaxStreams);
    auto streamOf = [&](int i) { return nst > 1 ? m->pool[i % nst] : s; };
    for (const std::vector<int>& grp : groups) {
        if (merged && !m->mergedEstimates(s, prev, curr, grp)) return false;
        if (nst > 1) {
            if (cudaEventRecord(m->fork, s) != cudaSuccess) { m->err = cudaGetErrorString(cudaGetLastError()); return false; }
            for (int k = 0; k < nst; k++)
                if (cudaStreamWaitEvent(m->pool[k], m->fork, 0) != cudaSuccess) {
                    m->err = cudaGetErrorString(cudaGetLastError());
                    return false;
                }
        }
        for (int i : grp) {
            Interpolator& I = *m->slots[i];
            if (!merged) {
                I.beginFrame();
                if (!I.recordEstimate(streamOf(i), prev[i], curr[i])) { m->err = "a slot's estimate was refused (frames?)"; return false; }
            }
            if (batched && !I.m->uiOn()) continue;   // in the persistent launches
            for (uint32_t k = 1; k < m->mult[i]; k++)
                if (!I.recordSynth(streamOf(i), prev[i], curr[i], outs[first[i] + k - 1], (float)k / (float)m->mult[i])) {
                    m->err = "a slot's synthesis was refused (frames?)";
                    return false;
                }
        }
    }
    if (nst > 1)
        for (int k = 0; k < nst; k++)
            if (cudaEventRecord(m->join[k], m->pool[k]) != cudaSuccess || cudaStreamWaitEvent(s, m->join[k], 0) != cudaSuccess) {
                m->err = cudaGetErrorString(cudaGetLastError());
                return false;
            }
    // 2. the work lists of the syntheses: one persistent launch per frame format (its items contiguous in the blob,
    //    each format's tile starts counted from 0, its own work counter after the items' untrusted counters), then
    //    the fallbacks of each format in one launch
    struct Item { int slot, k, tiles, fmt; };
    std::vector<Item> items;
    for (int i = 0; i < ns && batched; i++) {
        const Interpolator::Impl* im = m->slots[i]->m;
        if (im->uiOn()) continue;   // CrosshairV2 slots synthesize through recordSynth (tap rejection, paste-back)
        const int tiles = fgk::synthTilesX((int)im->W) * fgk::synthTilesY((int)im->H);
        for (uint32_t k = 1; k < m->mult[i]; k++) items.push_back({i, (int)k, tiles, (int)im->fmt});
    }
    std::stable_sort(items.begin(), items.end(), [&](const Item& x, const Item& y) {
        return x.fmt != y.fmt ? x.fmt < y.fmt : (m->shape.order == 1 && x.tiles > y.tiles);
    });
    const int n = (int)items.size();
    if (!n) return true;
    char* blob = m->host + (size_t)m->ring * m->blobBytes;
    m->ring = (m->ring + 1) % Impl::kRing;
    fgk::SynthParams* sp = (fgk::SynthParams*)blob;
    fgk::FallbackParams* fp = (fgk::FallbackParams*)(blob + m->oFall);
    int* start = (int*)(blob + m->oStart);
    int* tx = (int*)(blob + m->oTx);
    struct Segment { int first, count, total, fmt; size_t smem; };
    std::vector<Segment> segs;
    for (int j = 0; j < n; j++) {
        const Item& it = items[j];
        const Interpolator::Impl* im = m->slots[it.slot]->m;
        const Frame& out = outs[first[it.slot] + it.k - 1];
        if (!im->frameOk(out)) { m->err = "an output frame does not fit its slot"; return false; }
        if (segs.empty() || segs.back().fmt != it.fmt) segs.push_back({j, 0, 0, it.fmt, 0});
        Segment& g = segs.back();
        const float t = (float)it.k / (float)m->mult[it.slot];
        sp[j] = im->synthParams(prev[it.slot], curr[it.slot], out, t, m->counters + j);
        sp[j].emap = nullptr;
        fp[j] = im->fallbackParams(sp[j], nullptr);
        start[j] = g.total;
        tx[j] = fgk::synthTilesX((int)im->W);
        g.total += it.tiles;
        g.count++;
        g.smem = std::max(g.smem, it.fmt == (int)Format::Rgba8 ? fgk::synthKernelSmem((int)im->set.flowScale)
                                                               : fgk::synthFmtKernelSmem(sp[j].f.format, (int)im->set.flowScale));
    }
    if (cudaMemcpyAsync(m->dev, blob, m->blobBytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(m->counters, 0, (size_t)(n + Impl::kFormats) * 4, s) != cudaSuccess) {
        m->err = cudaGetErrorString(cudaGetLastError());
        return false;
    }
    const fgk::SynthParams* dItems = (const fgk::SynthParams*)m->dev;
    const fgk::FallbackParams* dFall = (const fgk::FallbackParams*)(m->dev + m->oFall);
    for (size_t g = 0; g < segs.size(); g++) {
        const Segment& sg = segs[g];
        fgk::SynthBatchArgs a{};
        a.items = dItems + sg.first;
        a.tileStart = (const int*)(m->dev + m->oStart) + sg.first;
        a.tilesX = (const int*)(m->dev + m->oTx) + sg.first;
        a.nItems = sg.count;
        a.total = sg.total;
        a.counter = m->counters + n + g;
        const bool rgba = sg.fmt == (int)Format::Rgba8;
        const int fmtK = rgba ? 0 : sp[sg.first].f.format;
        const int occ = rgba ? fgk::synthBatchCtasPerSm(sg.smem) : fgk::synthFmtBatchCtasPerSm(fmtK, sg.smem);
        const int grid = std::min(m->sms * std::max(1, std::min((int)m->shape.ctasPerSm, occ)), sg.total);
        const cudaError_t e = rgba ? fgk::launchSynthBatch(a, grid, sg.smem, s) : fgk::launchSynthFmtBatch(a, fmtK, grid, sg.smem, s);
        if (e != cudaSuccess) { cudaGetLastError(); m->err = cudaGetErrorString(e); return false; }
    }
    for (const Segment& sg : segs) {
        const cudaError_t e = sg.fmt == (int)Format::Rgba8 ? fgk::launchFallbackBatch(dFall + sg.first, sg.count, s)
                                                           : fgk::launchFallbackFmtBatch(dFall + sg.first, sg.count, s);
        if (e != cudaSuccess) { cudaGetLastError(); m->err = cudaGetErrorString(e); return false; }
    }
    return true;
}

int Batch::tune(cudaStream_t s, const Frame* prev, const Frame* curr, const Frame* outs, uint32_t reps) {
    static const Shape cand[] = {{0, 0, 1, 0}, {3, 1, 1, 0}, {0, 0, 4, 0}, {3, 1, 4, 0}, {0, 0, 8, 0}, {2, 1, 8, 0},
                                 {3, 0, 8, 0}, {3, 1, 8, 0}, {0, 0, 1, 1}, {3, 1, 1, 1}, {0, 0, 8, 1}, {3, 1, 8, 1},
                                 {0, 0, 8, 4}, {3, 1, 8, 4}, {0, 0, 8, 8}, {3, 1, 8, 8}};
    DeviceGuard g(m->device);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) { cudaGetLastError(); return -1; }
    int best = -1;
    float bestMs = 0.0f;
    for (int c = 0; c < (int)(sizeof(cand) / sizeof(cand[0])); c++) {
        m->shape = cand[c];
        bool ok = record(s, prev, curr, outs) && cudaStreamSynchronize(s) == cudaSuccess;   // warm
        ok = ok && cudaEventRecord(e0, s) == cudaSuccess;
        for (uint32_t r = 0; ok && r < std::max(reps, 1u); r++) {
            ok = record(s, prev, curr, outs);
            if ((r + 1) % (Impl::kRing / 2) == 0) ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
        }
        float ms = 0.0f;
        ok = ok && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
             cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
        if (!ok) { cudaGetLastError(); continue; }
        if (best < 0 || ms < bestMs) { best = c; bestMs = ms; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best >= 0) m->shape = cand[best];
    return best;
}

}  // namespace framegen

// ================================================================================================== C ABI
using namespace framegen;

struct fg_interpolator {
    Interpolator I;
};
struct fg_batch {
    Batch B;
};

static Settings fromC(const fg_settings* c) {
    Settings s;
    if (!c) return s;
    s.trustLow = c->trustLow; s.trustHigh = c->trustHigh; s.globalFallback = c->globalFallback;
    s.sceneCutSad = c->sceneCutSad; s.hudBonus = c->hudBonus; s.smoothBonus = c->smoothBonus;
    s.searchPenalty = c->searchPenalty; s.searchRadius = c->searchRadius; s.searchRadiusTop = c->searchRadiusTop;
    s.subpixel = c->subpixel != 0; s.uiProtection = (UiProtection)c->uiProtection; s.blurSamples = c->blurSamples;
    s.blurWeights = (BlurWeights)c->blurWeights; s.motionVersion = (MotionVersion)c->motionVersion;
    s.flowScale = c->flowScale; s.pyramidMinSide = c->pyramidMinSide;
    if (c->size >= offsetof(fg_settings, uiEstimateFill) + sizeof(c->uiEstimateFill)) {   // the UI fields
        s.uiHistory = c->uiHistory; s.uiBoxHeightFrac = c->uiBoxHeightFrac; s.uiBoxWidth = c->uiBoxWidth;
        s.uiBoxHeight = c->uiBoxHeight; s.uiCrosshairArea = c->uiCrosshairArea; s.uiBoxOffsetX = c->uiBoxOffsetX;
        s.uiBoxOffsetY = c->uiBoxOffsetY; s.uiStillFrames = c->uiStillFrames; s.uiStillThreshold = c->uiStillThreshold;
        s.uiInpaintReach = c->uiInpaintReach; s.uiMaxStillFraction = c->uiMaxStillFraction;
        s.uiContrastThreshold = c->uiContrastThreshold; s.uiLeaveFrames = c->uiLeaveFrames;
        s.uiReentryFrames = c->uiReentryFrames; s.uiEstimateFill = c->uiEstimateFill != 0;
    }
    return s;
}
static void toC(const Settings& s, fg_settings* c) {
    c->size = sizeof(fg_settings);
    c->trustLow = s.trustLow; c->trustHigh = s.trustHigh; c->globalFallback = s.globalFallback;
    c->sceneCutSad = s.sceneCutSad; c->hudBonus = s.hudBonus; c->smoothBonus = s.smoothBonus;
    c->searchPenalty = s.searchPenalty; c->searchRadius = s.searchRadius; c->searchRadiusTop = s.searchRadiusTop;
    c->subpixel = s.subpixel; c->uiProtection = (uint32_t)s.uiProtection; c->blurSamples = s.blurSamples;
    c->blurWeights = (uint32_t)s.blurWeights; c->motionVersion = (uint32_t)s.motionVersion;
    c->flowScale = s.flowScale; c->pyramidMinSide = s.pyramidMinSide;
    c->uiHistory = s.uiHistory; c->uiBoxHeightFrac = s.uiBoxHeightFrac; c->uiBoxWidth = s.uiBoxWidth;
    c->uiBoxHeight = s.uiBoxHeight; c->uiCrosshairArea = s.uiCrosshairArea; c->uiBoxOffsetX = s.uiBoxOffsetX;
    c->uiBoxOffsetY = s.uiBoxOffsetY; c->uiStillFrames = s.uiStillFrames; c->uiStillThreshold = s.uiStillThreshold;
    c->uiInpaintReach = s.uiInpaintReach; c->uiMaxStillFraction = s.uiMaxStillFraction;
    c->uiContrastThreshold = s.uiContrastThreshold; c->uiLeaveFrames = s.uiLeaveFrames;
    c->uiReentryFrames = s.uiReentryFrames; c->uiEstimateFill = s.uiEstimateFill;
}
static Frame fromC(const fg_frame* f) {
    return f ? Frame(f->data, (size_t)f->pitch, f->chroma, (size_t)f->chroma_pitch) : Frame();
}

extern "C" {

uint32_t fg_abi_version(void) { return 1; }
void fg_default_settings(fg_settings* s) {
    if (s) toC(Settings{}, s);
}
void fg_default_init_info(fg_init_info* ii) {
    if (!ii) return;
    InitInfo d;
    std::memset(ii, 0, sizeof(*ii));
    ii->size = sizeof(fg_init_info);
    ii->view_format = d.viewFormat;
    ii->transfer = (uint32_t)d.transfer;
    ii->linear_white_nits = d.linearWhiteNits;
    ii->yuv_matrix = (uint32_t)d.yuvMatrix;
    ii->yuv_full_range = d.yuvFullRange;
    ii->device = d.device;
    toC(d.settings, &ii->settings);
}
int fg_format_of(uint32_t vf, uint32_t* out) {
    Format f;
    if (!formatOf(vf, &f)) return 0;
    if (out) *out = (uint32_t)f;
    return 1;
}
fg_interpolator* fg_create(void) { return new fg_interpolator(); }
void fg_destroy(fg_interpolator* fg) { delete fg; }
int fg_init(fg_interpolator* fg, const fg_init_info* c) {
    if (!fg || !c) return 0;
    InitInfo ii;
    ii.width = c->width; ii.height = c->height; ii.viewFormat = c->view_format; ii.transfer = (Transfer)c->transfer;
    ii.linearWhiteNits = c->linear_white_nits; ii.yuvMatrix = (YuvMatrix)c->yuv_matrix;
    ii.yuvFullRange = c->yuv_full_range != 0; ii.device = c->device; ii.settings = fromC(&c->settings);
    return fg->I.init(ii);
}
const char* fg_init_error(const fg_interpolator* fg) { return fg ? fg->I.initError() : "null interpolator"; }
uint32_t fg_format(const fg_interpolator* fg) { return fg ? (uint32_t)fg->I.format() : 0; }
int fg_resize(fg_interpolator* fg, uint32_t w, uint32_t h, uint32_t vf) { return fg && fg->I.resize(w, h, vf); }
int fg_validate(const fg_settings* s) { return s && Interpolator::validate(fromC(s)); }
const char* fg_settings_error_format(const fg_settings* s, uint32_t f) {
    return Interpolator::settingsError(fromC(s), (Format)f);
}
const char* fg_settings_error(const fg_interpolator* fg, const fg_settings* s) {
    return fg ? fg->I.settingsError(fromC(s)) : Interpolator::settingsError(fromC(s), Format::Rgba8);
}
const char* fg_size_error(const fg_interpolator* fg, uint32_t w, uint32_t h) {
    return fg ? fg->I.sizeError(w, h) : "not initialised";
}
int fg_set_settings(fg_interpolator* fg, const fg_settings* s) { return fg && s && fg->I.setSettings(fromC(s)); }
int fg_reconfigure(fg_interpolator* fg, const fg_settings* s) { return fg && s && fg->I.reconfigure(fromC(s)); }
void fg_get_settings(const fg_interpolator* fg, fg_settings* s) {
    if (s) toC(fg ? fg->I.settings() : Settings{}, s);
}
void fg_begin_frame(fg_interpolator* fg) {
    if (fg) fg->I.beginFrame();
}
void fg_release_unused_ui(fg_interpolator* fg) {
    if (fg) fg->I.releaseUnusedUi();
}
void fg_release_unused_motion(fg_interpolator* fg) {
    if (fg) fg->I.releaseUnusedMotion();
}
int fg_record_estimate(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr) {
    return fg && prev && curr && fg->I.recordEstimate((cudaStream_t)stream, fromC(prev), fromC(curr));
}
uint64_t fg_ui_trace_bytes(const fg_interpolator* fg) { return fg ? (uint64_t)fg->I.uiTraceBytes() : 0; }
int fg_ui_trace(fg_interpolator* fg, void* stream, const void* frame, void* dst) {
    return fg && fg->I.uiTrace((cudaStream_t)stream, frame, dst);
}
int fg_record_observe(fg_interpolator* fg, void* stream, const fg_frame* f) {
    return fg && f && fg->I.recordObserve((cudaStream_t)stream, fromC(f));
}
int fg_record_track(fg_interpolator* fg, void* stream, const fg_frame* f) {
    return fg && f && fg->I.recordTrack((cudaStream_t)stream, fromC(f));
}
void fg_box_size(const fg_settings* s, uint32_t w, uint32_t h, uint32_t* bw, uint32_t* bh) {
    uint32_t a = 0, b = 0;
    Interpolator::boxSize(fromC(s), w, h, &a, &b);
    if (bw) *bw = a;
    if (bh) *bh = b;
}
void fg_box_rect(const fg_settings* s, uint32_t w, uint32_t h, int32_t rect[4]) {
    if (rect) Interpolator::boxRect(fromC(s), w, h, rect);
}
uint32_t fg_box_margin(const fg_settings* s) { return Interpolator::boxMargin(fromC(s)); }
void fg_work_rect(const fg_settings* s, uint32_t w, uint32_t h, int32_t rect[4]) {
    if (rect) Interpolator::workRect(fromC(s), w, h, rect);
}
int fg_record_synth(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* out,
                    float t) {
    return fg && prev && curr && out && fg->I.recordSynth((cudaStream_t)stream, fromC(prev), fromC(curr), fromC(out), t);
}
int fg_record_synth_blur(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr,
                         const fg_frame* out, float t0, float t1) {
    return fg && prev && curr && out &&
           fg->I.recordSynthBlur((cudaStream_t)stream, fromC(prev), fromC(curr), fromC(out), t0, t1);
}
uint32_t fg_blur_plan(uint32_t samples, uint32_t weights, float t0, float t1, float* times, uint32_t* q) {
    if (weights > 1u) return 0;
    return Interpolator::blurPlan(samples, (BlurWeights)weights, t0, t1, times, q);
}
int fg_record(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* out, float t) {
    return fg && prev && curr && out && fg->I.record((cudaStream_t)stream, fromC(prev), fromC(curr), fromC(out), t);
}
int fg_set_profiling(fg_interpolator* fg, int on) { return fg && fg->I.setProfiling(on != 0); }
int fg_read_costs(fg_interpolator* fg, fg_costs* c) {
    if (!fg || !c) return 0;
    Interpolator::CostTimings t;
    const bool ok = fg->I.readCosts(t);
    c->estimate_ms = t.estimateMs; c->synth_ms = t.synthMs; c->seq = t.seq; c->synths = t.synths;
    return ok;
}
int fg_read_timings(fg_interpolator* fg, const char** names, uint64_t* ns, uint32_t capacity, uint32_t* count) {
    if (!fg) return 0;
    std::vector<const char*> n;
    std::vector<uint64_t> t;
    if (!fg->I.readTimings(n, t)) return 0;
    for (uint32_t i = 0; i < capacity && i < n.size(); i++) {
        if (names) names[i] = n[i];
        if (ns) ns[i] = t[i];
    }
    if (count) *count = (uint32_t)n.size();
    return 1;
}
int fg_record_debug_counters(fg_interpolator* fg, void* stream, void* dst) {
    return fg && fg->I.recordDebugCounters((cudaStream_t)stream, dst);
}
uint32_t fg_debug_sad_blocks(const fg_interpolator* fg) { return fg ? fg->I.debugSadBlocks() : 0; }
int fg_get_debug_map_layout(const fg_interpolator* fg, fg_debug_map_layout* l) {
    Interpolator::DebugMapLayout d;
    if (!fg || !l || !fg->I.debugMapLayout(d)) return 0;
    l->W = d.W; l->H = d.H; l->fw = d.fw; l->fh = d.fh; l->bw = d.bw; l->bh = d.bh; l->fscale = d.fscale;
    l->eStride = d.eStride; l->blockOff = d.blockOff; l->pixOff = d.pixOff; l->eOff = d.eOff; l->size = d.size;
    return 1;
}
int fg_record_debug_maps(fg_interpolator* fg, void* stream, void* dst) {
    return fg && fg->I.recordDebugMaps((cudaStream_t)stream, dst);
}
int fg_set_debug_capture(fg_interpolator* fg, int on) { return fg && fg->I.setDebugCapture(on != 0); }
int fg_get_trace_layout(const fg_interpolator* fg, fg_trace_layout* l) {
    Interpolator::TraceLayout t;
    if (!fg || !l || !fg->I.traceLayout(t)) return 0;
    static_assert(sizeof(fg_trace_layout) == sizeof(Interpolator::TraceLayout), "trace layout mirrors");
    std::memcpy(l, &t, sizeof(t));
    return 1;
}
int fg_record_trace(fg_interpolator* fg, void* stream, void* dst) { return fg && fg->I.recordTrace((cudaStream_t)stream, dst); }
int fg_set_seed_net(fg_interpolator* fg, const float* host_params, uint32_t level) {
    return fg && fg->I.setSeedNet(host_params, level);
}
uint32_t fg_seed_net_level(const fg_interpolator* fg) { return fg ? fg->I.seedNetLevel() : UINT32_MAX; }

static InitInfo fromC(const fg_init_info* c) {
    InitInfo ii;
    ii.width = c->width; ii.height = c->height; ii.viewFormat = c->view_format; ii.transfer = (Transfer)c->transfer;
    ii.linearWhiteNits = c->linear_white_nits; ii.yuvMatrix = (YuvMatrix)c->yuv_matrix;
    ii.yuvFullRange = c->yuv_full_range != 0; ii.device = c->device; ii.settings = fromC(&c->settings);
    return ii;
}
fg_batch* fg_batch_create(void) { return new fg_batch(); }
void fg_batch_destroy(fg_batch* b) { delete b; }
int fg_batch_add(fg_batch* b, const fg_init_info* ii, uint32_t multiplier) {
    return b && ii ? b->B.add(fromC(ii), multiplier) : -1;
}
const char* fg_batch_error(const fg_batch* b) { return b ? b->B.error() : "null batch"; }
uint32_t fg_batch_slots(const fg_batch* b) { return b ? b->B.slots() : 0; }
static std::vector<Frame> framesOf(const fg_frame* f, size_t n) {
    std::vector<Frame> v(n);
    for (size_t i = 0; i < n; i++) v[i] = fromC(f + i);
    return v;
}
static size_t batchOuts(fg_batch* b) {
    size_t n = 0;
    for (uint32_t i = 0; i < b->B.slots(); i++) n += b->B.synthsOf(i);
    return n;
}
int fg_batch_record(fg_batch* b, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* outs) {
    if (!b || !prev || !curr || !outs) return 0;
    const size_t ns = b->B.slots();
    const std::vector<Frame> p = framesOf(prev, ns), c = framesOf(curr, ns), o = framesOf(outs, batchOuts(b));
    return b->B.record((cudaStream_t)stream, p.data(), c.data(), o.data());
}
int fg_batch_tune(fg_batch* b, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* outs,
                  uint32_t reps) {
    if (!b || !prev || !curr || !outs) return -1;
    const size_t ns = b->B.slots();
    const std::vector<Frame> p = framesOf(prev, ns), c = framesOf(curr, ns), o = framesOf(outs, batchOuts(b));
    return b->B.tune((cudaStream_t)stream, p.data(), c.data(), o.data(), reps);
}
void fg_batch_get_shape(const fg_batch* b, uint32_t* ctas_per_sm, uint32_t* order, uint32_t* streams) {
    if (!b) return;
    const Batch::Shape s = b->B.shape();
    if (ctas_per_sm) *ctas_per_sm = s.ctasPerSm;
    if (order) *order = s.order;
    if (streams) *streams = s.streams;
}
uint32_t fg_batch_merge_estimates(const fg_batch* b) { return b ? b->B.shape().mergeEstimates : 0u; }
int fg_batch_set_shape(fg_batch* b, uint32_t ctas_per_sm, uint32_t order, uint32_t streams) {
    return fg_batch_set_shape_merged(b, ctas_per_sm, order, streams, 0);
}
int fg_batch_set_shape_merged(fg_batch* b, uint32_t ctas_per_sm, uint32_t order, uint32_t streams, uint32_t merge_estimates) {
    Batch::Shape s;
    s.ctasPerSm = ctas_per_sm;
    s.order = order;
    s.streams = streams;
    s.mergeEstimates = merge_estimates;
    return b && b->B.setShape(s);
}
int fg_batch_trace(fg_batch* b, uint32_t slot, void* stream, void* dst) {
    Interpolator* I = b ? b->B.slot(slot) : nullptr;
    return I && I->recordTrace((cudaStream_t)stream, dst);
}
int fg_batch_trace_layout(fg_batch* b, uint32_t slot, fg_trace_layout* l) {
    Interpolator* I = b ? b->B.slot(slot) : nullptr;
    return I && l && I->traceLayout(*reinterpret_cast<Interpolator::TraceLayout*>(l));
}
const char* fg_last_error(const fg_interpolator* fg) { return fg ? fg->I.lastCudaError() : nullptr; }

}  // extern "C"
