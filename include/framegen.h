// framegen (B200 build): image-only frame interpolation, MotionVersion::V1, on CUDA (sm_100a).
//
// Drop-in for the V1 path of frame-gen-ritz's gpu/framegen.h: the same namespace, class, enums, Settings fields,
// defaults, ranges, bool-returning conventions and error strings, with these replacements:
//   VkCommandBuffer          -> cudaStream_t (records are kernel launches on the caller's stream; nothing is
//                               synchronised with the host, nothing is allocated while recording, so a caller may
//                               capture records into a CUDA graph)
//   Frame{VkImageView, ...}  -> Frame{device pointer, row pitch in bytes} (+ the CbCr plane for the two-plane formats)
//   InitInfo Vulkan members  -> dropped; InitInfo::device selects the CUDA device (-1: the current one)
//   VkBuffer debug targets   -> device pointers
//   VkFormat viewFormat      -> the same VkFormat numbers as plain uint32_t (kVkFormat* below; no Vulkan headers)
// Out of scope here (rejected with a reason by settingsError / initError): MotionVersion V2 / Learned / V3, static-UI
// protection modes other than Off.
//
// Threading / streams: not thread-safe. All records of one Interpolator must go to ONE stream, in recording order:
// its internal buffers are shared between records and only ordered by stream order.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

typedef struct CUstream_st* cudaStream_t;

namespace framegen {

// gpu/framegen.h:15-24
enum class UiProtection : uint32_t { Off = 0, Crosshair = 1, WholeScreen = 2, CrosshairV2 = 3 };
// gpu/framegen.h:28-59 (V1 is the only version this library runs)
enum class MotionVersion : uint32_t { V1 = 0, V2 = 1, Learned = 2, V3 = 3 };
// gpu/framegen.h:63-92 (the Learned version's nets: accepted, unused here)
enum class LearnedNet : uint32_t { E2v3 = 0, E1v3 = 1, E2v4 = 2, E1v4 = 3, E2v5 = 4, E1v5 = 5, G2v2 = 6, G2v3 = 7, M2v2 = 8, M2v3 = 9 };
constexpr uint32_t kLearnedNets = 10;
// gpu/framegen.h:99-108, 115-121 (V2 / V3 options: accepted, unused here)
enum class V2Mode : uint32_t { Quality = 0, Performance = 1 };
enum class V3Guard : uint32_t { Off = 0, Guard = 1, V2Motion = 2 };
// gpu/framegen.h:125-129
enum class BlurWeights : uint32_t { Even = 0, Gaussian = 1 };
// gpu/framegen.h:138
enum class Format : uint32_t { Rgba8 = 0, Rgb10 = 1, RgbaF16 = 2, Nv12 = 3, P010 = 4 };
// The VkFormat values a viewFormat may take (their numbers in the Vulkan registry).
enum : uint32_t {
    kVkFormatR8Unorm = 9,
    kVkFormatR8G8B8A8Unorm = 37,
    kVkFormatB8G8R8A8Unorm = 44,
    kVkFormatA2R10G10B10UnormPack32 = 58,
    kVkFormatA2B10G10R10UnormPack32 = 64,
    kVkFormatR16Unorm = 70,
    kVkFormatR16G16B16A16Sfloat = 97,
};
// gpu/framegen.h:140: the format class of a view format, false if the library does not know it.
bool formatOf(uint32_t viewFormat, Format* out);
// gpu/framegen.h:144-147
enum class Transfer : uint32_t { Encoded = 0, Linear = 1 };
// gpu/framegen.h:150
enum class YuvMatrix : uint32_t { Bt601 = 0, Bt709 = 1, Bt2020 = 2 };

// gpu/framegen.h:154-159: one image as the library takes it. Device memory; rows `pitch` bytes apart (a multiple of
// 4 for the 4-byte formats); pixels packed as the viewFormat says. The two-plane formats add the CbCr plane. A frame
// whose first plane spans more than 2^34 bytes ((height - 1) * pitch + the row's bytes) is refused: the 8-bit kernels
// address it in 32-bit words.
struct Frame {
    void* data = nullptr;
    size_t pitch = 0;
    void* chroma = nullptr;
    size_t chromaPitch = 0;
    Frame() = default;
    Frame(void* d, size_t p, void* c = nullptr, size_t cp = 0) : data(d), pitch(p), chroma(c), chromaPitch(cp) {}
};

// gpu/framegen.h:167-409, the fields the V1 path reads (same names, types, defaults, ranges).
struct Settings {
    // runtime: setSettings() at any time
    float trustLow = 12.0f;         // [0, 255], trustHigh >= trustLow + 1
    float trustHigh = 40.0f;
    float globalFallback = 0.15f;   // (0, 1]
    float sceneCutSad = 30.0f;      // (0, 255]
    float hudBonus = 1.0f;          // [0, 255]
    float smoothBonus = 0.5f;       // [0, 255]
    float searchPenalty = 0.5f;     // [0, 255]
    uint32_t searchRadius = 2;      // [1, 12]
    uint32_t searchRadiusTop = 6;   // [1, 12]
    bool subpixel = true;
    // Static-UI protection (gpu/framegen.h:196-305): Off, or CrosshairV2 for the 8-bit RGBA / BGRA, Rgb10 and RgbaF16
    // formats (the box fields, uiHistory, uiStillFrames, uiStillThreshold, uiContrastThreshold, uiLeaveFrames,
    // uiReentryFrames and uiEstimateFill apply). Crosshair, WholeScreen and the YUV formats are refused by settingsError with a reason;
    // uiInpaintReach and uiMaxStillFraction (Crosshair / WholeScreen fields) are validated with the reference's ranges.
    UiProtection uiProtection = UiProtection::Off;
    uint32_t uiHistory = 3;                          // [3, 65]
    float uiBoxHeightFrac = 0.025f;                  // [0, 1]
    uint32_t uiBoxWidth = 0, uiBoxHeight = 0;        // [0, 16384]
    float uiCrosshairArea = 0.03f;                   // (0, 1]
    int32_t uiBoxOffsetX = 0, uiBoxOffsetY = 0;      // [-16384, 16384]
    uint32_t uiStillFrames = 8;                      // [1, 255]
    float uiStillThreshold = 3.5f;                   // [0, 255]
    uint32_t uiInpaintReach = 12;                    // [1, 16]
    float uiMaxStillFraction = 0.75f;                // (0, 1]
    float uiContrastThreshold = 20.0f;               // [0, 255]
    uint32_t uiLeaveFrames = 4;                      // [1, 255]
    uint32_t uiReentryFrames = 2;                    // [0, 255]
    bool uiEstimateFill = false;
    uint32_t blurSamples = 0;                        // [0, 16]: recordSynthBlur's sub-frames (< 2: blur off)
    BlurWeights blurWeights = BlurWeights::Gaussian;
    MotionVersion motionVersion = MotionVersion::V1; // V1 only
    // the other versions' fields (gpu/framegen.h:310-380): validated with the reference's ranges, unused here
    V2Mode v2Mode = V2Mode::Quality;
    bool v2StaticMask = true;
    float v3Smear = 0.35f;                           // [0, 1]
    float v3OcclSoft = 1.0f;                         // [0.25, 4]
    float v3Unsure = 1.0f;                           // [0.25, 4]
    float v3SceneCut = 0.0f;                         // [0, 4]
    bool v3ColourWindow = false;
    bool v3DetailSplit = false;
    V3Guard v3Guard = V3Guard::Off;
    LearnedNet learnedNet = LearnedNet::E2v5;
    bool learnedHalf = false;
    bool learnedZeroTest = true;
    bool learnedStaticGuard = false;
    // structural: init() or reconfigure()
    uint32_t flowScale = 2;         // 1, 2, 4
    uint32_t pyramidMinSide = 48;   // [16, 256]
};

// gpu/framegen.h:411-441 without the Vulkan members.
struct InitInfo {
    uint32_t width = 0, height = 0;                  // >= kMinSize each
    uint32_t viewFormat = kVkFormatB8G8R8A8Unorm;
    Transfer transfer = Transfer::Encoded;           // RgbaF16 only
    float linearWhiteNits = 80.0f;                   // Transfer::Linear: (0, 10000]
    YuvMatrix yuvMatrix = YuvMatrix::Bt709;          // Nv12 / P010 only
    bool yuvFullRange = false;
    Settings settings{};
    int device = -1;                                 // CUDA device ordinal, -1 = the current device at init()
};

class Interpolator {
public:
    Interpolator() = default;
    ~Interpolator();
    Interpolator(const Interpolator&) = delete;
    Interpolator& operator=(const Interpolator&) = delete;

    // gpu/framegen.h:451-461. init/resize/destroy free memory earlier records use: the caller must have retired
    // them (stream or device synchronize) first.
    bool init(const InitInfo&);
    const char* initError() const { return err_; }
    Format format() const;
    void destroy();
    bool resize(uint32_t w, uint32_t h, uint32_t viewFormat);

    // gpu/framegen.h:464-480
    static bool validate(const Settings&);
    static const char* settingsError(const Settings&, Format format);
    const char* settingsError(const Settings&) const;
    const char* sizeError(uint32_t width, uint32_t height) const;
    // gpu/framegen.h:500-507
    bool setSettings(const Settings&);
    bool reconfigure(const Settings&);
    Settings settings() const;

    // gpu/framegen.h:511: resets the per-submission record counts (kSetRing each)
    void beginFrame();
    // gpu/framegen.h:693: frees the kept-frame masks Settings::uiHistory no longer keeps (they stay allocated when it is
    // lowered; everything when protection is off). Every earlier record must have retired. gpu/framegen.h:700: V1 is
    // the only motion version here, so releaseUnusedMotion has nothing to free (kept so a host that calls it links).
    void releaseUnusedUi();
    void releaseUnusedMotion();

    // Static-UI protection, CrosshairV2 (gpu/framegen.h:576-691). recordObserve(stream, frame): once per new real
    // frame, in presentation order, after its pixels are final and before the recordEstimate that uses it: advances
    // the per-pixel state of the box (still / contrasty / in the mask, with hysteresis and fast re-entry) and keeps
    // the frame's mask (the frame's device pointer is the key; LRU by observe order, Settings::uiHistory frames kept).
    // recordTrack: the same state update for a frame passed through without generating, no mask kept (and an entry
    // of the same frame forgotten). A host that never calls recordObserve gets the implicit observe in recordEstimate
    // (prev if not kept, curr if it is not the most recently observed frame). A synthesis of a pair whose frames are
    // both kept rejects warp taps that land on a frame's own UI pixels and pastes curr's UI pixels that did not change
    // in the pair; a pair without both entries is interpolated unprotected. recordSynth returns false if an entry the
    // estimate used was evicted or replaced since. Protection Off: both return true and record nothing. false: not
    // initialised, a bad frame, or the first-use allocation failed.
    bool recordObserve(cudaStream_t stream, Frame frame);
    bool recordTrack(cudaStream_t stream, Frame frame);
    // gpu/framegen.h:484-494: the box size, the box rectangle {x, y, w, h} (centred plus the offsets, clamped into the
    // frame), the margin past it the mode protects (1 for CrosshairV2, 2 Crosshair, 0 otherwise) and the work
    // rectangle (the box grown by the margin, clamped to the frame). They do not check validity.
    static void boxSize(const Settings&, uint32_t w, uint32_t h, uint32_t* boxW, uint32_t* boxH);
    static void boxRect(const Settings&, uint32_t w, uint32_t h, int32_t rect[4]);
    static uint32_t boxMargin(const Settings&);
    static void workRect(const Settings&, uint32_t w, uint32_t h, int32_t rect[4]);
    // B200-build extension (no reference counterpart; for parity tests): the size of uiTrace's output, and a copy
    // (on `stream`) of the protection's per-pixel state (4 words per work-rectangle pixel) followed by the kept mask
    // of `frame` (header + bytes; zeros if that frame is not kept). false if the protection is off or unallocated.
    size_t uiTraceBytes() const;
    bool uiTrace(cudaStream_t stream, const void* frame, void* dst);

    // gpu/framegen.h:549-551: passes 1-8 once per real pair, passes 9-11 per generated time t in (0, 1), or both.
    // false (and nothing recorded, out untouched) if not initialised, t outside (0, 1), a ring overflow since
    // beginFrame(), a synth without an estimate since init/resize/reconfigure, or prev/curr not the estimate's frames.
    bool recordEstimate(cudaStream_t stream, Frame prev, Frame curr);
    bool recordSynth(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t);
    bool record(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t = 0.5f);

    // gpu/framegen.h:553-573: out = the weighted average of Settings::blurSamples (N) sub-frames of the latest
    // estimate's pair at t_k = t0 + (t1 - t0)(k + 0.5) / N (double arithmetic, rounded to float, clamped to [t0, t1]),
    // weights Settings::blurWeights (Gaussian: exp(-2 x_k^2), x_k = (2k + 1 - N) / N). A sub-frame is exactly the 8-bit
    // frame recordSynth(t_k) gives (its scene-cut and whole-frame fallbacks included; prev / curr at t_k <= 0 / >= 1);
    // the average is rounded once: out = (sum q_k v_k + 2^15) >> 16 per byte, q_k = the normalised weights in units
    // of 2^-16 (largest-remainder rounding, blurPlan). N < 2 or t0 == t1: the single instant t1 (recordSynth(t1); a copy
    // of prev / curr at t1 = 0 / 1). false (nothing recorded) unless 0 <= t0 <= t1 <= 1, and in recordSynth's cases.
    // Other formats: the stored values are averaged the same way (Rgb10 / Nv12 / P010 codes, exact integer sums);
    // RgbaF16 sums fl32(q_k 2^-16 h_k) in sample order in float32 and rounds to half once. Takes one synth of the ring.
    // 8-bit RGBA with blur on keeps one stored sub-frame per sample (allocated by init / setSettings / reconfigure
    // while they fit 1 GiB): each synthesized sample is one synthesis launch into its sub-frame, then one blend launch
    // (profile groups "blur samples", "blur blend"). Otherwise (other formats, or past the cap) two launches whatever
    // N is, the samples accumulated in registers ("blur resolve", "blur fixup"). The bytes are the same either way.
    bool recordSynthBlur(cudaStream_t stream, Frame prev, Frame curr, Frame out, float t0, float t1);
    // the samples of a blur: their times and weights (units of 2^-16, summing to 2^16); returns their count (0 if
    // refused: t0, t1 out of order or range)
    static uint32_t blurPlan(uint32_t samples, BlurWeights weights, float t0, float t1, float* times, uint32_t* q);

    // gpu/framegen.h:705-717: CUDA events after every pass group; readTimings waits for them and returns the
    // group names and the nanoseconds of each group (the reference returns timestamp ticks; here 1 tick = 1 ns).
    bool setProfiling(bool on);
    bool readTimings(std::vector<const char*>& names, std::vector<uint64_t>& ticks);
    // B200-build extension: the cost-guard inputs of gpu/pacing.h:869-871 (Pacer::Inputs::estimateMs / synthMs /
    // costSeq) from the last profile: estimateMs = the estimate's pass groups (luma .. pixel field), synthMs = the
    // synth-side groups (synth, fallback; blur samples, blur blend or blur resolve, blur fixup) per recorded synthesis;
    // -1 where the profile has none; seq changes with every new profile read. false if profiling is off or nothing was
    // recorded.
    struct CostTimings {
        float estimateMs = -1.0f, synthMs = -1.0f;
        uint32_t seq = 0, synths = 0;
    };
    bool readCosts(CostTimings& c);

    // gpu/framegen.h:726-741: debug copies into device memory at dst (stream-ordered).
    bool recordDebugCounters(cudaStream_t stream, void* dst);   // 2 uint32: [untrusted px, finest SAD sum x 256]
    uint32_t debugSadBlocks() const;
    struct DebugMapLayout {
        uint32_t W, H, fw, fh, bw, bh, fscale, eStride;   // eStride in uint32 words
        uint64_t blockOff, pixOff, eOff, size;            // byte offsets in dst and the total size
    };
    bool debugMapLayout(DebugMapLayout& l) const;
    // The e part is written only by synths recorded while setDebugCapture(true) (a B200-build switch: the fused synth
    // otherwise never stores the per-pixel mismatch).
    bool recordDebugMaps(cudaStream_t stream, void* dst);
    bool setDebugCapture(bool on);

    // B200-build extension for stage-by-stage parity tests: every intermediate of the latest estimate.
    struct TraceLayout {
        uint32_t nLevels, fw, fh;
        uint32_t lw[16], lh[16], bw[16], bh[16];
        uint64_t lumaOff, lumaBytes;     // per level: a (lw*lh float) then c
        uint64_t fieldOff, fieldBytes;   // per level: search then median3 (bw*bh float2 each), then sub0, sub1
        uint64_t medOff;                 // 2 floats per level: 2 x the global median used for its seeds
        uint64_t sadOff;                 // finest bw*bh float: the SADs of the scene-cut mean
        uint64_t pfOff;                  // fw*fh float2
        uint64_t stateOff;               // 4 uint32: cut, float sadMean bits, sad sum x 256, error bits
        uint64_t size;
        uint32_t seedLevel;              // the level the seed net read (UINT32_MAX: plain estimate)
        uint64_t seedOff;                // that level's bw*bh x 8 floats of net output (seedLevel != UINT32_MAX)
    };
    bool traceLayout(TraceLayout& l) const;
    bool recordTrace(cudaStream_t stream, void* dst);

    // B200-build extension (no reference counterpart): CNN-seeded estimates. params = the seed net's flat parameters
    // (fg_seednet_param_count() floats in host memory; see framegen_c.h), or null to switch the net off; level = the
    // pyramid level it reads (0 = finest; clamped to the coarsest level of the size). With the net on, recordEstimate
    // skips the levels above that level, seeds its integer search with the net's two candidates and zero (the first
    // free of the penalty when the net is confident) and runs the levels below as usual. Allocates (like resize):
    // call it outside stream capture, with earlier work retired.
    bool setSeedNet(const float* params, uint32_t level);
    uint32_t seedNetLevel() const;   // the level the next estimate seeds from, UINT32_MAX when the net is off

    // The CUDA error string of the last record that failed at a launch (null if none): a B200-build diagnostic.
    const char* lastCudaError() const;

    static constexpr uint32_t kSetRing = 32;
    static constexpr uint32_t kBlurMaxSamples = 16;
    static constexpr uint32_t kMinSize = 16;
    struct Impl;

private:
    friend class Batch;
    Impl* m = nullptr;
    const char* err_ = nullptr;
};

// B200-build extension (no counterpart in the reference): many frame pairs of any sizes and formats recorded
// together, one Interpolator per pair ("slot"). record() records every slot's estimate as recordEstimate does; the
// syntheses of all slots and times then run in one persistent launch per frame format whose CTAs take output tiles
// from a shared work counter (mixed sizes balance across the SMs) and their whole-frame fallbacks in one more launch
// per format (or one launch per synthesis: Shape::ctasPerSm = 0). The slots' estimate chains (small,
// launch-latency bound passes) are forked onto a pool of streams (events join them back), so independent slots
// overlap on the GPU, or merged into one launch per pass (Shape::mergeEstimates). A slot of multiplier m gets the generated frames at
// t = k/m, k = 1 .. m-1 (outs: each slot's m - 1 output frames, slots in order). Records allocate nothing and can be
// captured in a CUDA graph; their small parameter upload goes through a ring of 8 pinned buffers, so at most 8 records
// may be in flight. tune() times the candidate launch shapes on the device (synchronising the stream) and keeps the
// fastest. Not thread-safe, like Interpolator.
class Batch {
public:
    struct Shape {
        // the default is the shape tune() picks on the 64-pair mixed batch (one launch per synthesis, 8 streams)
        uint32_t ctasPerSm = 0;   // CTAs per SM of the persistent synthesis launches; 0: one launch per synthesis
        uint32_t order = 0;       // work order: 0 the slots as added, 1 the largest syntheses first
        uint32_t streams = 8;     // the slots' estimates run on this many forked streams (1 = the caller's only)
        uint32_t mergeEstimates = 0;   // G = 1..8: the slots' estimates as merged launches (one per pass and level
                                       // for all slots of a group) on the caller's stream, in G groups whose
                                       // syntheses start as soon as the group's estimates are recorded; 0: per slot
                                       // (slots with UI protection, a seed net or profiling fall back to per slot)
    };
    Batch();
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    int add(const InitInfo& ii, uint32_t multiplier);   // the slot's index, or -1 (see error())
    const char* error() const;
    uint32_t slots() const;
    uint32_t synthsOf(uint32_t slot) const;             // the slot's multiplier - 1
    Interpolator* slot(uint32_t i);
    bool record(cudaStream_t stream, const Frame* prev, const Frame* curr, const Frame* outs);
    int tune(cudaStream_t stream, const Frame* prev, const Frame* curr, const Frame* outs, uint32_t reps = 3);
    Shape shape() const;
    bool setShape(const Shape& s);
    struct Impl;

private:
    Impl* m = nullptr;
};

}  // namespace framegen
