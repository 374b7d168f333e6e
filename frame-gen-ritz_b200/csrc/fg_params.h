// Kernel parameter blocks and launch entry points of the V1 path (host <-> device contract inside the library).
// Every kernel takes one of these by value; the host (framegen.cpp) fills them from the size layout and Settings.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace fgk {

constexpr int kBlock = 8;          // block size at every pyramid level (proto/interp.py:43 BLOCK)
constexpr int kMaxLevels = 16;
constexpr int kPyrInKernel = 6;    // levels 0..5 come out of the luma kernel (a 32x32 tile of level 0 -> 1x1 of level 5)
constexpr int kSeedNetOut = 8;    // seed net outputs per block: c1x, c1y, c2x, c2y, confidence logit, 3 unused
constexpr int kMaxRadius = 12;     // Settings::searchRadius / searchRadiusTop upper bound (gpu/framegen.cpp validate)
// the most bytes rows 0..H-1 of a frame's first plane may span: the 8-bit kernels form pixel offsets in 32-bit words
constexpr size_t kMaxPlaneSpan = (size_t)1 << 34;

// Device-side counters and small results of one estimate / synth (one allocation, zeroed at init).
struct DevState {
    unsigned int untrusted[2];         // per synth parity: pixels whose trust ramp is past 0.5 (interp.py:238)
    unsigned int sadSum256;            // finest-level sum of roundEven(block SAD * 256) (debug counters)
    unsigned int cut;                  // scene-cut decision of the latest estimate (interp.py:190)
    float sadMean;                     // the float32 mean block SAD the cut test compares (interp.py:164)
    unsigned int medDone[kMaxLevels];  // last-block tickets of the median histograms
    unsigned int subDone;              // leaves of the scene-cut sum completed in the sub-pixel pass
    float med[kMaxLevels][2];          // per fine level: 2 x the global median of the own-parent vectors (interp.py:142)
    unsigned int err;                  // sticky error bits (bound checks that could only fail on a library bug)
};

enum : unsigned int { kErrHistRange = 1u, kErrPlan = 2u, kErrSeedNet = 4u };

// Frame formats other than 8-bit RGBA (framegen::Format) and their constants, computed on the host from InitInfo
enum : int { kFmtRgba8 = 0, kFmtRgb10 = 1, kFmtF16 = 2, kFmtNv12 = 3, kFmtP010 = 4 };
struct FmtConst {
    int format;                    // kFmt*
    int rHigh;                     // Rgb10: R in bits 20..29 (A2R10G10B10) rather than 0..9 (A2B10G10R10)
    int linear;                    // RgbaF16: Transfer::Linear, the mismatch in PQ codes
    float kWhite;                  // RgbaF16 linear: fl32(linearWhiteNits / 10000)
    float k10, k10i;               // Rgb10: fl32(255 / 1023), fl32(1023 / 255)
    float black, ys, rcr, bcb, gcb, gcr;   // YUV: luma black level, luma gain, Cr/Cb -> R'G'B' (gpu/framegen.cpp:1518-1533)
};

struct LumaPyrParams {
    const uint8_t* a;
    const uint8_t* c;
    size_t pitch;          // bytes per row of both frames
    int W, H, fs;          // frame size, flow scale (1, 2, 4)
    int ri, gi, bi;        // byte offsets of R, G, B in a 4-byte pixel
    int nlev;              // levels written here (<= kPyrInKernel)
    int vec16;             // flowScale 2 with 16-byte aligned frames and rows: the uint4 path
    const float* pq;       // RgbaF16 linear: the PQ level (fmtPq255) of every half value, indexed by its bits, or null
    int lw[kPyrInKernel], lh[kPyrInKernel];
    float* la[kPyrInKernel];
    float* lc[kPyrInKernel];
    FmtConst f;            // the luma kernel of the other formats (k_luma_fmt)
};

struct DownParams {         // one further pyramid level (INTER_AREA 0.5)
    const float* sa; const float* sc; int sw, sh;
    float* da; float* dc; int dw, dh;
    int round10;               // the other formats: round each mean to a multiple of 2^-10
};

struct SearchParams {
    const float* la; const float* lc;
    int w, h, bw, bh;
    int top;                   // coarsest level: the seed is zero
    const float2* parent;      // the parent level's median-filtered field (pw x ph)
    int pw, ph;
    const float* med;          // 2 floats: the seed candidate "global median" (already 2x)
    int R;
    float lambda;              // fl32(searchPenalty): the seed stage's penalty (interp.py:143)
    float pen[2 * kMaxRadius + 1];   // fl32(lambda * n), n = |dx| + |dy| (interp.py:121)
    float2* out;
    float* sadOut;             // optional: the winner's SAD (finest level when sub-pixel refinement is off)
    const float* cnn;          // optional: the seed net's output at this level (kSeedNetOut floats per block)
};

struct Median3Params {
    const float2* in; float2* out; int bw, bh;
    // histogram of the own-parent vectors of the next finer level (fine grid fbw x fbh), 0 = none
    int doHist, fbw, fbh, B;   // bins [-B, B] per axis
    unsigned int* hist;        // 2 * (2B + 1) bins, zero on entry, zeroed again by the last block
    unsigned int* done;
    float* medOut;             // 2 floats
    unsigned int* err;
};

struct CutPlan {               // numpy's pairwise float32 summation tree of N elements (built on the host)
    const int2* leaves;        // (start, len) per leaf, in node-slot order 0..nLeaves-1
    const int2* inner;         // (left slot, right slot) per inner node, deepest depth first
    const int* depthStart;     // inner[depthStart[d] .. depthStart[d + 1]) are computed in step d
    int nLeaves, nInner, nSteps, root;
    float* gvals;              // nLeaves + nInner floats of global scratch (k_cutmean: when they exceed kPlanSmemMax)
    const int* leafOf;         // k_subpix: the leaf of every element
    unsigned int* leafCnt;     // k_subpix: arrivals per leaf (zero between launches)
    unsigned int* leafS256;    // k_subpix: per leaf, the sum of roundEven(sad * 256)
};
constexpr size_t kPlanSmemMax = 96 * 1024;   // node values kept in shared memory up to this size

struct SubpixParams {
    const float* la; const float* lc;
    int w, h, bw, bh;
    const float2* in; float2* out; float* sads;
    float2* out0;              // optional: the vectors after the 0.5 px step
    float pen[2][3];           // fl32(lambda * step * n), step 0.5 / 0.25, n = 0..2
    // scene-cut mean in the last block
    CutPlan plan;
    float cutSad;
    DevState* st;
};

struct CutMeanParams {         // the same scene-cut reduction as a separate pass (sub-pixel refinement off)
    const float* sads; int n;
    CutPlan plan;
    float cutSad;
    DevState* st;
};

struct PixfieldParams {
    const float* ya; const float* yc; int w, h;
    const float2* v; int bw, bh;   // the finest block field
    float smooth, zero;            // bonuses (interp.py:181-182)
    float2* pf;
};

struct SynthParams {
    const uint8_t* a; const uint8_t* c; size_t pitch;
    uint8_t* out; size_t outPitch;
    int W, H, fs, fw, fh;
    int ri, gi, bi;
    const float2* pf;
    int lookup;                    // t != 0.5: the field at t by 2 fixed-point steps (interp.py:194-205)
    int mid;                       // t == 0.5: blend 0.5 * (wa + wc)
    int nearC;                     // t > 0.5: the nearer frame is curr
    float s, ka, kc, wA, wC;       // fl32(2t - 1), fl32(2t), fl32(2(1 - t)), fl32(1 - t), fl32(t)
    float trust0, trustSpan;       // trustLow, fl32(trustHigh - trustLow)
    int sZero, sOne;               // 7x7 sums S <= sZero give u = 0, S >= sOne give u = 1 (host-derived shortcuts)
    DevState* st;
    unsigned int* untrusted;       // this synth's counter (zero on entry)
    uint8_t* emap;                 // optional: per-pixel mismatch before the box (debug maps), W bytes per row
    // the other formats (k_synth_fmt): constants and the CbCr planes of YUV frames (chroma pitch shared by a and c)
    FmtConst f;
    const uint8_t* ac; const uint8_t* cc; size_t cpitch;
    uint8_t* outc; size_t outCPitch;
    // CrosshairV2's warp-tap rejection (8-bit RGBA): the UI masks of prev and curr (header + bytes, see UiV2Params);
    // both null = off
    const uint32_t* uiA; const uint32_t* uiC;
};

// One estimate pass of many frame pairs ("items") in one launch: the parameters of every item travel in the launch's
// own parameter block (a captured graph holds them; nothing is uploaded per record). The grid is one-dimensional:
// item i owns CTAs [first[i], first[i + 1]), laid out as its own grid of gx[i] CTAs across. At most kMergeMax items
// per launch (the host splits larger sets).
constexpr int kMergeMax = 48;
template <class P>
struct Merged {
    P item[kMergeMax];
    int first[kMergeMax + 1];
    int gx[kMergeMax];
    int n;
};

struct SynthBatchArgs {             // k_synth_batch: a work list of syntheses
    const SynthParams* items;      // per item (device array)
    const int* tileStart;          // nItems + 1: the first tile of each item in the list, then the total
    const int* tilesX;             // per item: output tiles across
    int nItems, total;
    unsigned int* counter;         // the next tile to take (zero before the launch)
};

// Motion blur (recordSynthBlur, gpu/framegen.h:553-573): one output = the weighted average of n sub-frames, each
// exactly the 8-bit frame recordSynth(t_k) gives; the weights are integers summing to 2^16 (out = (sum q_k v_k +
// 2^15) >> 16 per byte).
constexpr int kBlurMax = 16;
struct BlurSample {
    int mode;                      // 0: a synthesis at t_k; 1: the real frame prev (t_k <= 0); 2: curr (t_k >= 1)
    int lookup, mid, nearC;        // recordSynth(t_k)'s SynthParams fields
    float s, ka, kc, wA, wC;
    uint32_t q;                    // weight, units of 2^-16
};
struct BlurParams {
    SynthParams base;              // the t-independent fields (untrusted and emap unused)
    BlurSample smp[kBlurMax];
    int n;
    int fix;                       // 0: main pass, counts each synthesis' untrusted pixels into cnt[k]; 1: the fix-up
    double frac;                   // globalFallback (interp.py:238): a sample past it is its nearer real frame
    unsigned int* cnt;             // kBlurMax counters, zero before the main pass
};

struct FallbackParams {
    const uint8_t* a; const uint8_t* c; size_t pitch;
    uint8_t* out; size_t outPitch;
    int W, H, nearC;
    double frac;                   // globalFallback
    const unsigned int* untrusted;
    unsigned int* untrustedNext;   // the next synth's counter, zeroed here
    // the other formats (k_fallback_fmt): bytes per row of plane 0, and the CbCr planes (rows of cbytes bytes, ch rows)
    size_t rowBytes, cbytes;
    int ch;
    const uint8_t* ac; const uint8_t* cc; size_t cpitch;
    uint8_t* outc; size_t outCPitch;
};

// once per process and device: the dynamic shared-memory limits of the kernels that need more than 48 KB
cudaError_t prepareKernels();
size_t synthSmemBytes(int fs);

// launchers (fg_kernels.cu); each returns the launch's cudaError_t
cudaError_t launchLumaPyr(const LumaPyrParams& p, cudaStream_t s);
cudaError_t launchDown(const DownParams& p, cudaStream_t s);
cudaError_t launchSearch(const SearchParams& p, cudaStream_t s);
cudaError_t launchMedian3(const Median3Params& p, cudaStream_t s);
cudaError_t launchSubpix(const SubpixParams& p, cudaStream_t s);
cudaError_t launchCutMean(const CutMeanParams& p, cudaStream_t s);
cudaError_t launchPixfield(const PixfieldParams& p, cudaStream_t s);
cudaError_t launchSynth(const SynthParams& p, cudaStream_t s);
cudaError_t launchFallback(const FallbackParams& p, cudaStream_t s);
// batches (framegen.cpp Batch): many syntheses in one persistent launch, their fallbacks in one launch
cudaError_t launchSynthBatch(const SynthBatchArgs& b, int grid, size_t smem, cudaStream_t s);
// merged estimate passes (every item of a launch takes the same kernel variant; the host groups them by
// searchVariant / median3Variant); the CTA counts per item (first, gx) are filled in by the launchers
cudaError_t launchLumaPyrMerged(Merged<LumaPyrParams>& m, cudaStream_t s);
cudaError_t launchLumaFmtMerged(Merged<LumaPyrParams>& m, int format, cudaStream_t s);
int searchVariant(const SearchParams& p);     // the kernel a search runs: R (1..6) x 2 + latency form, or 100 + R
int median3Variant(const Median3Params& p);   // 0: one CTA, 1: cluster, 2: grid with a last-CTA ticket
cudaError_t launchSearchMerged(Merged<SearchParams>& m, cudaStream_t s);
cudaError_t launchMedian3Merged(Merged<Median3Params>& m, cudaStream_t s);
cudaError_t launchSubpixMerged(Merged<SubpixParams>& m, cudaStream_t s);
cudaError_t launchPixfieldMerged(Merged<PixfieldParams>& m, cudaStream_t s);
// one pass of a motion blur, 8-bit RGBA frames: the main pass (fix = 0), then the fix-up (fix = 1)
cudaError_t launchSynthBlur(const BlurParams& bp, int fix, cudaStream_t s);
int synthBatchCtasPerSm(size_t smem);
cudaError_t launchFallbackBatch(const FallbackParams* items, int nItems, cudaStream_t s);
size_t synthKernelSmem(int fs);   // k_synth's / k_synth_batch's dynamic shared memory at this flow scale
int synthTilesX(int W);           // output tiles of a synthesis across / down
int synthTilesY(int H);
// the other formats (fg_formats.cu)
cudaError_t prepareFormatKernels();
cudaError_t launchLumaFmt(const LumaPyrParams& p, cudaStream_t s);
// the PQ level of every half value (65536 floats) for a linear RgbaF16 luma at this white level
cudaError_t launchPqTable(float* tab, float kWhite, cudaStream_t s);
cudaError_t launchSynthFmt(const SynthParams& p, cudaStream_t s);
// many syntheses of one of the other formats in one persistent launch (as launchSynthBatch), and their fallbacks
cudaError_t launchSynthFmtBatch(const SynthBatchArgs& b, int format, int grid, size_t smem, cudaStream_t s);
int synthFmtBatchCtasPerSm(int format, size_t smem);
size_t synthFmtKernelSmem(int format, int fs);   // k_synth_fmt's / k_synth_fmt_batch's dynamic shared memory
cudaError_t launchFallbackFmtBatch(const FallbackParams* items, int nItems, cudaStream_t s);
// one pass of a motion blur in the other formats (bp.base.f.format): the main pass (fix = 0), then the fix-up
cudaError_t launchSynthBlurFmt(const BlurParams& bp, int fix, cudaStream_t s);
cudaError_t launchFallbackFmt(const FallbackParams& p, cudaStream_t s);

// CrosshairV2 static-UI protection (gpu/shaders/ui_v2_update.comp, ui_v2_mask.comp, ui_patch.comp), 8-bit RGBA.
// State: 4 words per pixel of the work rectangle (the box grown by 1 px, clamped to the frame):
//   w0 = previous original (r | g << 8 | b << 16) | still-and-contrasty count << 24
//   w1 = last confirmed colour | flags << 24 (bit 0 in the mask, bit 1 has a stored colour, bit 2 still in this pair)
//   w2 = consecutive changed frames while in the mask | consecutive stored-colour matches while out of it << 8
// Mask buffer of one kept frame: header words [1] = x | y << 16, [2] = w | h << 16, [3] = words per row; from word 4
// the bytes (4 pixels per word): 255 = UI and unchanged in this pair (pasted), 64 = UI but changed, 0 = not UI.
constexpr int kUiMaskHeader = 4;
struct UiV2Params {
    const uint8_t* frame; size_t pitch;
    int W, H, ri, gi, bi;
    FmtConst f;                    // the frame format
    const float* pq;               // linear RgbaF16: the PQ level of every half value (LumaPyrParams::pq)
    const uint8_t* frameC; size_t cpitch;   // YUV: the frame's CbCr plane
    int bx, by, bw, bh;            // the box (detection)
    int wx, wy, ww, wh;            // the work rectangle (state and mask)
    uint32_t* st;
    int reset;                     // the state describes no previous frame
    float thr, cthr;               // uiStillThreshold, uiContrastThreshold (8-bit levels)
    int still, leave, reentry;     // uiStillFrames, uiLeaveFrames, uiReentryFrames
    uint32_t* mask;                // observe: this frame's mask buffer; recordTrack: null
    int maskStride;                // words per mask row
};
struct UiPatchParams {
    const uint8_t* curr; size_t pitch;
    uint8_t* out; size_t outPitch;
    const uint32_t* mask;
    int format;                    // kFmt*
    const uint8_t* currC; size_t cpitch;     // YUV: the CbCr planes of curr and of the output
    uint8_t* outC; size_t outCPitch;
};
// the estimate fill (Settings::uiEstimateFill): level-0 luma cells holding UI pixels re-averaged over their not-UI
// pixels, prev's (mask ma, luma la) and curr's (mc, lc); cells of the rectangle (cx0, cy0) .. + (ncx, ncy)
struct UiFillParams {
    const uint8_t* a; const uint8_t* c; size_t pitch;
    int W, H, ri, gi, bi, fs, fw, fh;
    const uint32_t* ma; const uint32_t* mc;
    float* la; float* lc;
    int cx0, cy0, ncx, ncy;
    FmtConst f;                    // Rgb10 / RgbaF16 (launchUiFillFmt): the format's luma
    const float* pq;
};
cudaError_t launchUiFill(const UiFillParams& p, cudaStream_t s);
cudaError_t launchUiFillFmt(const UiFillParams& p, cudaStream_t s);   // the estimate fill of Rgb10 / RgbaF16 frames
cudaError_t launchUiV2Update(const UiV2Params& p, cudaStream_t s);
cudaError_t launchUiV2Mask(const UiV2Params& p, cudaStream_t s);
cudaError_t launchUiPatch(const UiPatchParams& p, int wx, int wy, int ww, int wh, cudaStream_t s);

// Streaming multiprocessors of the current device (cached per device); grids of the grid-stride kernels are sized in
// multiples of it.
int smCount();

// The trust ramp of interp.py:236, u(S) = clip((float(S / 49) - trustLow) / (trustHigh - trustLow), 0, 1) for the 7x7
// mismatch sums S = 0 .. 49 * 255, is monotone in S: S <= sZero gives exactly 0 and S >= sOne exactly 1 (the synthesis
// kernels compute the ramp in between). Host-side, from the settings' thresholds.
inline void trustShortcuts(float trustLow, float trustHigh, int& sZero, int& sOne) {
    const float t0 = trustLow, span = (float)((double)trustHigh - (double)trustLow);
    auto u = [&](int S) {
        const float eb = (float)((double)S * (1.0 / 49.0));
        float v = (eb - t0) / span;
        return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    };
    sZero = -1;
    for (int S = 0; S <= 49 * 255 && u(S) == 0.0f; S++) sZero = S;
    sOne = 49 * 255 + 1;
    for (int S = 49 * 255; S >= 0 && u(S) == 1.0f; S--) sOne = S;
}

}  // namespace fgk
