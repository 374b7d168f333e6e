/* framegen_c.h -- the C ABI of the B200 framegen library (libframegen_b200.so).
 *
 * Plain pointers, sizes and POD structs only: the binding surface for hosts that cannot take the C++ header
 * (ctypes, cgo, JNI, N-API). Every entry point is a thin forward to framegen::Interpolator (include/framegen.h),
 * whose methods each replace the like-named member of frame-gen-ritz's gpu/framegen.h (cited per function).
 * Booleans are int (1 = true). Strings are static literals owned by the library. Streams are cudaStream_t passed as
 * void* (NULL = the legacy default stream). Frames are device pointers with a row pitch in bytes.
 */
#ifndef FRAMEGEN_C_H
#define FRAMEGEN_C_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fg_interpolator fg_interpolator;

/* framegen::Settings (gpu/framegen.h:167-409, the V1 fields and the static-UI protection fields). `size` =
 * sizeof(fg_settings) for ABI growth: a caller built against the shorter struct (ending at pyramidMinSide) gets the
 * UI fields' defaults. */
typedef struct fg_settings {
    uint32_t size;
    float trustLow, trustHigh, globalFallback, sceneCutSad, hudBonus, smoothBonus, searchPenalty;
    uint32_t searchRadius, searchRadiusTop, subpixel;
    uint32_t uiProtection, blurSamples, blurWeights, motionVersion;
    uint32_t flowScale, pyramidMinSide;
    /* static-UI protection (gpu/framegen.h:196-305) */
    uint32_t uiHistory;
    float uiBoxHeightFrac;
    uint32_t uiBoxWidth, uiBoxHeight;
    float uiCrosshairArea;
    int32_t uiBoxOffsetX, uiBoxOffsetY;
    uint32_t uiStillFrames;
    float uiStillThreshold;
    uint32_t uiInpaintReach;
    float uiMaxStillFraction, uiContrastThreshold;
    uint32_t uiLeaveFrames, uiReentryFrames, uiEstimateFill;
} fg_settings;

/* framegen::Frame (gpu/framegen.h:154-159); the first plane spans at most 2^34 bytes */
typedef struct fg_frame {
    void* data;
    uint64_t pitch;
    void* chroma;
    uint64_t chroma_pitch;
} fg_frame;

/* framegen::InitInfo (gpu/framegen.h:411-441) */
typedef struct fg_init_info {
    uint32_t size;
    uint32_t width, height;
    uint32_t view_format;      /* VkFormat number, e.g. 44 = B8G8R8A8_UNORM, 37 = R8G8B8A8_UNORM */
    uint32_t transfer;
    float linear_white_nits;
    uint32_t yuv_matrix, yuv_full_range;
    int32_t device;
    fg_settings settings;
} fg_init_info;

/* Interpolator::DebugMapLayout (gpu/framegen.h:736-739) */
typedef struct fg_debug_map_layout {
    uint32_t W, H, fw, fh, bw, bh, fscale, eStride;
    uint64_t blockOff, pixOff, eOff, size;
} fg_debug_map_layout;

/* Interpolator::TraceLayout (B200-build extension, no reference counterpart: stage parity tests) */
typedef struct fg_trace_layout {
    uint32_t nLevels, fw, fh;
    uint32_t lw[16], lh[16], bw[16], bh[16];
    uint64_t lumaOff, lumaBytes, fieldOff, fieldBytes, medOff, sadOff, pfOff, stateOff, size;
    uint32_t seedLevel;
    uint64_t seedOff;
} fg_trace_layout;

uint32_t fg_abi_version(void);
void fg_default_settings(fg_settings* s);                    /* Settings{} defaults */
void fg_default_init_info(fg_init_info* ii);                 /* InitInfo{} defaults */
int fg_format_of(uint32_t view_format, uint32_t* format);    /* gpu/framegen.h:140 formatOf */

fg_interpolator* fg_create(void);
void fg_destroy(fg_interpolator* fg);                        /* destroy() + free; gpu/framegen.h:456 */
int fg_init(fg_interpolator* fg, const fg_init_info* ii);    /* gpu/framegen.h:451 */
const char* fg_init_error(const fg_interpolator* fg);        /* gpu/framegen.h:453 */
uint32_t fg_format(const fg_interpolator* fg);               /* gpu/framegen.h:455 */
int fg_resize(fg_interpolator* fg, uint32_t w, uint32_t h, uint32_t view_format);   /* gpu/framegen.h:461 */

int fg_validate(const fg_settings* s);                                              /* gpu/framegen.h:464 */
const char* fg_settings_error_format(const fg_settings* s, uint32_t format);        /* gpu/framegen.h:468 */
const char* fg_settings_error(const fg_interpolator* fg, const fg_settings* s);     /* gpu/framegen.h:472 */
const char* fg_size_error(const fg_interpolator* fg, uint32_t w, uint32_t h);       /* gpu/framegen.h:480 */
int fg_set_settings(fg_interpolator* fg, const fg_settings* s);                     /* gpu/framegen.h:500 */
int fg_reconfigure(fg_interpolator* fg, const fg_settings* s);                      /* gpu/framegen.h:505 */
void fg_get_settings(const fg_interpolator* fg, fg_settings* s);                    /* gpu/framegen.h:507 */

void fg_begin_frame(fg_interpolator* fg);                                           /* gpu/framegen.h:511 */
void fg_release_unused_ui(fg_interpolator* fg);                                     /* gpu/framegen.h:693 */
void fg_release_unused_motion(fg_interpolator* fg);                                 /* gpu/framegen.h:700 (no-op here) */
int fg_record_estimate(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr);   /* :549 */
/* Static-UI protection, CrosshairV2: gpu/framegen.h:610 recordObserve, :691 recordTrack (Interpolator::recordObserve) */
int fg_record_observe(fg_interpolator* fg, void* stream, const fg_frame* frame);
int fg_record_track(fg_interpolator* fg, void* stream, const fg_frame* frame);
/* gpu/framegen.h:484-494: Interpolator::boxSize / boxRect / boxMargin / workRect (rect = {x, y, w, h}) */
void fg_box_size(const fg_settings* s, uint32_t w, uint32_t h, uint32_t* box_w, uint32_t* box_h);
void fg_box_rect(const fg_settings* s, uint32_t w, uint32_t h, int32_t rect[4]);
uint32_t fg_box_margin(const fg_settings* s);
void fg_work_rect(const fg_settings* s, uint32_t w, uint32_t h, int32_t rect[4]);
/* B200-build extension (parity tests): Interpolator::uiTraceBytes / uiTrace, the CrosshairV2 state and a kept mask */
uint64_t fg_ui_trace_bytes(const fg_interpolator* fg);
int fg_ui_trace(fg_interpolator* fg, void* stream, const void* frame, void* dst);
int fg_record_synth(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr,
                    const fg_frame* out, float t);                                                        /* :550 */
int fg_record(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr,
              const fg_frame* out, float t);                                                              /* :551 */
/* gpu/framegen.h:573 recordSynthBlur: the weighted average of settings.blurSamples sub-frames over [t0, t1]
 * (framegen.h documents the samples, weights and rounding), every format */
int fg_record_synth_blur(fg_interpolator* fg, void* stream, const fg_frame* prev, const fg_frame* curr,
                         const fg_frame* out, float t0, float t1);
/* Interpolator::blurPlan (host only): the sample times and weights (units of 2^-16) of a blur into arrays of 16;
 * weights 0 = Even, 1 = Gaussian; returns the number of samples, 0 if refused */
uint32_t fg_blur_plan(uint32_t samples, uint32_t weights, float t0, float t1, float* times, uint32_t* q);

int fg_set_profiling(fg_interpolator* fg, int on);                                   /* gpu/framegen.h:705 */
/* gpu/framegen.h:717 readTimings: up to `capacity` names and nanoseconds; *count = the number of groups */
int fg_read_timings(fg_interpolator* fg, const char** names, uint64_t* ns, uint32_t capacity, uint32_t* count);

/* Interpolator::readCosts: the pacer's cost-guard inputs (gpu/pacing.h:869-871) from the last profile */
typedef struct fg_costs {
    float estimate_ms, synth_ms;   /* -1: none in the profile */
    uint32_t seq, synths;          /* seq changes with every new profile; synths: syntheses in it */
} fg_costs;
int fg_read_costs(fg_interpolator* fg, fg_costs* c);

int fg_record_debug_counters(fg_interpolator* fg, void* stream, void* dst);          /* gpu/framegen.h:726 */
uint32_t fg_debug_sad_blocks(const fg_interpolator* fg);                             /* gpu/framegen.h:727 */
int fg_get_debug_map_layout(const fg_interpolator* fg, fg_debug_map_layout* l);          /* gpu/framegen.h:740 */
int fg_record_debug_maps(fg_interpolator* fg, void* stream, void* dst);              /* gpu/framegen.h:741 */
int fg_set_debug_capture(fg_interpolator* fg, int on);      /* B200-build switch: synths store e for debug maps */
int fg_get_trace_layout(const fg_interpolator* fg, fg_trace_layout* l);                  /* B200-build extension */
int fg_record_trace(fg_interpolator* fg, void* stream, void* dst);                   /* B200-build extension */
const char* fg_last_error(const fg_interpolator* fg);   /* the last CUDA error a record met (null if none) */

/* Batches -- no counterpart in the reference (B200-build extension; framegen::Batch in include/framegen.h): many
 * frame pairs of any sizes and formats recorded together, one interpolator per slot; the syntheses of all slots run
 * in one persistent launch per frame format. fg_batch_add: the slot's init info and multiplier m (t = k/m, k = 1 .. m-1);
 * returns its index or -1. fg_batch_record: prev[i], curr[i] per slot and outs = every slot's m - 1 output frames,
 * slots in order. fg_batch_tune: times the launch shapes on these frames (synchronises the stream), keeps the
 * fastest, returns its index (-1 on failure). */
typedef struct fg_batch fg_batch;
fg_batch* fg_batch_create(void);
void fg_batch_destroy(fg_batch* b);
int fg_batch_add(fg_batch* b, const fg_init_info* ii, uint32_t multiplier);
const char* fg_batch_error(const fg_batch* b);
uint32_t fg_batch_slots(const fg_batch* b);
int fg_batch_record(fg_batch* b, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* outs);
int fg_batch_tune(fg_batch* b, void* stream, const fg_frame* prev, const fg_frame* curr, const fg_frame* outs,
                  uint32_t reps);
void fg_batch_get_shape(const fg_batch* b, uint32_t* ctas_per_sm, uint32_t* order, uint32_t* streams);
int fg_batch_set_shape(fg_batch* b, uint32_t ctas_per_sm, uint32_t order, uint32_t streams);
/* the same with Batch::Shape::mergeEstimates (fg_batch_set_shape sets it to 0); fg_batch_merge_estimates reads it */
int fg_batch_set_shape_merged(fg_batch* b, uint32_t ctas_per_sm, uint32_t order, uint32_t streams, uint32_t merge_estimates);
uint32_t fg_batch_merge_estimates(const fg_batch* b);
int fg_batch_trace_layout(fg_batch* b, uint32_t slot, fg_trace_layout* l);   /* a slot's Interpolator::traceLayout */
int fg_batch_trace(fg_batch* b, uint32_t slot, void* stream, void* dst);     /* a slot's Interpolator::recordTrace */

/* The seed proposer -- no counterpart in the reference's V1 path (B200-build extension). A 6-layer 3x3 conv net
 * (csrc/fg_seednet.cu) reading one pyramid level's luma (prev, curr) and proposing, per 8x8 block of that level, two
 * candidate half-vectors and a confidence logit for the integer block search. Inputs are NHWC bfloat16 [B][h][w][2]
 * made by fg_seednet_pack; outputs float [B][ceil(h/8)][ceil(w/8)][8] (c1x, c1y, c2x, c2y, logit, 3 unused);
 * training targets float [B][ceil(h/8)][ceil(w/8)][6] (truth x, y, search x, y, weight, unused). Parameters: a flat
 * float array of fg_seednet_param_count() values, per layer weights [cout][3*ky+kx][cin] then biases [cout].
 * All device pointers; calls go to the net's device, stream-ordered; returns 1 on success, 0 otherwise. */
typedef struct fg_seednet fg_seednet;
/* Interpolator::setSeedNet / seedNetLevel (include/framegen.h): CNN-seeded estimates from level `level` (null = off) */
int fg_set_seed_net(fg_interpolator* fg, const float* host_params, uint32_t level);
uint32_t fg_seed_net_level(const fg_interpolator* fg);
uint32_t fg_seednet_param_count(void);
fg_seednet* fg_seednet_create(int device, int max_batch, int max_h, int max_w);   /* workspace for inputs up to this */
void fg_seednet_destroy(fg_seednet* net);
const char* fg_seednet_error(const fg_seednet* net);
int fg_seednet_set_params(fg_seednet* net, const float* host_params);   /* also resets Adam's state */
int fg_seednet_get_params(fg_seednet* net, float* host_params);
int fg_seednet_get_grads(fg_seednet* net, float* host_grads);         /* the gradient accumulated since the last step */
int fg_seednet_pack(void* stream, const float* luma_prev, const float* luma_curr, int n, void* x);
int fg_seednet_forward(fg_seednet* net, void* stream, const void* x, int batch, int h, int w, float* out);
/* the same from the float luma planes [B][h][w] of prev and curr (the first layer packs them as it reads) */
int fg_seednet_forward_luma(fg_seednet* net, void* stream, const float* luma_prev, const float* luma_curr, int batch, int h,
                           int w, float* out);
/* forward + loss + backward: adds dLoss/dParams to the gradient; *loss (device float, optional) = the batch's loss */
/* The same forward as fg_seednet_forward_luma, fused into two launches on the tensor cores (tcgen05, accumulators in
 * tensor memory); the Interpolator's seed net runs this one. Same outputs up to the order of the f32 accumulation. */
int fg_seednet_forward_fused(fg_seednet* net, void* stream, const float* luma_prev, const float* luma_curr, int batch,
                            int h, int w, float* out);
/* The fused forward's sticky error bits (4: a tensor-core wait gave up) on the net's own flag; synchronous. */
uint32_t fg_seednet_fused_errors(fg_seednet* net);
int fg_seednet_backward(fg_seednet* net, void* stream, const void* x, int batch, int h, int w, const float* targets,
                        float* loss);
int fg_seednet_zero_grads(fg_seednet* net, void* stream);
int fg_seednet_adam(fg_seednet* net, void* stream, float lr);          /* one Adam step (0.9, 0.999, 1e-8); zeroes grads */
/* Data-parallel training: the float32 gradient accumulator on the net's device (fg_seednet_param_count() values, valid
 * until destroy), for an in-place all-reduce (sum) between backward and the step; the step then reads it scaled by
 * grad_scale (1 / ranks), which gives every rank the update of the whole global batch. */
float* fg_seednet_grad_buffer(fg_seednet* net);
int fg_seednet_adam_scaled(fg_seednet* net, void* stream, float lr, float grad_scale);

/* fg_record_synth_noalloc -- no counterpart in the reference. The synthesis of one generated frame (what
 * fg_record_synth records after an estimate) for hosts that cannot allocate device memory when they generate frames:
 * a compositor or overlay running inside another program's frame callback under that program's memory budget, a
 * real-time presentation thread that must not block on cudaMalloc / cudaFree, a plugin that is handed buffers but no
 * allocator. It allocates nothing and needs no fg_interpolator: the caller passes the two frames, the output, the
 * pair's per-pixel half-vector field (fw x fh float2 on the device, 8-byte aligned, fw = rint(width / flowScale), fh
 * likewise: the field fg_record_estimate computes, e.g. read with fg_record_trace) and the pair's scene-cut decision;
 * the rest lives in one static device array inside the library (about 24 MiB), sized for at most 3,145,728 flow pixels
 * (3840x2160 at flowScale 2). Larger frames are refused with an error, before anything is launched. Every call shares
 * that array and it keeps the last call's contents; calls that overlap on the GPU race on it. The first call on a
 * device looks the array's device address up (host set-up work), and with CUDA's lazy module loading that is also when
 * the driver places the 24 MiB array on the device, so the first call can fail for lack of device memory: make it at
 * set-up time, before any stream capture. Returns 1 on success; 0 with *error (if error is not null) set to a static
 * message otherwise. view_format: 37 (R8G8B8A8) or 44 (B8G8R8A8); t in (0, 1). */
int fg_record_synth_noalloc(void* stream, uint32_t view_format, uint32_t width, uint32_t height, const fg_frame* prev,
                            const fg_frame* curr, const fg_frame* out, const float* field, int cut, float t,
                            const fg_settings* settings, const char** error);

#ifdef __cplusplus
}
#endif
#endif
