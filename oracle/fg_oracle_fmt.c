/*
 * fg_oracle_fmt.c -- CPU restatement of frame-gen-ritz's V1 path for the frame formats other than 8-bit RGBA:
 * Rgb10 (A2B10G10R10 / A2R10G10B10), RgbaF16 (encoded, or linear light measured as PQ codes), Nv12 and P010.
 *
 * TEST INFRASTRUCTURE ONLY, like fg_oracle.c: the checker of the CUDA path for these formats.
 *
 * proto/interp.py is 8-bit BGR only, so these formats have no NumPy reference; the reference defines them in its
 * Vulkan shaders: gpu/shaders/format.glsl:29-106 (levels, the mismatch metric, the stores), luma.comp:9-27 (the luma
 * of each format), motion_v1.glsl:86-144 (warp taps, chroma siting), resolve.comp:48-83 (blend and store per
 * format) and gpu/framegen.cpp:1508-1539 (the YUV constants). This file restates that math, with these definitions
 * where the shaders leave the rounding to the GPU (texture filtering, float -> UNORM conversion, summation order):
 *
 *   levels      Rgb10: code * K10 with K10 = fl32(255/1023); RgbaF16: v * 255, or with Transfer::Linear
 *               pq(v) * 255 (pq below); Nv12: the code; P010: the 16-bit word * 2^-8 (= code10 / 4).
 *               YUV luma for the motion estimate: (level - black) * ys (format.glsl fgLuma).
 *   est. luma   y = ((4899 r + 9617 g) + 1868 b) * 2^-14 on the levels (RGB formats; luma.comp:12-21), the YUV luma
 *               above; then Q = clamp(rint(4 y), 0, 1020), quarter levels (the 10-bit code grid). Level 0 =
 *               rint(4 sum(Q) / n) / 16 over the n valid pixels of each flowScale cell; pyramid levels = the 2x2
 *               mean rounded half-even to a multiple of 2^-10. With every luma on these grids, each SAD, tap and box
 *               sum of the estimate is exact in float32 whatever the order, as for 8-bit RGBA.
 *   warp taps   the sample point rounded half-even to 1/32 px (motion_v1.glsl:93-97), then the bilinear tap of the
 *               4 texels with cv2's float formula ((p00 w00 + p01 w01) + p10 w10) + p11 w11, clamped to the edge.
 *               RGB formats filter the raw channel (Rgb10 codes, F16 values) and then scale to levels; the chroma
 *               plane of a YUV frame is sampled at the same normalised position, i.e. chroma texel
 *               (x + 0.5) / 2 - 0.5 = (X - 16) / 64 for the 1/32-px coordinate X (6-bit fractions), so a block
 *               centre at zero motion gives its own chroma texel back. For odd sizes the last chroma column / row
 *               covers one pixel (the shaders' normalised coordinates would stretch the plane by (W + 1) / 2W).
 *   mismatch    e = (uint) min(max over the channels of |metric(a) - metric(c)|, 255) (format.glsl FG_DIFF,
 *               FG_PACKE); YUV: the (Y, Cb, Cr) level differences converted to R'G'B' differences (fgYuvDiff).
 *   blend       m = 0.5 (wa + wc) at t = 0.5, else fl32(wA wa) + fl32(wC wc); o = fl32(m (1 - u)) + fl32(n u),
 *               in the source's own space (levels for Rgb10 / YUV, values for F16). Stores: Rgb10 code =
 *               floor(clamp(o, 0, 255) * fl32(1023/255) + 0.5); F16 half round-to-nearest-even; YUV code =
 *               clamp(floor(o / ql + 0.5), 0, codes) (fgOut). Alpha (RGB formats): the nearer frame's.
 *   YUV chroma  written for the even-even pixel of each 2x2 block with that pixel's trust; the warp starts at the
 *               block centre (x + 0.5, y + 0.5) with the pixel's half-vector (motion_v1.glsl:134-144).
 *   pq          y = clamp(v * fl32(white / 10000), 0, 1); p = y^m1; pq = ((c1 + c2 p) / (1 + c3 p))^m2 with the
 *               SMPTE ST 2084 constants; x^e = exp2(e log2 x) with the log2 / exp2 series below (float ops only, the
 *               same in the CUDA kernels).
 * The whole-frame decisions, the field at t, its upsampling, the 7x7 box and the trust ramp are the Rgba8 path's.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fg_oracle_internal.h"

enum { FMT_RGB10 = 1, FMT_F16 = 2, FMT_NV12 = 3, FMT_P010 = 4 };

/* the per-format constants, computed by fgo_fmt_init the way the library's host code computes them */
typedef struct fgo_fmt {
    int format;       /* 1 Rgb10, 2 RgbaF16, 3 Nv12, 4 P010 */
    int rHigh;        /* Rgb10: R in bits 20..29 (A2R10G10B10) instead of 0..9 (A2B10G10R10) */
    int linear;       /* RgbaF16: Transfer::Linear */
    float kWhite;     /* RgbaF16 linear: fl32(white / 10000) */
    float k10, k10i;  /* Rgb10: fl32(255/1023), fl32(1023/255) */
    float black, ys, rcr, bcb, gcb, gcr;   /* YUV (format.glsl YU_*) */
} fgo_fmt;

/* one frame: plane 0 (RGB pixels, or the Y plane) and the CbCr plane of the YUV formats */
typedef struct fgo_frame {
    const uint8_t* p;
    long pitch;
    const uint8_t* c;
    long cpitch;
} fgo_frame;

/* gpu/framegen.cpp:1508-1539: BT.601 / 709 / 2020 constants, full or limited range */
void fgo_fmt_init(fgo_fmt* f, int format, int rHigh, int linear, float whiteNits, int matrix, int fullRange) {
    memset(f, 0, sizeof(*f));
    f->format = format;
    f->rHigh = rHigh;
    f->linear = linear;
    f->kWhite = whiteNits / 10000.0f;
    f->k10 = (float)(255.0 / 1023.0);
    f->k10i = (float)(1023.0 / 255.0);
    double kr = 0.2126, kb = 0.0722;
    if (matrix == 0) { kr = 0.299; kb = 0.114; }
    if (matrix == 2) { kr = 0.2627; kb = 0.0593; }
    const double kg = 1.0 - kr - kb;
    const double sY = fullRange ? 1.0 : 255.0 / 219.0, sC = fullRange ? 1.0 : 255.0 / 224.0;
    f->black = fullRange ? 0.0f : 16.0f;
    f->ys = (float)sY;
    f->rcr = (float)(sC * 2.0 * (1.0 - kr));
    f->bcb = (float)(sC * 2.0 * (1.0 - kb));
    f->gcb = (float)(-sC * 2.0 * (1.0 - kb) * kb / kg);
    f->gcr = (float)(-sC * 2.0 * (1.0 - kr) * kr / kg);
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float absf(float v) { return v < 0.0f ? -v : v; }
static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* ---------------------------------------------------------------------------------------------- float helpers */

/* log2 of a positive normal float: x = 2^e m with m in [sqrt(1/2), sqrt(2)); log2 m = 2/ln2 atanh(s),
 * s = (m - 1) / (m + 1), by its odd series to s^9 (|s| <= 0.172: truncation below 1e-9) */
float fgo_log2(float x) {
    const uint32_t b = f2u(x);
    int e = (int)((b >> 23) & 255u) - 127;
    float m = u2f((b & 0x7FFFFFu) | 0x3F800000u);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e += 1; }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = 0x1.484b14p-2f;
    p = p * z;
    p = p + 0x1.a61762p-2f;
    p = p * z;
    p = p + 0x1.2776c6p-1f;
    p = p * z;
    p = p + 0x1.ec709ep-1f;
    p = p * z;
    p = p + 0x1.715476p+1f;
    return (float)e + s * p;
}

/* 2^x for -126 <= x < 128 (0 below): x = n + g + 1/2 with n = floor(x), 2^(g + 1/2) = sqrt2 e^(g ln2), the
 * exponential's series to degree 7 (|g ln2| <= 0.347: truncation below 1e-8) */
float fgo_exp2(float x) {
    if (!(x >= -126.0f)) return 0.0f;
    const float n = floorf(x);
    const float g = (x - n) - 0.5f;
    float p = 0x1.ffcbfcp-17f;
    p = p * g;
    p = p + 0x1.430912p-13f;
    p = p * g;
    p = p + 0x1.5d87fep-10f;
    p = p * g;
    p = p + 0x1.3b2ab6p-7f;
    p = p * g;
    p = p + 0x1.c6b08ep-5f;
    p = p * g;
    p = p + 0x1.ebfbe0p-3f;
    p = p * g;
    p = p + 0x1.62e430p-1f;
    p = p * g;
    p = p + 1.0f;
    p = p * 0x1.6a09e6p+0f;
    return p * u2f((uint32_t)((int)n + 127) << 23);
}

/* format.glsl fgPq * 255: the level of a linear value as an 8-bit PQ code */
float fgo_pq255(float v, float kWhite) {
    float y = v * kWhite;
    y = clampf(y, 0.0f, 1.0f);
    float p = 0.0f;
    if (y >= 0x1p-126f) p = fgo_exp2(0.1593017578125f * fgo_log2(y));
    const float num = 0.8359375f + 18.8515625f * p;
    const float den = 1.0f + 18.6875f * p;
    const float r = num / den;
    return fgo_exp2(78.84375f * fgo_log2(r)) * 255.0f;
}

/* IEEE half <-> float, round to nearest even */
float fgo_h2f(uint16_t h) {
    const uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 31u, m = h & 1023u;
    if (e == 0) {
        const float v = (float)m * 0x1p-24f;
        return s ? -v : v;
    }
    if (e == 31) return u2f(s | 0x7F800000u | (m << 13));
    return u2f(s | ((e + 112u) << 23) | (m << 13));
}

uint16_t fgo_f2h(float f) {
    const uint32_t x = f2u(f), sign = (x >> 16) & 0x8000u, ax = x & 0x7FFFFFFFu;
    if (ax > 0x7F800000u) return (uint16_t)(sign | 0x7E00u);        /* NaN */
    if (ax >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);       /* >= 65520: infinity */
    if (ax < 0x38800000u) {                                          /* below 2^-14: a subnormal half (or 0) */
        const int e = (int)(ax >> 23);
        if (e < 102) return (uint16_t)sign;                          /* below 2^-25: 0 */
        const uint32_t m = (ax & 0x7FFFFFu) | 0x800000u;
        const int sh = 126 - e;                                      /* value / 2^-24 = m >> sh */
        uint32_t q = m >> sh;
        const uint32_t rem = m & ((1u << sh) - 1u), half = 1u << (sh - 1);
        if (rem > half || (rem == half && (q & 1u))) q++;
        return (uint16_t)(sign | q);
    }
    uint32_t h = ((ax >> 13) - (112u << 10));
    const uint32_t rem = ax & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return (uint16_t)(sign | h);
}

/* integer num / n rounded half to even (num >= 0, n > 0) */
static inline int rne_div(int num, int n) {
    int q = num / n;
    const int r = num - q * n;
    if (2 * r > n || (2 * r == n && (q & 1))) q++;
    return q;
}

/* ---------------------------------------------------------------------------------------------- pixel access */

static inline uint32_t ld32(const fgo_frame* F, int x, int y) {
    uint32_t w;
    memcpy(&w, F->p + (size_t)y * F->pitch + (size_t)x * 4, 4);
    return w;
}
static inline uint16_t ld16(const uint8_t* p, long pitch, int x, int y, int k, int cn) {
    uint16_t w;
    memcpy(&w, p + (size_t)y * pitch + ((size_t)x * cn + k) * 2, 2);
    return w;
}

/* channel k (0 R, 1 G, 2 B) of an Rgb10 pixel word */
static inline int rgb10(const fgo_fmt* f, uint32_t w, int k) {
    const int sh = f->rHigh ? 20 - 10 * k : 10 * k;
    return (int)((w >> sh) & 1023u);
}

/* the raw value of channel k at texel (x, y): Rgb10 code, F16 value, YUV: k = 0 the Y level, 1 / 2 Cb / Cr levels
 * of chroma texel (x, y) */
static inline float raw(const fgo_fmt* f, const fgo_frame* F, int x, int y, int k) {
    switch (f->format) {
    case FMT_RGB10: return (float)rgb10(f, ld32(F, x, y), k);
    case FMT_F16: return fgo_h2f(ld16(F->p, F->pitch, x, y, k, 4));
    case FMT_NV12:
        if (k == 0) return (float)F->p[(size_t)y * F->pitch + x];
        return (float)F->c[(size_t)y * F->cpitch + (size_t)x * 2 + (k - 1)];
    default:   /* P010 */
        if (k == 0) return (float)ld16(F->p, F->pitch, x, y, 0, 1) * 0x1p-8f;
        return (float)ld16(F->c, F->cpitch, x, y, k - 1, 2) * 0x1p-8f;
    }
}

/* a raw value -> the level the metric and the luma use (RGB formats) */
static inline float level(const fgo_fmt* f, float r) {
    if (f->format == FMT_RGB10) return r * f->k10;
    if (f->format == FMT_F16) return f->linear ? fgo_pq255(r, f->kWhite) : r * 255.0f;
    return r;
}

/* the estimate's luma of pixel (x, y) in quarter levels */
static int lumaQ(const fgo_fmt* f, const fgo_frame* F, int x, int y) {
    float yl;
    if (f->format == FMT_NV12 || f->format == FMT_P010) {
        yl = (raw(f, F, x, y, 0) - f->black) * f->ys;
    } else {
        const float r = level(f, raw(f, F, x, y, 0)), g = level(f, raw(f, F, x, y, 1)), b = level(f, raw(f, F, x, y, 2));
        float d = 4899.0f * r;
        d = d + 9617.0f * g;
        d = d + 1868.0f * b;
        yl = d * (1.0f / 16384.0f);
    }
    const float q = nearbyintf(clampf(yl, 0.0f, 255.0f) * 4.0f);
    return (int)q;
}

/* ---------------------------------------------------------------------------------------------- estimate */

/* CrosshairV2's estimate fill (gpu/shaders/ui_v2_lumafill.comp) for these formats: every level-0 cell of the mask
 * rectangle that holds a UI pixel takes the luma of its not-UI pixels, the window widened by fs px per step up to 8 px
 * while it has none, formed as the luma pass forms a cell (quarter levels summed, rne_div(4 sum, n) / 16). */
static void ui_fill_fmt(const fgo_fmt* f, const fgo_frame* F, int W, int H, const fgo_uimask* u, int fs, float* L0, int fw,
                        int fh) {
    if (!u || !u->m || u->w <= 0 || u->h <= 0) return;
    const int cx0 = u->x / fs, cx1 = (u->x + u->w - 1) / fs, cy0 = u->y / fs, cy1 = (u->y + u->h - 1) / fs;
    for (int cy = cy0; cy <= cy1 && cy < fh; cy++)
        for (int cx = cx0; cx <= cx1 && cx < fw; cx++) {
            const int px = cx * fs, py = cy * fs;
            int has = 0;
            for (int j = 0; j < fs && !has; j++)
                for (int i = 0; i < fs; i++)
                    if (px + i < W && py + j < H && ui_px(u, px + i, py + j)) { has = 1; break; }
            if (!has) continue;
            for (int k = 0; k <= 8; k += fs) {
                int sum = 0, n = 0;
                for (int y = py - k; y < py + fs + k; y++)
                    for (int x = px - k; x < px + fs + k; x++) {
                        if (x < 0 || y < 0 || x >= W || y >= H || ui_px(u, x, y)) continue;
                        sum += lumaQ(f, F, x, y);
                        n++;
                    }
                if (n > 0) {
                    L0[(size_t)cy * fw + cx] = (float)rne_div(4 * sum, n) * (1.0f / 16.0f);
                    break;
                }
            }
        }
}

int fgo_estimate_fmt_ui(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                        float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf, float* sad_mean,
                        int* cut, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc);
int fgo_estimate_fmt(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                     float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf, float* sad_mean,
                     int* cut, int nthreads) {
    return fgo_estimate_fmt_ui(A, C, W, H, f, s, luma, fields, seeds, meds, sads, pf, sad_mean, cut, nthreads, NULL, NULL);
}

/* the same with CrosshairV2's estimate fill of both frames' level 0 (ua, uc: their UI masks; none when either is NULL) */
int fgo_estimate_fmt_ui(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                        float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf, float* sad_mean,
                        int* cut, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int fw, fh, lw[MAXLV], lh[MAXLV];
    const int n = fgo_layout(W, H, s->flowScale, s->pyramidMinSide, &fw, &fh, lw, lh, MAXLV);
    if (n < 1) return -1;
    const int fs = s->flowScale;
    float* L[MAXLV][2];
    for (int l = 0; l < n; l++)
        for (int k = 0; k < 2; k++) L[l][k] = malloc(sizeof(float) * (size_t)lw[l] * lh[l]);
    for (int k = 0; k < 2; k++) {
        const fgo_frame* F = k ? C : A;
        float* out = L[0][k];
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < fh; y++)
            for (int x = 0; x < fw; x++) {
                int sum = 0, cnt = 0;
                for (int j = 0; j < fs; j++)
                    for (int i = 0; i < fs; i++) {
                        const int yy = y * fs + j, xx = x * fs + i;
                        if (yy < H && xx < W) { sum += lumaQ(f, F, xx, yy); cnt++; }
                    }
                out[(size_t)y * fw + x] = (float)rne_div(4 * sum, cnt) * (1.0f / 16.0f);
            }
    }
    if (ua && uc) {
        ui_fill_fmt(f, A, W, H, ua, fs, L[0][0], fw, fh);
        ui_fill_fmt(f, C, W, H, uc, fs, L[0][1], fw, fh);
    }
    for (int l = 1; l < n; l++)
        for (int k = 0; k < 2; k++) fgo_i_area_half(L[l - 1][k], lw[l - 1], lh[l - 1], L[l][k], lw[l], lh[l], 1);
    const int r = fgo_i_estimate_levels(L, n, lw, lh, s, -1, NULL, luma, fields, seeds, meds, sads, pf, sad_mean, cut);
    for (int l = 0; l < n; l++) { free(L[l][0]); free(L[l][1]); }
    return r;
}

/* ---------------------------------------------------------------------------------------------- synth */

/* bilinear taps of one sample: texel corners and cv2's float weights */
typedef struct { int x0, x1, y0, y1; float w00, w01, w10, w11; } taps;

/* X, Y: the sample point in units of 1/2^bits texel (the fraction has `bits` bits) */
static taps mktaps(int X, int Y, int bits, int w, int h) {
    taps t;
    const int ix = X >> bits, iy = Y >> bits, mask = (1 << bits) - 1;
    const float sc = 1.0f / (float)(1 << bits);
    const float fx = (float)(X & mask) * sc, fy = (float)(Y & mask) * sc;
    t.w00 = (1.0f - fy) * (1.0f - fx);
    t.w01 = (1.0f - fy) * fx;
    t.w10 = fy * (1.0f - fx);
    t.w11 = fy * fx;
    t.x0 = clampi(ix, 0, w - 1); t.x1 = clampi(ix + 1, 0, w - 1);
    t.y0 = clampi(iy, 0, h - 1); t.y1 = clampi(iy + 1, 0, h - 1);
    return t;
}

static inline float tapv(const fgo_fmt* f, const fgo_frame* F, const taps* t, int k) {
    float r = raw(f, F, t->x0, t->y0, k) * t->w00;
    r = r + raw(f, F, t->x1, t->y0, k) * t->w01;
    r = r + raw(f, F, t->x0, t->y1, k) * t->w10;
    r = r + raw(f, F, t->x1, t->y1, k) * t->w11;
    return r;
}

/* the warped sample at (px, py): out[0..2] = RGB levels (Rgb10), F16 values, or (Y, Cb, Cr) levels */
static void warp(const fgo_fmt* f, const fgo_frame* F, int W, int H, float px, float py, float out[3]) {
    const int X = (int)nearbyintf(px * 32.0f), Y = (int)nearbyintf(py * 32.0f);
    const taps t = mktaps(X, Y, 5, W, H);
    if (f->format == FMT_NV12 || f->format == FMT_P010) {
        out[0] = tapv(f, F, &t, 0);
        const taps tc = mktaps(X - 16, Y - 16, 6, (W + 1) / 2, (H + 1) / 2);
        out[1] = tapv(f, F, &tc, 1);
        out[2] = tapv(f, F, &tc, 2);
    } else {
        for (int k = 0; k < 3; k++) {
            const float r = tapv(f, F, &t, k);
            out[k] = f->format == FMT_RGB10 ? r * f->k10 : r;
        }
    }
}

/* the chroma of a YUV frame warped to (px, py) (block-centre coordinates) */
static void warpC(const fgo_fmt* f, const fgo_frame* F, int W, int H, float px, float py, float out[2]) {
    const int X = (int)nearbyintf(px * 32.0f), Y = (int)nearbyintf(py * 32.0f);
    const taps tc = mktaps(X - 16, Y - 16, 6, (W + 1) / 2, (H + 1) / 2);
    out[0] = tapv(f, F, &tc, 1);
    out[1] = tapv(f, F, &tc, 2);
}

static int mismatch(const fgo_fmt* f, const float wa[3], const float wc[3]) {
    float m;
    if (f->format == FMT_NV12 || f->format == FMT_P010) {
        const float dy = wa[0] - wc[0], db = wa[1] - wc[1], dr = wa[2] - wc[2];
        const float y = f->ys * dy;
        const float r = y + f->rcr * dr;
        float g = y + f->gcb * db;
        g = g + f->gcr * dr;
        const float b = y + f->bcb * db;
        m = absf(r);
        if (absf(g) > m) m = absf(g);
        if (absf(b) > m) m = absf(b);
    } else {
        m = 0.0f;
        for (int k = 0; k < 3; k++) {
            float d;
            if (f->format == FMT_F16 && f->linear) d = absf(fgo_pq255(wa[k], f->kWhite) - fgo_pq255(wc[k], f->kWhite));
            else if (f->format == FMT_F16) d = absf(wa[k] * 255.0f - wc[k] * 255.0f);
            else d = absf(wa[k] - wc[k]);
            if (d > m) m = d;
        }
    }
    if (m > 255.0f) m = 255.0f;
    return (int)m;
}

static inline float blend(float a, float c, float n, float u, float iu, int mid, float wA, float wC) {
    float m;
    if (mid) m = 0.5f * (a + c);
    else { const float p = wA * a, q = wC * c; m = p + q; }
    const float p1 = m * iu, p2 = n * u;
    return p1 + p2;
}

static void copy_near(const fgo_fmt* f, const fgo_frame* N, const fgo_frame* O, int W, int H) {
    const int bpp = f->format == FMT_F16 ? 8 : (f->format == FMT_NV12 ? 1 : (f->format == FMT_P010 ? 2 : 4));
    for (int y = 0; y < H; y++) memcpy((uint8_t*)O->p + (size_t)y * O->pitch, N->p + (size_t)y * N->pitch, (size_t)W * bpp);
    if (f->format == FMT_NV12 || f->format == FMT_P010) {
        const int cw = (W + 1) / 2, ch = (H + 1) / 2;
        for (int y = 0; y < ch; y++)
            memcpy((uint8_t*)O->c + (size_t)y * O->cpitch, N->c + (size_t)y * N->cpitch, (size_t)cw * 2 * bpp);
    }
}

/* interp.synth for the other formats; arguments as fgo_synth, frames as fgo_frame (O: the output planes) */
/* The pixels a YUV sample at p reads with a non-zero weight (gpu/shaders/ui_reject.glsl uiFootprint, FG_YUV): the 2x2
 * texels of the half-resolution chroma plane around it, c = roundEven(32 p) - 16 in 1/64 chroma texels, i = c >> 6,
 * the second texel only if the fraction is not 0: pixels 2 i .. 2 (i + n) + 1 per axis (they contain the luma taps) */
static int ui_hit_yuv(const fgo_uimask* u, float px, float py) {
    if (!u || !u->m || u->w <= 0 || u->h <= 0) return 0;
    const int cx = (int)nearbyintf(px * 32.0f) - 16, cy = (int)nearbyintf(py * 32.0f) - 16;
    const int ix = cx >> 6, iy = cy >> 6;
    int x0 = 2 * ix - u->x, y0 = 2 * iy - u->y;
    int x1 = 2 * (ix + ((cx & 63) != 0)) + 1 - u->x, y1 = 2 * (iy + ((cy & 63) != 0)) + 1 - u->y;
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 > u->w - 1) x1 = u->w - 1;
    if (y1 > u->h - 1) y1 = u->h - 1;
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++)
            if (u->m[(size_t)y * u->stride + x]) return 1;
    return 0;
}

/* CrosshairV2's warp-tap rejection (gpu/shaders/ui_reject.glsl uiReject / uiRejectC): a tap whose footprint touches
 * its own frame's UI mask takes the other frame's tap (both or neither: unchanged); n values (3, or YUV chroma: 2) */
static inline void ui_reject(const fgo_fmt* f, const fgo_uimask* ua, const fgo_uimask* uc, float pax, float pay,
                             float pcx, float pcy, float* wa, float* wc, int n) {
    if (!ua && !uc) return;
    const int yuv = f->format == FMT_NV12 || f->format == FMT_P010;
    const int ha = yuv ? ui_hit_yuv(ua, pax, pay) : ui_hit(ua, pax, pay);
    const int hc = yuv ? ui_hit_yuv(uc, pcx, pcy) : ui_hit(uc, pcx, pcy);
    if (ha == hc) return;
    for (int k = 0; k < n; k++) {
        if (ha) wa[k] = wc[k];
        else wc[k] = wa[k];
    }
}

int fgo_synth_fmt_ui(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                     const float* pf, int cut, float t, const fgo_frame* O, float* field_t, uint8_t* emap,
                     long long* untrusted, int* reason, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc);
int fgo_synth_fmt(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                  const float* pf, int cut, float t, const fgo_frame* O, float* field_t, uint8_t* emap,
                  long long* untrusted, int* reason, int nthreads) {
    return fgo_synth_fmt_ui(A, C, W, H, f, s, pf, cut, t, O, field_t, emap, untrusted, reason, nthreads, NULL, NULL);
}

/* the same with CrosshairV2's warp-tap rejection (ua, uc: prev's and curr's UI masks, either may be NULL; RGB formats
 * only) */
int fgo_synth_fmt_ui(const fgo_frame* A, const fgo_frame* C, int W, int H, const fgo_fmt* f, const fgo_settings* s,
                     const float* pf, int cut, float t, const fgo_frame* O, float* field_t, uint8_t* emap,
                     long long* untrusted, int* reason, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (!(t > 0.0f && t < 1.0f)) return -1;
    const fgo_frame* N = t <= 0.5f ? A : C;
    if (untrusted) *untrusted = 0;
    if (cut) {
        copy_near(f, N, O, W, H);
        *reason = 1;
        return 0;
    }
    const int fs = s->flowScale;
    const int fw = (int)nearbyint(W * (1.0 / fs)), fh = (int)nearbyint(H * (1.0 / fs));
    const double td = t;
    const float sf = (float)(2.0 * td - 1.0);
    float* g = malloc(sizeof(float) * (size_t)fw * fh * 2);
    if (sf == 0.0f) memcpy(g, pf, sizeof(float) * (size_t)fw * fh * 2);
    else fgo_i_field_at(pf, fw, fh, sf, g);
    if (field_t) memcpy(field_t, g, sizeof(float) * (size_t)fw * fh * 2);
    const int uw = fw * fs, uh = fh * fs;
    float* hv = malloc(sizeof(float) * (size_t)uw * uh * 2);
    fgo_i_resize_lin2(g, fw, fh, hv, uw, uh);
    free(g);
    const float ka = (float)(2.0 * td), kc = (float)(2.0 * (1.0 - td));
    const float wA = (float)(1.0 - td), wC = t;
    const int mid = t == 0.5f;
    uint8_t* e = malloc((size_t)W * H);
    float* ef = malloc(sizeof(float) * (size_t)W * H);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const int sy = y < uh ? y : uh - 1, sx = x < uw ? x : uw - 1;
            const float hx = hv[((size_t)sy * uw + sx) * 2] * (float)fs, hy = hv[((size_t)sy * uw + sx) * 2 + 1] * (float)fs;
            float wa[3], wc[3];
            warp(f, A, W, H, (float)x - ka * hx, (float)y - ka * hy, wa);
            warp(f, C, W, H, (float)x + kc * hx, (float)y + kc * hy, wc);
            ui_reject(f, ua, uc, (float)x - ka * hx, (float)y - ka * hy, (float)x + kc * hx, (float)y + kc * hy, wa, wc, 3);
            const int m = mismatch(f, wa, wc);
            e[(size_t)y * W + x] = (uint8_t)m;
            ef[(size_t)y * W + x] = (float)m;
        }
    if (emap) memcpy(emap, e, (size_t)W * H);
    float* eb = malloc(sizeof(float) * (size_t)W * H);
    fgo_i_box_blur(ef, W, H, 7, eb);
    const float t0 = s->trustLow, span = (float)((double)s->trustHigh - (double)s->trustLow);
    long long cnt = 0;
    #pragma omp parallel for schedule(static) reduction(+ : cnt)
    for (size_t q = 0; q < (size_t)W * H; q++) {
        float u = (eb[q] - t0) / span;
        u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
        eb[q] = u;
        cnt += u > 0.5f;
    }
    if (untrusted) *untrusted = cnt;
    if ((double)cnt / ((double)W * (double)H) > (double)s->globalFallback) {
        copy_near(f, N, O, W, H);
        *reason = 2;
    } else {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const size_t q = (size_t)y * W + x;
                const int sy = y < uh ? y : uh - 1, sx = x < uw ? x : uw - 1;
                const float hx = hv[((size_t)sy * uw + sx) * 2] * (float)fs, hy = hv[((size_t)sy * uw + sx) * 2 + 1] * (float)fs;
                float wa[3], wc[3];
                warp(f, A, W, H, (float)x - ka * hx, (float)y - ka * hy, wa);
                warp(f, C, W, H, (float)x + kc * hx, (float)y + kc * hy, wc);
                ui_reject(f, ua, uc, (float)x - ka * hx, (float)y - ka * hy, (float)x + kc * hx, (float)y + kc * hy, wa, wc, 3);
                const float u = eb[q], iu = 1.0f - u;
                uint8_t* o = (uint8_t*)O->p + (size_t)y * O->pitch;
                if (f->format == FMT_RGB10) {
                    const uint32_t nw = ld32(N, x, y);
                    uint32_t ow = nw & 0xC0000000u;
                    for (int k = 0; k < 3; k++) {
                        const float nl = (float)rgb10(f, nw, k) * f->k10;
                        const float v = clampf(blend(wa[k], wc[k], nl, u, iu, mid, wA, wC), 0.0f, 255.0f);
                        const float sc = v * f->k10i;
                        int code = (int)floorf(sc + 0.5f);
                        code = clampi(code, 0, 1023);
                        ow |= (uint32_t)code << (f->rHigh ? 20 - 10 * k : 10 * k);
                    }
                    memcpy(o + (size_t)x * 4, &ow, 4);
                } else if (f->format == FMT_F16) {
                    uint16_t hs[4];
                    for (int k = 0; k < 3; k++) {
                        const float nv = fgo_h2f(ld16(N->p, N->pitch, x, y, k, 4));
                        hs[k] = fgo_f2h(blend(wa[k], wc[k], nv, u, iu, mid, wA, wC));
                    }
                    hs[3] = ld16(N->p, N->pitch, x, y, 3, 4);
                    memcpy(o + (size_t)x * 8, hs, 8);
                } else {
                    const float ql = f->format == FMT_P010 ? 4.0f : 1.0f;   /* 1 / YU_QL */
                    const int codes = f->format == FMT_P010 ? 1023 : 255;
                    const float ny = raw(f, N, x, y, 0);
                    const float v = blend(wa[0], wc[0], ny, u, iu, mid, wA, wC);
                    const int code = clampi((int)floorf(v * ql + 0.5f), 0, codes);
                    if (f->format == FMT_P010) { const uint16_t w16 = (uint16_t)(code << 6); memcpy(o + (size_t)x * 2, &w16, 2); }
                    else o[x] = (uint8_t)code;
                    if (((x | y) & 1) == 0) {
                        float ca[2], cc[2];
                        const float bx = (float)x + 0.5f, by = (float)y + 0.5f;
                        warpC(f, A, W, H, bx - ka * hx, by - ka * hy, ca);
                        warpC(f, C, W, H, bx + kc * hx, by + kc * hy, cc);
                        ui_reject(f, ua, uc, bx - ka * hx, by - ka * hy, bx + kc * hx, by + kc * hy, ca, cc, 2);
                        uint8_t* oc = (uint8_t*)O->c + (size_t)(y / 2) * O->cpitch;
                        for (int k = 0; k < 2; k++) {
                            const float nc = raw(f, N, x / 2, y / 2, 1 + k);
                            const float vc = blend(ca[k], cc[k], nc, u, iu, mid, wA, wC);
                            const int cd = clampi((int)floorf(vc * ql + 0.5f), 0, codes);
                            if (f->format == FMT_P010) { const uint16_t w16 = (uint16_t)(cd << 6); memcpy(oc + ((size_t)(x / 2) * 2 + k) * 2, &w16, 2); }
                            else oc[(size_t)(x / 2) * 2 + k] = (uint8_t)cd;
                        }
                    }
                }
            }
        *reason = 0;
    }
    free(hv); free(e); free(ef); free(eb);
    return 0;
}
