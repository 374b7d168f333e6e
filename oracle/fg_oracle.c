/*
 * fg_oracle.c -- CPU restatement of frame-gen-ritz's MotionVersion::V1 interpolation (proto/interp.py).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA path and the timed CPU baseline of bench.py.
 * Nothing in the product (the CUDA library, its C ABI, its host code) includes, links or calls it.
 *
 * What is restated, and from where:
 *   - the algorithm of proto/interp.py (flow :147-164, search :116-124, block_sad :97-103, pick :106-113,
 *     seed_from :131-144, median3 :127-128, pyramid :73-77, pad_to_block :68-70, pixel_field :167-183,
 *     estimate :186-191, field_at :194-205, warp_t :208-216, synth :219-246);
 *   - the OpenCV primitives it calls, as the installed opencv-python-headless 4.13.0.92 computes them (each was
 *     checked against cv2 on random inputs, see tests/golden/gen_golden.py):
 *       cvtColor BGR2GRAY 8u : (B*3735 + G*19235 + R*9798 + 16384) >> 15   (all 2^24 colours)
 *       resize INTER_AREA 1/k: mean of the valid pixels of each k x k cell (sum*1/k^2 if full, sum/count at edges),
 *                              output size rint-half-even(size/k)
 *       resize INTER_LINEAR  : fx = (float)((dx+0.5)*scale-0.5); x taps clamped with weights (1,0) at the borders,
 *                              y rows clamped but weights NOT clamped; h = S0*a0 + S1*a1, v = R0*b0 + R1*b1 (no FMA)
 *       remap INTER_LINEAR, BORDER_REPLICATE: X = rint-half-even(x*32); taps at X>>5, +1 clamped per tap;
 *                              float images: ((p00*w00 + p01*w01) + p10*w10) + p11*w11, w from (1-f) and f in 1/32;
 *                              uint8 images: integer weights (32-fx)(32-fy)*32 ..., (sum + 2^14) >> 15
 *       blur (box, normalised, BORDER_REPLICATE) on float32: the window sum in double, times 1.0/(k*k), to float
 *       medianBlur 3 on float32: the exact per-channel median of the 3x3 replicate-bordered window
 *   - numpy's float32 mean (used for the scene-cut SAD mean): pairwise summation from 0 (8 accumulators for
 *     blocks of <= 128 elements, recursive halving rounded down to a multiple of 8 above that), then a float32
 *     division by the count.
 * All float arithmetic is IEEE binary32/binary64 with round-to-nearest and no contraction (-ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fg_oracle_internal.h"

/* pixel layout of an 8-bit frame: 0 = R,G,B,A; 1 = B,G,R,A; 2 = B,G,R (interp.py's own, 3 bytes per pixel) */
typedef struct img8 {
    const uint8_t* p;
    int W, H, pitch, cn, ri, gi, bi;
} img8;

static img8 mkimg(const uint8_t* p, int W, int H, int pitch, int order) {
    img8 m;
    m.p = p; m.W = W; m.H = H; m.pitch = pitch;
    m.cn = order == 2 ? 3 : 4;
    m.ri = order == 0 ? 0 : 2; m.gi = 1; m.bi = order == 0 ? 2 : 0;
    return m;
}

static int rint_he(double v) { return (int)nearbyint(v); }   /* cv2 saturate_cast<int>(double): round half to even */
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float absf(float v) { return v < 0.0f ? -v : v; }

/* ---------------------------------------------------------------------------------------------- layout */

/* interp.flow / interp.pyramid: flow size rint(W/fs) and the pyramid level sizes (stop when min//2 < minSide).
 * Returns the number of levels. */
int fgo_layout(int W, int H, int fs, int minSide, int* fw, int* fh, int* lw, int* lh, int maxLevels) {
    int w = rint_he(W * (1.0 / fs)), h = rint_he(H * (1.0 / fs));
    *fw = w; *fh = h;
    int n = 0;
    for (;;) {
        if (n >= maxLevels) return -1;
        lw[n] = w; lh[n] = h; n++;
        if ((w < h ? w : h) / 2 < minSide) break;
        w = rint_he(w * 0.5);
        h = rint_he(h * 0.5);
    }
    return n;
}

/* ---------------------------------------------------------------------------------------------- luma */

static inline int gray8(const img8* m, int x, int y) {   /* cv2 BGR2GRAY, 8u, 4.13 */
    const uint8_t* q = m->p + (size_t)y * m->pitch + (size_t)x * m->cn;
    return (q[m->bi] * 3735 + q[m->gi] * 19235 + q[m->ri] * 9798 + 16384) >> 15;
}

/* interp.flow :149-151: luma then INTER_AREA 1/fs (fs = 1: the luma itself) */
static void luma_area(const img8* m, int fs, float* out, int fw, int fh) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < fh; y++)
        for (int x = 0; x < fw; x++) {
            if (fs == 1) { out[(size_t)y * fw + x] = (float)gray8(m, x, y); continue; }
            int sum = 0, n = 0;
            for (int j = 0; j < fs; j++)
                for (int i = 0; i < fs; i++) {
                    int yy = y * fs + j, xx = x * fs + i;
                    if (yy < m->H && xx < m->W) { sum += gray8(m, xx, yy); n++; }
                }
            out[(size_t)y * fw + x] = n == fs * fs ? (float)sum * (1.0f / (float)(fs * fs)) : (float)sum / (float)n;
        }
}

/* interp.pyramid :76: INTER_AREA 0.5 of a float level (round10: then rounded half-even to a multiple of 2^-10, the
 * grid the restatement of the other frame formats keeps its coarse levels on) */
void fgo_i_area_half(const float* src, int sw, int sh, float* dst, int dw, int dh, int round10) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < dh; y++)
        for (int x = 0; x < dw; x++) {
            float s = 0.0f;
            int n = 0;
            for (int j = 0; j < 2; j++)
                for (int i = 0; i < 2; i++) {
                    int yy = 2 * y + j, xx = 2 * x + i;
                    if (yy < sh && xx < sw) { s += src[(size_t)yy * sw + xx]; n++; }
                }
            float v = n == 4 ? s * 0.25f : s / (float)n;
            if (round10) v = nearbyintf(v * 1024.0f) * (1.0f / 1024.0f);
            dst[(size_t)y * dw + x] = v;
        }
}

/* ---------------------------------------------------------------------------------------------- cv2 remap */

/* one cv2.remap INTER_LINEAR / BORDER_REPLICATE sample of a float plane (stride `cs` floats between pixels) */
float fgo_i_remap_f(const float* img, int w, int h, int cs, float x, float y) {
    int X = (int)nearbyintf(x * 32.0f), Y = (int)nearbyintf(y * 32.0f);
    int ix = X >> 5, iy = Y >> 5;
    float fx = (float)(X & 31) * (1.0f / 32.0f), fy = (float)(Y & 31) * (1.0f / 32.0f);
    float w00 = (1.0f - fy) * (1.0f - fx), w01 = (1.0f - fy) * fx, w10 = fy * (1.0f - fx), w11 = fy * fx;
    int x0 = clampi(ix, 0, w - 1), x1 = clampi(ix + 1, 0, w - 1), y0 = clampi(iy, 0, h - 1), y1 = clampi(iy + 1, 0, h - 1);
    float p00 = img[((size_t)y0 * w + x0) * cs], p01 = img[((size_t)y0 * w + x1) * cs];
    float p10 = img[((size_t)y1 * w + x0) * cs], p11 = img[((size_t)y1 * w + x1) * cs];
    float r = p00 * w00;
    r = r + p01 * w01;
    r = r + p10 * w10;
    r = r + p11 * w11;
    return r;
}

/* one cv2.remap INTER_LINEAR / BORDER_REPLICATE sample of an 8-bit frame: all channels */
static inline void remap_u8(const img8* m, float x, float y, int out[4]) {
    int X = (int)nearbyintf(x * 32.0f), Y = (int)nearbyintf(y * 32.0f);
    int ix = X >> 5, iy = Y >> 5, fx = X & 31, fy = Y & 31;
    int w00 = (32 - fy) * (32 - fx) * 32, w01 = (32 - fy) * fx * 32, w10 = fy * (32 - fx) * 32, w11 = fy * fx * 32;
    int x0 = clampi(ix, 0, m->W - 1), x1 = clampi(ix + 1, 0, m->W - 1), y0 = clampi(iy, 0, m->H - 1), y1 = clampi(iy + 1, 0, m->H - 1);
    const uint8_t *q00 = m->p + (size_t)y0 * m->pitch + (size_t)x0 * m->cn, *q01 = m->p + (size_t)y0 * m->pitch + (size_t)x1 * m->cn;
    const uint8_t *q10 = m->p + (size_t)y1 * m->pitch + (size_t)x0 * m->cn, *q11 = m->p + (size_t)y1 * m->pitch + (size_t)x1 * m->cn;
    for (int k = 0; k < m->cn; k++)
        out[k] = (q00[k] * w00 + q01[k] * w01 + q10[k] * w10 + q11[k] * w11 + (1 << 14)) >> 15;
}

/* ---------------------------------------------------------------------------------------------- cv2 resize linear */

typedef struct { int* i0; int* i1; float* a0; float* a1; } lincoef;

/* cv2 resize INTER_LINEAR coefficients along one axis; clampw: x rule (weights forced to (1,0) at the borders) */
static lincoef lin_coeffs(int n_dst, int n_src, int clampw) {
    lincoef c;
    c.i0 = malloc(sizeof(int) * n_dst); c.i1 = malloc(sizeof(int) * n_dst);
    c.a0 = malloc(sizeof(float) * n_dst); c.a1 = malloc(sizeof(float) * n_dst);
    double scale = 1.0 / ((double)n_dst / (double)n_src);
    for (int d = 0; d < n_dst; d++) {
        float f = (float)((d + 0.5) * scale - 0.5);
        int s = (int)floorf(f);
        f -= (float)s;
        if (clampw) {
            if (s < 0) { s = 0; f = 0.0f; }
            if (s >= n_src - 1) { s = n_src - 1; f = 0.0f; }
        }
        c.i0[d] = clampi(s, 0, n_src - 1);
        c.i1[d] = clampi(s + 1, 0, n_src - 1);
        c.a0[d] = 1.0f - f;
        c.a1[d] = f;
    }
    return c;
}
static void lin_free(lincoef c) { free(c.i0); free(c.i1); free(c.a0); free(c.a1); }

/* cv2.resize(src (sh x sw x 2 float), (dw, dh), INTER_LINEAR) */
void fgo_i_resize_lin2(const float* src, int sw, int sh, float* dst, int dw, int dh) {
    lincoef cx = lin_coeffs(dw, sw, 1), cy = lin_coeffs(dh, sh, 0);
    float* rows = malloc(sizeof(float) * (size_t)sh * dw * 2);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < sh; y++)
        for (int x = 0; x < dw; x++)
            for (int k = 0; k < 2; k++) {
                float p0 = src[((size_t)y * sw + cx.i0[x]) * 2 + k], p1 = src[((size_t)y * sw + cx.i1[x]) * 2 + k];
                float t0 = p0 * cx.a0[x], t1 = p1 * cx.a1[x];
                rows[((size_t)y * dw + x) * 2 + k] = t0 + t1;
            }
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < dh; y++)
        for (int x = 0; x < dw * 2; x++) {
            float r0 = rows[(size_t)cy.i0[y] * dw * 2 + x], r1 = rows[(size_t)cy.i1[y] * dw * 2 + x];
            float t0 = r0 * cy.a0[y], t1 = r1 * cy.a1[y];
            dst[(size_t)y * dw * 2 + x] = t0 + t1;
        }
    free(rows);
    lin_free(cx); lin_free(cy);
}

/* ---------------------------------------------------------------------------------------------- numpy pairwise */

/* numpy's pairwise float32 summation of a contiguous array (the reduction interp's sad.mean() runs) */
static float pairwise_f32(const float* a, long n) {
    if (n < 8) {
        float r = 0.0f;
        for (long i = 0; i < n; i++) r += a[i];
        return r;
    }
    if (n <= 128) {
        float r[8];
        for (int j = 0; j < 8; j++) r[j] = a[j];
        long i;
        for (i = 8; i < n - (n % 8); i += 8)
            for (int j = 0; j < 8; j++) r[j] += a[i + j];
        float res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; i++) res += a[i];
        return res;
    }
    long n2 = n / 2;
    n2 -= n2 % 8;
    return pairwise_f32(a, n2) + pairwise_f32(a + n2, n - n2);
}

float fgo_mean_f32(const float* a, long n) { return pairwise_f32(a, n) / (float)n; }

/* ---------------------------------------------------------------------------------------------- search */

/* interp.block_sad for one block at (bx, by) with half-vector (vx, vy): mean |a(q - v) - c(q + v)| over its 8x8.
 * The level is addressed unpadded with clamped taps (pad_to_block's replicate border then remap's replicate
 * border give the same texels). */
static float block_sad1(const float* la, const float* lc, int w, int h, int bx, int by, float vx, float vy) {
    double sum = 0.0;
    for (int y = 0; y < BLOCK; y++)
        for (int x = 0; x < BLOCK; x++) {
            float gx = (float)(bx * BLOCK + x), gy = (float)(by * BLOCK + y);
            float a = fgo_i_remap_f(la, w, h, 1, gx - vx, gy - vy);
            float c = fgo_i_remap_f(lc, w, h, 1, gx + vx, gy + vy);
            sum += (double)absf(a - c);
        }
    return (float)sum / 64.0f;
}

/* interp.search: every offset (dx, dy) * step within +-radius of each block's seed; cost = SAD + penalty; the
 * first minimum in (dy, dx) raster order wins. Writes the chosen vectors and their SADs. */
static void search(const float* la, const float* lc, int w, int h, int bw, int bh, const float* seed, int radius,
                   float step, float lambda, float* vout, float* sadout) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < bw * bh; b++) {
        int bx = b % bw, by = b / bw;
        float best = 0.0f, bs = 0.0f, bvx = 0.0f, bvy = 0.0f;
        int first = 1;
        for (int dy = -radius; dy <= radius; dy++)
            for (int dx = -radius; dx <= radius; dx++) {
                float vx = seed[2 * b] + (float)(dx * (double)step), vy = seed[2 * b + 1] + (float)(dy * (double)step);
                float s = block_sad1(la, lc, w, h, bx, by, vx, vy);
                float pen = (float)((double)lambda * (double)step * (double)(abs(dx) + abs(dy)));
                float cost = s + pen;
                if (first || cost < best) { best = cost; bs = s; bvx = vx; bvy = vy; first = 0; }
            }
        vout[2 * b] = bvx; vout[2 * b + 1] = bvy;
        if (sadout) sadout[b] = bs;
    }
}

static int cmpf(const void* x, const void* y) {
    float a = *(const float*)x, b = *(const float*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* interp.median3: per-component cv2.medianBlur(., 3), replicate border */
static void median3(const float* v, int bw, int bh, float* out) {
    #pragma omp parallel for schedule(static)
    for (int b = 0; b < bw * bh; b++) {
        int bx = b % bw, by = b / bw;
        for (int k = 0; k < 2; k++) {
            float t[9];
            int n = 0;
            for (int j = -1; j <= 1; j++)
                for (int i = -1; i <= 1; i++)
                    t[n++] = v[2 * (clampi(by + j, 0, bh - 1) * bw + clampi(bx + i, 0, bw - 1)) + k];
            qsort(t, 9, sizeof(float), cmpf);
            out[2 * b + k] = t[4];
        }
    }
}

/* np.median of n float32 values (partition; the mean of the two middle ones in float32 for even n) */
static float np_median(float* t, int n) {
    qsort(t, n, sizeof(float), cmpf);
    if (n % 2) return t[n / 2];
    float s = 0.0f;
    s += t[n / 2 - 1];
    s += t[n / 2];
    return s / 2.0f;
}

/* interp.seed_from: the fine level's seeds from the parent field v (pw x ph). med receives 2 x the global median. */
static void seed_from(const float* v, int pw, int ph, const float* la, const float* lc, int w, int h, int bw, int bh,
                      float lambda, float* seed, float med[2]) {
    int n = bw * bh;
    float* own = malloc(sizeof(float) * 2 * n);
    float* tmp = malloc(sizeof(float) * n);
    for (int b = 0; b < n; b++) {
        int ix = b % bw, iy = b / bw;
        int px = ix / 2 < pw - 1 ? ix / 2 : pw - 1, py = iy / 2 < ph - 1 ? iy / 2 : ph - 1;
        own[2 * b] = v[2 * (py * pw + px)] * 2.0f;
        own[2 * b + 1] = v[2 * (py * pw + px) + 1] * 2.0f;
    }
    for (int k = 0; k < 2; k++) {
        for (int b = 0; b < n; b++) tmp[b] = own[2 * b + k];
        med[k] = np_median(tmp, n);
    }
    float lam = lambda;
    #pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < n; b++) {
        int ix = b % bw, iy = b / bw;
        int px = ix / 2 < pw - 1 ? ix / 2 : pw - 1, py = iy / 2 < ph - 1 ? iy / 2 : ph - 1;
        int sy = iy % 2 == 0 ? -1 : 1, sx = ix % 2 == 0 ? -1 : 1;
        int oy[4] = {0, sy, 0, sy}, ox[4] = {0, 0, sx, sx};
        float cx[6], cy[6];
        for (int k = 0; k < 4; k++) {
            int qy = clampi(py + oy[k], 0, ph - 1), qx = clampi(px + ox[k], 0, pw - 1);
            cx[k] = v[2 * (qy * pw + qx)] * 2.0f;
            cy[k] = v[2 * (qy * pw + qx) + 1] * 2.0f;
        }
        cx[4] = 0.0f; cy[4] = 0.0f;
        cx[5] = med[0]; cy[5] = med[1];
        float best = 0.0f, sx_ = 0.0f, sy_ = 0.0f;
        for (int k = 0; k < 6; k++) {
            float s = block_sad1(la, lc, w, h, ix, iy, cx[k], cy[k]);
            float cost = k == 0 ? s + 0.0f : s + lam;
            if (k == 0 || cost < best) { best = cost; sx_ = cx[k]; sy_ = cy[k]; }
        }
        seed[2 * b] = sx_; seed[2 * b + 1] = sy_;
    }
    free(own); free(tmp);
}

/* The seeds of the level the seed net reads (no counterpart in interp.py): per block the net's two candidates
 * (rounded half-even after clamping to +-256) and zero, scored like seed_from's candidates (block SAD + lambda), the
 * first free of lambda when the net's confidence logit is >= 0; the first minimum wins. cnn: bw*bh x 8 floats. */
static void seed_cnn(const float* cnn, const float* la, const float* lc, int w, int h, int bw, int bh, float lambda,
                     float* seed) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < bw * bh; b++) {
        const float* o = cnn + (size_t)b * 8;
        float cx[3], cy[3];
        for (int k = 0; k < 2; k++) {
            cx[k] = nearbyintf(fminf(fmaxf(o[2 * k], -256.0f), 256.0f));
            cy[k] = nearbyintf(fminf(fmaxf(o[2 * k + 1], -256.0f), 256.0f));
        }
        cx[2] = 0.0f; cy[2] = 0.0f;
        const int free0 = o[4] >= 0.0f;
        float best = 0.0f, sx = 0.0f, sy = 0.0f;
        for (int k = 0; k < 3; k++) {
            float sd = block_sad1(la, lc, w, h, b % bw, b / bw, cx[k], cy[k]);
            float cost = (k == 0 && free0) ? sd + 0.0f : sd + lambda;
            if (k == 0 || cost < best) { best = cost; sx = cx[k]; sy = cy[k]; }
        }
        seed[2 * b] = sx; seed[2 * b + 1] = sy;
    }
}

/* ---------------------------------------------------------------------------------------------- pixel field */

/* cv2.blur(err, (k, k), BORDER_REPLICATE) of a float plane: the window sum in double times 1/(k*k), to float */
void fgo_i_box_blur(const float* src, int w, int h, int k, float* dst) {
    int r = k / 2;
    double* hs = malloc(sizeof(double) * (size_t)w * h);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            double s = 0.0;
            for (int i = -r; i <= r; i++) s += (double)src[(size_t)y * w + clampi(x + i, 0, w - 1)];
            hs[(size_t)y * w + x] = s;
        }
    double sc = 1.0 / (double)(k * k);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            double s = 0.0;
            for (int j = -r; j <= r; j++) s += hs[(size_t)clampi(y + j, 0, h - 1) * w + x];
            dst[(size_t)y * w + x] = (float)(s * sc);
        }
    free(hs);
}

/* interp.pixel_field: per flow pixel, 7 candidates, each scored by the 5x5 box of its own error image */
static void pixel_field(const float* v, int bw, int bh, const float* ya, const float* yc, int w, int h,
                        float smooth, float zero, float* pf) {
    size_t np_ = (size_t)w * h;
    float* bil = malloc(sizeof(float) * (size_t)bw * BLOCK * bh * BLOCK * 2);
    fgo_i_resize_lin2(v, bw, bh, bil, bw * BLOCK, bh * BLOCK);
    float* cand = malloc(sizeof(float) * np_ * 2 * 7);
    float* err = malloc(sizeof(float) * np_);
    float* cost = malloc(sizeof(float) * np_ * 7);
    int oy[4] = {-1, 1, 0, 0}, ox[4] = {0, 0, -1, 1};
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            size_t q = (size_t)y * w + x;
            int bx = x / BLOCK, by = y / BLOCK;
            float* cq = cand + q * 14;
            cq[0] = bil[((size_t)y * bw * BLOCK + x) * 2];
            cq[1] = bil[((size_t)y * bw * BLOCK + x) * 2 + 1];
            cq[2] = v[2 * (by * bw + bx)];
            cq[3] = v[2 * (by * bw + bx) + 1];
            for (int k = 0; k < 4; k++) {
                int qy = clampi(by + oy[k], 0, bh - 1), qx = clampi(bx + ox[k], 0, bw - 1);
                cq[4 + 2 * k] = v[2 * (qy * bw + qx)];
                cq[5 + 2 * k] = v[2 * (qy * bw + qx) + 1];
            }
            cq[12] = 0.0f; cq[13] = 0.0f;
        }
    for (int k = 0; k < 7; k++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                size_t q = (size_t)y * w + x;
                float hx = cand[q * 14 + 2 * k], hy = cand[q * 14 + 2 * k + 1];
                float a = fgo_i_remap_f(ya, w, h, 1, (float)x - hx, (float)y - hy);
                float c = fgo_i_remap_f(yc, w, h, 1, (float)x + hx, (float)y + hy);
                err[q] = absf(a - c);
            }
        fgo_i_box_blur(err, w, h, 5, cost + np_ * k);
    }
    #pragma omp parallel for schedule(static)
    for (size_t q = 0; q < np_; q++) {
        float best = 0.0f;
        int bk = 0;
        for (int k = 0; k < 7; k++) {
            float c = cost[np_ * k + q];
            if (k == 0) c = c - smooth;
            if (k == 6) c = c - zero;
            if (k == 0 || c < best) { best = c; bk = k; }
        }
        pf[2 * q] = cand[q * 14 + 2 * bk];
        pf[2 * q + 1] = cand[q * 14 + 2 * bk + 1];
    }
    free(bil); free(cand); free(err); free(cost);
}

/* ---------------------------------------------------------------------------------------------- estimate */

/* CrosshairV2's estimate fill (Settings::uiEstimateFill; gpu/shaders/ui_v2_lumafill.comp), restated for this
 * library's level-0 luma: every flow cell of the mask rectangle's cells that holds a UI pixel (mask byte != 0) takes
 * the mean gray level of its not-UI pixels, the window widened by S px on every side per step, up to 8 px, while it has
 * none (no such pixel within 8 px: the cell keeps its luma). The mean is rounded half up to the level-0 grid (a
 * multiple of 1 / S^2), where the reference keeps it unrounded, so the estimate's sums stay exact in any order. */
static void ui_fill(const img8* m, const fgo_uimask* u, int fs, float* L0, int fw, int fh) {
    if (!u || !u->m || u->w <= 0 || u->h <= 0) return;
    const int cx0 = u->x / fs, cx1 = (u->x + u->w - 1) / fs, cy0 = u->y / fs, cy1 = (u->y + u->h - 1) / fs;
    for (int cy = cy0; cy <= cy1 && cy < fh; cy++)
        for (int cx = cx0; cx <= cx1 && cx < fw; cx++) {
            const int px = cx * fs, py = cy * fs;
            int has = 0;
            for (int j = 0; j < fs && !has; j++)
                for (int i = 0; i < fs; i++)
                    if (px + i < m->W && py + j < m->H && ui_px(u, px + i, py + j)) { has = 1; break; }
            if (!has) continue;
            for (int k = 0; k <= 8; k += fs) {
                long sum = 0;
                int n = 0;
                for (int y = py - k; y < py + fs + k; y++)
                    for (int x = px - k; x < px + fs + k; x++) {
                        if (x < 0 || y < 0 || x >= m->W || y >= m->H || ui_px(u, x, y)) continue;
                        sum += gray8(m, x, y);
                        n++;
                    }
                if (n > 0) {
                    const long s2 = (long)fs * fs;
                    L0[(size_t)cy * fw + cx] = (float)((2 * sum * s2 + n) / (2 * (long)n)) / (float)s2;
                    break;
                }
            }
        }
}

/* interp.estimate (flow + the cut test + pixel_field). Output buffers (any may be NULL except pf):
 *   luma   : per level l, a (lw*lh floats) then c
 *   fields : per level l, the search output then the median3 output (2*bw*bh floats each); then sub1 and sub2
 *            (the finest level after the 0.5 and 0.25 px steps)
 *   seeds  : per level l, the seed field of the search (zeros at the coarsest)
 *   meds   : per level l, 2 x the global median (the seed candidate), 0 at the coarsest
 *   sads   : the finest level's per-block SAD the cut test averages
 * Returns the number of levels, or -1. pf is written even for a cut (interp skips it: its pf is None). */
int fgo_estimate_cnn(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                     int cnnLevel, const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads,
                     float* pf, float* sad_mean, int* cut, int nthreads);

int fgo_estimate(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                 float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf, float* sad_mean, int* cut,
                 int nthreads) {
    return fgo_estimate_cnn(a8, c8, W, H, pitch, order, s, -1, NULL, luma, fields, seeds, meds, sads, pf, sad_mean, cut,
                            nthreads);
}

/* fgo_estimate with the seed net's output at level cnnLevel (cnn: that level's bw*bh x 8 floats, NULL = plain): the
 * levels above it are skipped and its search is seeded by seed_cnn */
static int estimate_impl(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                         int cnnLevel, const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads,
                         float* pf, float* sad_mean, int* cut, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc);

int fgo_estimate_cnn(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                     int cnnLevel, const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads,
                     float* pf, float* sad_mean, int* cut, int nthreads) {
    return estimate_impl(a8, c8, W, H, pitch, order, s, cnnLevel, cnn, luma, fields, seeds, meds, sads, pf, sad_mean, cut,
                         nthreads, NULL, NULL);
}

/* fgo_estimate with CrosshairV2's estimate fill of prev's / curr's level-0 luma from their UI masks */
int fgo_estimate_ui(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                    float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf, float* sad_mean, int* cut,
                    int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
    return estimate_impl(a8, c8, W, H, pitch, order, s, -1, NULL, luma, fields, seeds, meds, sads, pf, sad_mean, cut,
                         nthreads, ua, uc);
}

static int estimate_impl(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                         int cnnLevel, const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads,
                         float* pf, float* sad_mean, int* cut, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int fw, fh, lw[MAXLV], lh[MAXLV];
    int n = fgo_layout(W, H, s->flowScale, s->pyramidMinSide, &fw, &fh, lw, lh, MAXLV);
    if (n < 1) return -1;
    img8 A = mkimg(a8, W, H, pitch, order), C = mkimg(c8, W, H, pitch, order);
    float* L[MAXLV][2];
    for (int l = 0; l < n; l++)
        for (int k = 0; k < 2; k++) L[l][k] = malloc(sizeof(float) * (size_t)lw[l] * lh[l]);
    luma_area(&A, s->flowScale, L[0][0], fw, fh);
    luma_area(&C, s->flowScale, L[0][1], fw, fh);
    ui_fill(&A, ua, s->flowScale, L[0][0], fw, fh);
    ui_fill(&C, uc, s->flowScale, L[0][1], fw, fh);
    for (int l = 1; l < n; l++)
        for (int k = 0; k < 2; k++) fgo_i_area_half(L[l - 1][k], lw[l - 1], lh[l - 1], L[l][k], lw[l], lh[l], 0);
    int r = fgo_i_estimate_levels(L, n, lw, lh, s, cnnLevel, cnn, luma, fields, seeds, meds, sads, pf, sad_mean, cut);
    for (int l = 0; l < n; l++) { free(L[l][0]); free(L[l][1]); }
    return r;
}

int fgo_i_estimate_levels(float* L[][2], int n, const int* lw, const int* lh, const fgo_settings* s, int cnnLevel,
                          const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf,
                          float* sad_mean, int* cut) {
    if (n < 1 || n > MAXLV) return -1;
    int bw[MAXLV] = {0}, bh[MAXLV] = {0};
    size_t lofs = 0, fofs = 0, sofs = 0;
    for (int l = 0; l < n; l++) { bw[l] = (lw[l] + 7) / 8; bh[l] = (lh[l] + 7) / 8; }
    if (luma)
        for (int l = 0; l < n; l++)
            for (int k = 0; k < 2; k++) {
                memcpy(luma + lofs, L[l][k], sizeof(float) * (size_t)lw[l] * lh[l]);
                lofs += (size_t)lw[l] * lh[l];
            }
    /* field offsets per level (coarse to fine loop writes each level's slots) */
    size_t fo[MAXLV], so[MAXLV];
    for (int l = 0; l < n; l++) { fo[l] = fofs; fofs += (size_t)4 * bw[l] * bh[l]; so[l] = sofs; sofs += (size_t)2 * bw[l] * bh[l]; }
    float* v = NULL;
    int pw = 0, ph = 0;
    float* sadbuf = malloc(sizeof(float) * (size_t)bw[0] * bh[0]);
    const int top = cnn ? (cnnLevel < n - 1 ? cnnLevel : n - 1) : n - 1;
    for (int l = top; l >= 0; l--) {
        int nb = bw[l] * bh[l];
        float* seed = calloc((size_t)2 * nb, sizeof(float));
        float med[2] = {0.0f, 0.0f};
        float* vs = malloc(sizeof(float) * 2 * nb);
        float* vm = malloc(sizeof(float) * 2 * nb);
        float* sd = malloc(sizeof(float) * nb);
        int radius = s->searchRadius;
        if (cnn && l == top) seed_cnn(cnn, L[l][0], L[l][1], lw[l], lh[l], bw[l], bh[l], s->searchPenalty, seed);
        else if (v == NULL) radius = s->searchRadiusTop;
        else seed_from(v, pw, ph, L[l][0], L[l][1], lw[l], lh[l], bw[l], bh[l], s->searchPenalty, seed, med);
        search(L[l][0], L[l][1], lw[l], lh[l], bw[l], bh[l], seed, radius, 1.0f, s->searchPenalty, vs, sd);
        median3(vs, bw[l], bh[l], vm);
        if (fields) {
            memcpy(fields + fo[l], vs, sizeof(float) * 2 * nb);
            memcpy(fields + fo[l] + 2 * nb, vm, sizeof(float) * 2 * nb);
        }
        if (seeds) memcpy(seeds + so[l], seed, sizeof(float) * 2 * nb);
        if (meds) { meds[2 * l] = med[0]; meds[2 * l + 1] = med[1]; }
        if (l == 0) memcpy(sadbuf, sd, sizeof(float) * nb);
        free(seed); free(vs); free(sd);
        free(v);
        v = vm; pw = bw[l]; ph = bh[l];
    }
    int nb0 = bw[0] * bh[0];
    if (s->subpixel) {
        float* v2 = malloc(sizeof(float) * 2 * nb0);
        float steps[2] = {0.5f, 0.25f};
        for (int i = 0; i < 2; i++) {
            search(L[0][0], L[0][1], lw[0], lh[0], bw[0], bh[0], v, 1, steps[i], s->searchPenalty, v2, sadbuf);
            memcpy(v, v2, sizeof(float) * 2 * nb0);
            if (fields) memcpy(fields + fofs + (size_t)i * 2 * nb0, v, sizeof(float) * 2 * nb0);
        }
        free(v2);
    }
    float mean = fgo_mean_f32(sadbuf, nb0);
    if (sads) memcpy(sads, sadbuf, sizeof(float) * nb0);
    *sad_mean = mean;
    *cut = (double)mean > (double)s->sceneCutSad;
    pixel_field(v, bw[0], bh[0], L[0][0], L[0][1], lw[0], lh[0], s->smoothBonus, s->hudBonus, pf);
    free(v); free(sadbuf);
    return n;
}

/* ---------------------------------------------------------------------------------------------- synth */

/* interp.field_at: the midpoint-grid field looked up at time t (2 fixed-point bilinear steps) */
void fgo_i_field_at(const float* pf, int w, int h, float sf, float* out) {
    float* g = malloc(sizeof(float) * (size_t)w * h * 2);
    memcpy(g, pf, sizeof(float) * (size_t)w * h * 2);
    for (int it = 0; it < 2; it++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                size_t q = (size_t)y * w + x;
                float px = (float)x - sf * g[2 * q], py = (float)y - sf * g[2 * q + 1];
                out[2 * q] = fgo_i_remap_f(pf, w, h, 2, px, py);
                out[2 * q + 1] = fgo_i_remap_f(pf + 1, w, h, 2, px, py);
            }
        memcpy(g, out, sizeof(float) * (size_t)w * h * 2);
    }
    free(g);
}

/* interp.synth: the frame at time t from the estimate. out has the input's pixel layout (alpha = the nearer
 * frame's). reason: 0 = interpolated, 1 = scene cut, 2 = untrusted share. Optional: field_t (fw*fh*2, the field
 * at t), emap (W*H bytes: the per-pixel mismatch before the 7x7 box), *untrusted (pixels with trust past 0.5). */
static int synth_impl(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                      const float* pf, int cut, float t, uint8_t* out, int out_pitch, float* field_t, uint8_t* emap,
                      long long* untrusted, int* reason, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc);

int fgo_synth(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
              const float* pf, int cut, float t, uint8_t* out, int out_pitch, float* field_t, uint8_t* emap,
              long long* untrusted, int* reason, int nthreads) {
    return synth_impl(a8, c8, W, H, pitch, order, s, pf, cut, t, out, out_pitch, field_t, emap, untrusted, reason, nthreads,
                      NULL, NULL);
}

/* fgo_synth with CrosshairV2's tap rejection: ua / uc are prev's / curr's UI masks (either may be NULL) */
int fgo_synth_ui(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                 const float* pf, int cut, float t, uint8_t* out, int out_pitch, float* field_t, uint8_t* emap,
                 long long* untrusted, int* reason, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
    return synth_impl(a8, c8, W, H, pitch, order, s, pf, cut, t, out, out_pitch, field_t, emap, untrusted, reason, nthreads,
                      ua, uc);
}

static int synth_impl(const uint8_t* a8, const uint8_t* c8, int W, int H, int pitch, int order, const fgo_settings* s,
                      const float* pf, int cut, float t, uint8_t* out, int out_pitch, float* field_t, uint8_t* emap,
                      long long* untrusted, int* reason, int nthreads, const fgo_uimask* ua, const fgo_uimask* uc) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (!(t > 0.0f && t < 1.0f)) return -1;
    img8 A = mkimg(a8, W, H, pitch, order), C = mkimg(c8, W, H, pitch, order);
    const img8* N = t <= 0.5f ? &A : &C;
    int cn = A.cn;
    if (untrusted) *untrusted = 0;
    if (cut) {
        for (int y = 0; y < H; y++) memcpy(out + (size_t)y * out_pitch, N->p + (size_t)y * pitch, (size_t)W * cn);
        *reason = 1;
        return 0;
    }
    int fs = s->flowScale;
    int fw = rint_he(W * (1.0 / fs)), fh = rint_he(H * (1.0 / fs));
    double td = t;
    float sf = (float)(2.0 * td - 1.0);
    float* g = malloc(sizeof(float) * (size_t)fw * fh * 2);
    if (sf == 0.0f) memcpy(g, pf, sizeof(float) * (size_t)fw * fh * 2);
    else fgo_i_field_at(pf, fw, fh, sf, g);
    if (field_t) memcpy(field_t, g, sizeof(float) * (size_t)fw * fh * 2);
    int uw = fw * fs, uh = fh * fs;
    float* hv = malloc(sizeof(float) * (size_t)uw * uh * 2);
    fgo_i_resize_lin2(g, fw, fh, hv, uw, uh);
    free(g);
    float ka = (float)(2.0 * td), kc = (float)(2.0 * (1.0 - td));
    float wA = (float)(1.0 - td), wC = t;
    int mid = t == 0.5f;
    uint8_t* e = malloc((size_t)W * H);
    float* ef = malloc(sizeof(float) * (size_t)W * H);
    int* wab = malloc(sizeof(int) * (size_t)W * H * 8);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            int sy = y < uh ? y : uh - 1, sx = x < uw ? x : uw - 1;   /* crop [:H, :W], then edge pad */
            float hx = hv[((size_t)sy * uw + sx) * 2] * (float)fs, hy = hv[((size_t)sy * uw + sx) * 2 + 1] * (float)fs;
            int* wa = wab + ((size_t)y * W + x) * 8;
            int* wc = wa + 4;
            float pax, pay, pcx, pcy;
            if (mid) {
                pax = (float)x - hx; pay = (float)y - hy; pcx = (float)x + hx; pcy = (float)y + hy;
            } else {
                pax = (float)x - ka * hx; pay = (float)y - ka * hy; pcx = (float)x + kc * hx; pcy = (float)y + kc * hy;
            }
            remap_u8(&A, pax, pay, wa);
            remap_u8(&C, pcx, pcy, wc);
            if (ua || uc) {   /* a tap on its own frame's UI takes the other frame's tap; both or neither: unchanged */
                int ha = ui_hit(ua, pax, pay), hc = ui_hit(uc, pcx, pcy);
                if (ha != hc) {
                    if (ha) memcpy(wa, wc, 4 * sizeof(int));
                    else memcpy(wc, wa, 4 * sizeof(int));
                }
            }
            int m = 0;
            int ch[3] = {A.ri, A.gi, A.bi};
            for (int k = 0; k < 3; k++) {
                int d = abs(wa[ch[k]] - wc[ch[k]]);
                if (d > m) m = d;
            }
            e[(size_t)y * W + x] = (uint8_t)m;
            ef[(size_t)y * W + x] = (float)m;
        }
    free(hv);
    if (emap) memcpy(emap, e, (size_t)W * H);
    float* eb = malloc(sizeof(float) * (size_t)W * H);
    fgo_i_box_blur(ef, W, H, 7, eb);
    float t0 = s->trustLow, span = (float)((double)s->trustHigh - (double)s->trustLow);
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
        for (int y = 0; y < H; y++) memcpy(out + (size_t)y * out_pitch, N->p + (size_t)y * pitch, (size_t)W * cn);
        *reason = 2;
    } else {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                size_t q = (size_t)y * W + x;
                const int* wa = wab + q * 8;
                const int* wc = wa + 4;
                const uint8_t* nq = N->p + (size_t)y * pitch + (size_t)x * cn;
                uint8_t* o = out + (size_t)y * out_pitch + (size_t)x * cn;
                float u = eb[q], iu = 1.0f - u;
                int ch[3] = {A.ri, A.gi, A.bi};
                for (int k = 0; k < 3; k++) {
                    int c = ch[k];
                    float fa = (float)wa[c], fc = (float)wc[c], mix;
                    if (mid) mix = 0.5f * (fa + fc);
                    else { float p = wA * fa, r = wC * fc; mix = p + r; }
                    float p1 = mix * iu, p2 = (float)nq[c] * u;
                    float v = p1 + p2;
                    v = v + 0.5f;
                    v = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
                    o[c] = (uint8_t)v;
                }
                if (cn == 4) o[3] = nq[3];
            }
        *reason = 0;
    }
    free(e); free(ef); free(wab); free(eb);
    return 0;
}
