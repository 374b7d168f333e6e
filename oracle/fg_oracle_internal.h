/*
 * fg_oracle_internal.h -- what fg_oracle.c (the Rgba8 / interp.py restatement) shares with fg_oracle_fmt.c (the
 * restatement of the other frame formats). TEST INFRASTRUCTURE ONLY, like both files.
 */
#ifndef FG_ORACLE_INTERNAL_H
#define FG_ORACLE_INTERNAL_H
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define BLOCK 8
#define MAXLV 16

typedef struct fgo_settings {
    float trustLow, trustHigh, globalFallback, sceneCutSad, hudBonus, smoothBonus, searchPenalty;
    int searchRadius, searchRadiusTop, subpixel, flowScale, pyramidMinSide;
} fgo_settings;

int fgo_layout(int W, int H, int fs, int minSide, int* fw, int* fh, int* lw, int* lh, int maxLevels);

/* INTER_AREA 0.5 of a float level; round10: the result rounded half-even to a multiple of 2^-10 */
void fgo_i_area_half(const float* src, int sw, int sh, float* dst, int dw, int dh, int round10);
/* one cv2.remap INTER_LINEAR / BORDER_REPLICATE sample of a float plane (stride cs floats between pixels) */
float fgo_i_remap_f(const float* img, int w, int h, int cs, float x, float y);
/* cv2.resize(src (sh x sw x 2 float), (dw, dh), INTER_LINEAR) */
void fgo_i_resize_lin2(const float* src, int sw, int sh, float* dst, int dw, int dh);
/* cv2.blur(src, (k, k), BORDER_REPLICATE) of a float plane */
void fgo_i_box_blur(const float* src, int w, int h, int k, float* dst);
/* interp.field_at: the field looked up at time t (sf = 2t - 1) */
void fgo_i_field_at(const float* pf, int w, int h, float sf, float* out);
/* interp.estimate from a built pyramid L[l][0] (a), L[l][1] (c), l < n: the search, median3, sub-pixel steps, the
 * cut test and the pixel field, with the outputs fgo_estimate documents; with cnn (the seed net's output at
 * cnnLevel) the search starts at that level, seeded by the net's candidates. */
int fgo_i_estimate_levels(float* L[][2], int n, const int* lw, const int* lh, const fgo_settings* s, int cnnLevel,
                          const float* cnn, float* luma, float* fields, float* seeds, float* meds, float* sads, float* pf,
                          float* sad_mean, int* cut);

/* CrosshairV2's warp-tap rejection (gpu/shaders/ui_reject.glsl; gpu/shaders/motion_v1.glsl:117-129): the UI mask of a
 * frame over its rectangle (bytes, 0 = not UI). A tap at p reads the pixels lo..hi with X = roundEven(32 p),
 * lo = X >> 5, hi = lo + (X & 31 != 0) per axis; does any of them lie on the mask? */
typedef struct { const uint8_t* m; int x, y, w, h, stride; } fgo_uimask;

static inline int ui_hit(const fgo_uimask* u, float px, float py) {
    if (!u || !u->m || u->w <= 0 || u->h <= 0) return 0;
    int X = (int)nearbyintf(px * 32.0f), Y = (int)nearbyintf(py * 32.0f);
    int lx = X >> 5, ly = Y >> 5, hx = lx + ((X & 31) != 0), hy = ly + ((Y & 31) != 0);
    int x0 = lx - u->x, y0 = ly - u->y, x1 = hx - u->x, y1 = hy - u->y;
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 > u->w - 1) x1 = u->w - 1;
    if (y1 > u->h - 1) y1 = u->h - 1;
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++)
            if (u->m[(size_t)y * u->stride + x]) return 1;
    return 0;
}

static inline int ui_px(const fgo_uimask* u, int x, int y) {
    x -= u->x;
    y -= u->y;
    return x >= 0 && y >= 0 && x < u->w && y < u->h && u->m[(size_t)y * u->stride + x] != 0;
}


#endif
