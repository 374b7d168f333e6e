/*
 * fg_oracle_internal.h -- what fg_oracle.c (the Rgba8 / interp.py restatement) shares with fg_oracle_fmt.c (the
 * restatement of the other frame formats). TEST INFRASTRUCTURE ONLY, like both files.
 */
#ifndef FG_ORACLE_INTERNAL_H
#define FG_ORACLE_INTERNAL_H
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
#endif
