/*
 * TEST INFRASTRUCTURE ONLY -- ROI extraction stage of the CPU oracle.
 *
 * Restates LDROIExtractData_TypeDef::ExtractMolecules (reference paths relative
 * to MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/SubregionExtraction/):
 *   filter taps                  LDROIExtraction_ImageFiltering.cu:22-81
 *   background removal           LDROIExtraction_ImageFiltering.cu:125-267
 *   image variance / threshold   LDROIExtraction.cu:140-177, _ImageFiltering.cu:503-533
 *   separable 5-tap Gaussian     LDROIExtraction_ImageFiltering.cu:286-454
 *   filtering sequence           LDROIExtraction_ImageFiltering.cu:85-121
 *   3x3 local maximum            LDROIExtraction_ROIExtraction.cu:25-164
 *   single/multi classification  LDROIExtraction_ROIExtraction.cu:181-243
 *   ROI cut and header           LDROIExtraction_ROIExtraction.cu:257-302
 *   batch accumulation           LDROIExtraction.cu:30-138, 181-216
 * Every float operation is separately rounded (this file is compiled with
 * -ffp-contract=off).  With flags 0 the variance is summed in pixel order, the
 * order a one-block-at-a-time run of the reference produces, and the result
 * equals the reference built for the host bit for bit.  QCSO_EXTRACT_FMA_CONV
 * accumulates the smoothing taps with fmaf, the contraction nvcc applies to
 * the reference's convolution loops; QCSO_EXTRACT_EXACT_VARIANCE takes the
 * mean and mean square from exact integer sums, each rounded once (the
 * reference adds its float terms with atomics, in whatever order the GPU
 * runs them, so its own value is not reproducible at the last bit; the exact
 * form is the deterministic value those sums approximate).  In GS2D with multi-emitter
 * fitting the reference smooths and sharpens into scratch buffers that the
 * detector never reads (the sharpen runs in place on its input,
 * _ImageFiltering.cu:675), so detection runs on the background-removed image;
 * that dead work is skipped here.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "qcs_oracle.h"

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static inline uint16_t to_u16(float v)
{
    if (!(v > 0.0f)) return 0;
    if (v >= 65535.0f) return 65535;
    return (uint16_t)v;
}

/* 5 normalised taps of the smoothing filter for this ROI size / mode. */
static void filter_taps(int R, int loc_type, int multi, float *taps)
{
    float sigma = 0.5f + (R - 7) * (1.0f - 0.5f) / (11 - 7);
    if (sigma < 0.5f) sigma = 0.5f;
    if (loc_type == QCS_LOCTYPE_AS3D)
        sigma *= 1.5f;
    else if (multi == 0 && loc_type == QCS_LOCTYPE_GS2D)
        sigma *= 1.2f;
    sigma = -1 / (2 * sigma * sigma);
    const float center = (float)(5 / 2);
    for (int c = 0; c < 5; ++c) taps[c] = expf((c - center) * (c - center) * sigma);
    float sum = 0;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) sum += taps[i] * taps[j];
    sum = sqrtf(1.0f / sum);
    for (int c = 0; c < 5; ++c) taps[c] = taps[c] * sum;
}

/* Background: per pixel the mean of the eight minima over opposite pairs of
 * the 9x9 border ring, averaged with the left and right neighbour inside its
 * aligned 32-column group, subtracted, clamped at 0. */
static float ring_background(const uint16_t *img, int W, int H, int x, int y)
{
    float l1[8], l2[8], l3[8], l4[8];
#define PX(xx, yy) ((float)img[(size_t)clampi((yy), 0, H - 1) * W + clampi((xx), 0, W - 1)])
    for (int i = 0; i < 8; ++i) {
        l1[i] = PX(x - 4 + i, y - 4);
        l3[i] = PX(x - 4 + i + 1, y + 4);
        l2[i] = PX(x + 4, y - 4 + i);
        l4[i] = PX(x - 4, y - 4 + i + 1);
    }
#undef PX
    for (int i = 0; i < 8; ++i) {
        l1[i] = fminf(l1[i], l2[i]);
        l3[i] = fminf(l3[i], l4[i]);
    }
    float b = 0;
    for (int i = 0; i < 8; ++i) b += fminf(l1[i], l3[7 - i]);
    return b / 8;
}

static void background_remove(const uint16_t *in, uint16_t *out, int W, int H)
{
    const int WT = (W + 31) / 32 * 32;
    float *bk = (float *)malloc(sizeof(float) * WT);
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < WT; ++x) bk[x] = ring_background(in, W, H, x, y);
        for (int x = 0; x < W; ++x) {
            const int g = x / 32 * 32, lane = x - g;
            const int s0 = lane - 1 < 0 ? 0 : lane - 1, s2 = lane + 1 > 31 ? 31 : lane + 1;
            const float mean = (bk[g + s0] + bk[g + lane] + bk[g + s2]) / 3.0f;
            float v = (float)in[(size_t)y * W + x] - mean;
            v = fmaxf(v, 0.0f);
            out[(size_t)y * W + x] = to_u16(v);
        }
    }
    free(bk);
}

/* Mean and mean square of the minimum of four quadrant pixels over a central
 * patch; variance floored at 100. */
static float image_variance(const uint16_t *img, int W, int H, int exact)
{
    const int cx = W / 2, cy = H / 2;
    int sw = W / 2 - 5, sh = H / 2 - 5;
    if (sw > 256) sw = 256;
    if (sh > 256) sh = 256;
    if (sw < 1) sw = 1;
    if (sh < 1) sh = 1;
    const int S = sw < sh ? sw : sh;
    const float total = (float)(S * S);
    float mx = 0, mx2 = 0;
    int64_t s1 = 0, s2 = 0;
    for (int gid = 0; gid < S * S; ++gid) {
        const int X = cx + gid % S, Y = cy + gid / S;
        uint16_t d1 = img[(size_t)Y * W + X];
        const uint16_t d2 = img[(size_t)Y * W + (X - S)];
        uint16_t d3 = img[(size_t)(Y - S) * W + X];
        const uint16_t d4 = img[(size_t)(Y - S) * W + (X - S)];
        d1 = d1 < d2 ? d1 : d2;
        d3 = d3 < d4 ? d3 : d4;
        d1 = d1 < d3 ? d1 : d3;
        if (exact) {
            s1 += d1;
            s2 += (int64_t)d1 * d1;
        } else {
            mx += (float)d1 / total;
            /* int product as the reference forms it (wraps above 46340) */
            mx2 += (float)(int32_t)((uint32_t)d1 * (uint32_t)d1) / total;
        }
    }
    if (exact) {
        mx = (float)((double)s1 / (double)(S * S));
        mx2 = (float)((double)s2 / (double)(S * S));
    }
    float var = mx2 - mx * mx;
    if (var < 100.0f) var = 100.0f;
    return var;
}

static inline float tap(float acc, float px, float t, int fma_conv)
{
    return fma_conv ? fmaf(px, t, acc) : acc + px * t;
}

static void conv_h(const uint16_t *in, uint16_t *out, int W, int H, const float *t, int fma_conv)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float acc = 0;
            for (int c = 0; c < 5; ++c)
                acc = tap(acc, (float)in[(size_t)y * W + clampi(x - 2 + c, 0, W - 1)], t[c], fma_conv);
            out[(size_t)y * W + x] = to_u16(acc);
        }
}

static void conv_v(const uint16_t *in, uint16_t *out, int W, int H, const float *t, int fma_conv)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float acc = 0;
            for (int c = 0; c < 5; ++c)
                acc = tap(acc, (float)in[(size_t)clampi(y - 2 + c, 0, H - 1) * W + x], t[c], fma_conv);
            out[(size_t)y * W + x] = to_u16(acc);
        }
}

struct extract_state {
    uint16_t *raw, *det, *tmp, *pos;
    int *cand;
};

/* One ExtractMolecules call over `nb` stacked frames; appends records. */
static int extract_batch(const qcs_loc_para *p, const uint16_t *frames, int nb, int start_frame, int flags,
                         struct extract_state *s, uint16_t *rois_out, float *wle_out, int cap, int *total)
{
    const int W = p->ImageWidth, H0 = p->ImageHigh, H = H0 * nb, R = p->ROISize, half = R / 2;
    const int whole = R * (R + 1);
    const size_t npx = (size_t)W * H;
    const int multi = p->MultiEmitterFitEn;
    memcpy(s->raw, frames, npx * sizeof(uint16_t));
    background_remove(s->raw, s->det, W, H);
    const float var = image_variance(s->det, W, H, (flags & QCSO_EXTRACT_EXACT_VARIANCE) != 0);
    if (!(p->LocType == QCS_LOCTYPE_GS2D && multi > 0)) {
        float taps[5];
        const int fma_conv = (flags & QCSO_EXTRACT_FMA_CONV) != 0;
        filter_taps(R, p->LocType, multi, taps);
        conv_h(s->det, s->tmp, W, H, taps, fma_conv);
        conv_v(s->tmp, s->det, W, H, taps, fma_conv);
    }
    /* local maxima */
    const float sd = sqrtf(var);
    float th = 9.5f * sd, th1 = 3.8f * sd;
    if (p->LocType == QCS_LOCTYPE_AS3D || (multi == 0 && p->LocType == QCS_LOCTYPE_GS2D)) {
        th = 8.5f * sd;
        th1 = 3.5f * sd;
    }
    memset(s->pos, 0, npx * sizeof(uint16_t));
    int ncand = 0;
    for (int y = 0; y < H; ++y) {
        const int ry = y % H0;
        for (int x = 0; x < W; ++x) {
            if (!(x >= half && ry >= half && x < W - half && ry < H0 - half)) continue;
            const int c = s->det[(size_t)y * W + x];
            if (!((float)c >= th)) continue;
            int v[3][3];
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) v[r][q] = s->det[(size_t)(y - 1 + r) * W + (x - 1 + q)];
            const int j1 = (v[0][0] > th1) + (v[0][1] > th1) + (v[0][2] > th1) + (v[1][0] > th1) + (v[1][2] > th1) +
                           (v[2][0] > th1) + (v[2][1] > th1) + (v[2][2] > th1);
            const int ji = (c > v[0][1]) + (c >= v[1][2]) + (c >= v[2][1]) + (c > v[1][0]);
            const int jo = (c > v[0][0]) + (c > v[0][2]) + (c > v[2][0]) + (c > v[2][2]);
            if (j1 >= 7 && ji == 4 && jo >= 3) {
                s->pos[(size_t)y * W + x] = 1;
                if (jo == 4) {
                    if (ncand < QCS_MAX_POINT_NUM) {
                        s->cand[2 * ncand] = x;
                        s->cand[2 * ncand + 1] = y;
                    }
                    ncand++;
                }
            }
        }
    }
    if (ncand > QCS_MAX_POINT_NUM) ncand = QCS_MAX_POINT_NUM;
    int base = *total;
    int written = 0;
    for (int k = 0; k < ncand; ++k) {
        const int x = s->cand[2 * k], y = s->cand[2 * k + 1];
        int type = QCS_ROITYPE_SINGLE;
        if (multi) {
            int nb_all = 0, nb3 = 0;
            for (int r = 0; r < R; ++r)
                for (int q = 0; q < R; ++q) nb_all += s->pos[(size_t)(y + r - half) * W + (x + q - half)];
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) nb3 += s->pos[(size_t)(y + r - 1) * W + (x + q - 1)];
            type = (nb_all - nb3 > 0) ? QCS_ROITYPE_MULTI : QCS_ROITYPE_SINGLE;
        }
        if (base + written >= cap) break;
        uint16_t *rec = rois_out + (size_t)(base + written) * whole;
        for (int r = 0; r < R; ++r)
            for (int q = 0; q < R; ++q) rec[r * R + q] = s->raw[(size_t)(y - half + r) * W + (x - half + q)];
        const int frame = start_frame + y / H0;
        rec[R * R + 0] = (uint16_t)x;
        rec[R * R + 1] = (uint16_t)(y % H0);
        rec[R * R + 2] = (uint16_t)(frame % 65536);
        rec[R * R + 3] = (uint16_t)(frame / 65536);
        rec[R * R + 4] = (uint16_t)type;
        written++;
    }
    if (written > 0) {
        int st = qcso_wle(p, rois_out + (size_t)base * whole, written, wle_out + (size_t)base * QCS_WLE_PARA_NUM);
        if (st) return st;
    }
    *total = base + written;
    return QCS_OK;
}

int qcso_extract(const qcs_loc_para *p, const uint16_t *frames, int n_frames, int batch, int start_frame,
                 int flags, uint16_t *rois_out, float *wle_out, int cap, int *n_roi, int *first_frame, int *end_frame)
{
    if (!p || !frames || !rois_out || !wle_out || !n_roi || n_frames < 0 || batch < 1) return QCS_ERR_ARG;
    if (p->ROISize < 5 || p->ROISize > 17 || (p->ROISize & 1) == 0) return QCS_ERR_ROISIZE;
    const int W = p->ImageWidth, H0 = p->ImageHigh;
    if (W < 16 || H0 < 16) return QCS_ERR_ARG;
    const size_t npx = (size_t)W * H0 * batch;
    struct extract_state s;
    s.raw = (uint16_t *)malloc(npx * sizeof(uint16_t));
    s.det = (uint16_t *)malloc(npx * sizeof(uint16_t));
    s.tmp = (uint16_t *)malloc(npx * sizeof(uint16_t));
    s.pos = (uint16_t *)malloc(npx * sizeof(uint16_t));
    s.cand = (int *)malloc(sizeof(int) * 2 * QCS_MAX_POINT_NUM);
    int total = 0, first = -1, end = -1, st = QCS_OK;
    for (int f = 0; f < n_frames && st == QCS_OK; f += batch) {
        const int nb = (n_frames - f) < batch ? (n_frames - f) : batch;
        if (first < 0 && end < 0) {
            first = start_frame + f;
            end = first + nb - 1;
        } else {
            end += nb;
        }
        st = extract_batch(p, frames + (size_t)f * W * H0, nb, start_frame + f, flags, &s, rois_out, wle_out, cap, &total);
    }
    free(s.raw);
    free(s.det);
    free(s.tmp);
    free(s.pos);
    free(s.cand);
    *n_roi = total;
    if (first_frame) *first_frame = first;
    if (end_frame) *end_frame = end;
    return st;
}
