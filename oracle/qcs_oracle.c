/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle of the QC-STORM MLEbfgs path.
 * See qcs_oracle.h.  Build: make -C oracle (gcc -O2 -ffp-contract=off -fopenmp).
 *
 * Float-only stages restated here (reference paths relative to
 * MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/):
 *   WLE PSF width      WLEParaEstimation/WLEParaEstimation_core.h:44-156,
 *                      WLEParaEstimation_core.cu:21-28 (index), 91-136 (peak, two-sided width),
 *                      natural cubic spline WLEParaEstimation/SplineInterpolation.h:40-202
 *   nearest neighbour  WLEParaEstimation_core.cu:140-183 (same-frame minimum distance)
 *   molecule type      WLEParaEstimation_core.cu:197-264
 *   CRLB               bfgsMLE_Loc_top/LocPrecCalc_GaussianCRLB.h:65-243
 * The fit engine (single and multi emitter, cascade) is in qcs_oracle_impl.h.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "qcs_oracle.h"

#define QCSO_MAXPAR 11
#define QCSO_MAXPIX (17 * 17)

enum { KIND_GS2D = 0, KIND_AS3D = 1, KIND_2E = 2, KIND_3E = 3, KIND_AS3D2E = 4 };

/* npar, iterations, loss clamp at 0.01 (else 0), weighted loss */
struct qcso_kind {
    int npar, iters, clamp_001, weighted;
};
static const struct qcso_kind KINDS[5] = {
    {5, 8, 0, 1},   /* GS2D    bfgsMLE_GS2D_core.h:25-30          */
    {6, 11, 1, 1},  /* AS3D    bfgsMLE_AS3D_core.h:25-30          */
    {8, 13, 0, 1},  /* GS2D 2E bfgsMLE_GS2D_2Emitter_core.h:26-31 */
    {11, 16, 0, 0}, /* GS2D 3E bfgsMLE_GS2D_3Emitter_core.h:26-31, weights off at :54 */
    {11, 16, 1, 0}, /* AS3D 2E bfgsMLE_AS3D_2Emitter_core.h:26-31, weights off at :54 */
};

struct qcso_job {
    const qcs_loc_para *p;
    const uint16_t *rois;
    const float *wle;
    int R;
};

static int g_threads = 0;

void qcso_set_threads(int n) { g_threads = n; }

int qcso_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

static void apply_threads(void)
{
#ifdef _OPENMP
    omp_set_num_threads(qcso_get_threads());
#endif
}

/* ---------------------------------------------------------------- CRLB --- */
/* Expected image of a Gaussian PSF on an n x n grid centred on the emitter. */
static void crlb_psf(int n, const float *par, float *img)
{
    const int half = n / 2;
    const float pi = 3.141592654f;
    const float peak = 1 / (((2 * pi) * par[4]) * par[5]) * par[0];
    const float ix = 1 / ((2 * par[4]) * par[4]);
    const float iy = 1 / ((2 * par[5]) * par[5]);
    for (int yc = 0; yc < n; ++yc) {
        const float y = (float)(yc - half);
        for (int xc = 0; xc < n; ++xc) {
            const float x = (float)(xc - half);
            img[yc * n + xc] =
                peak * expf(-(((x - par[2]) * (x - par[2])) * ix + ((y - par[3]) * (y - par[3])) * iy)) + par[1];
        }
    }
}

/* Diagonal Fisher information of one position coordinate from numerical
 * second derivatives (dh = 0.02) of the model and of its logarithm. */
static float crlb_std(int n, float *par, int id)
{
    float m0[15 * 15], mp[15 * 15], mn[15 * 15];
    const float dh = 0.02f;
    const int len = n * n;
    crlb_psf(n, par, m0);
    par[id] += dh;
    crlb_psf(n, par, mp);
    par[id] -= 2 * dh;
    crlb_psf(n, par, mn);
    par[id] += dh;
    float fi = 0;
    for (int k = 0; k < len; ++k) {
        const float d2 = (((mp[k] - 2 * m0[k]) + mn[k]) / dh) / dh;
        const float d2l = (((logf(mp[k]) - 2 * logf(m0[k])) + logf(mn[k])) / dh) / dh;
        fi += d2 - m0[k] * d2l;
    }
    if (fi == 0.0f) fi = 1;
    return sqrtf(1 / fi);
}

int qcso_crlb(const qcs_loc_para *p, float *loc, int n)
{
    if (!p || (!loc && n > 0) || n < 0) return QCS_ERR_ARG;
    const int grid = (p->LocType == QCS_LOCTYPE_AS3D) ? 15 : 9;
    apply_threads();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float *r = loc + (size_t)i * QCS_OUT_PARA_NUM;
        const float tp = r[QCS_POS_TPHO] * p->QE;
        float bg = r[QCS_POS_BAKG] * p->QE;
        const float sx = r[QCS_POS_SIGX], sy = r[QCS_POS_SIGY];
        float cx = 100.0f, cy = 100.0f;
        if (tp > 1 && bg > 1 && sx > 0.1 && sy > 0.1 && sx < 10 && sy < 10) {
            bg = (bg * p->QE + p->ReadNoise_e * p->ReadNoise_e) / p->QE;
            float par[6] = {tp, bg, 0, 0, sx, sy};
            cx = crlb_std(grid, par, 2) * p->PixelSize;
            cy = crlb_std(grid, par, 3) * p->PixelSize;
        }
        r[QCS_POS_CRBX] = cx;
        r[QCS_POS_CRBY] = cy;
    }
    return QCS_OK;
}

/* ------------------------------------------------------- WLE pre-pass --- */
/* Natural cubic spline through (i, y[i]), i = 0..n-1, sampled at k/10. */
static void spline_x10(int n, const float *y, float *out)
{
    float A[17], B[17], Cc[17], D[17], rhs[17], beta[17], z[17];
    const int m = (n - 1) * 10 + 1;
    /* tridiagonal system: first and last rows are the natural end conditions */
    for (int i = 0; i < n; ++i) A[i] = y[i];
    rhs[0] = 0;
    rhs[n - 1] = 0;
    for (int i = 1; i < n - 1; ++i) {
        const float h0 = (float)i - (float)(i - 1), h1 = (float)(i + 1) - (float)i;
        rhs[i] = (3 / h1) * (y[i + 1] - y[i]) - (3 / h0) * (y[i] - y[i - 1]);
    }
    /* Thomas algorithm with the reference's recurrences */
    for (int i = 0; i < n - 1; ++i) {
        const float hi = (i == 0) ? 0.0f : (float)i - (float)(i - 1);
        const float hn = (i == 0) ? 0.0f : (float)(i + 1) - (float)i;
        const float diag = (i == 0) ? 1.0f : 2 * (hi + hn);
        const float upper = (i == 0) ? 0.0f : hn;
        const float lower = hi;
        beta[i] = (i == 0) ? upper / diag : upper / (diag - lower * beta[i - 1]);
    }
    for (int i = 0; i < n; ++i) {
        float diag, lower;
        if (i == 0 || i == n - 1) {
            diag = 1.0f;
            lower = 0.0f;
        } else {
            const float h0 = (float)i - (float)(i - 1), h1 = (float)(i + 1) - (float)i;
            diag = 2 * (h0 + h1);
            lower = h0;
        }
        z[i] = (i == 0) ? rhs[i] / diag : (rhs[i] - lower * z[i - 1]) / (diag - lower * beta[i - 1]);
    }
    for (int i = n - 1; i >= 0; --i) Cc[i] = (i == n - 1) ? z[i] : z[i] - beta[i] * Cc[i + 1];
    for (int i = 0; i < n - 1; ++i) {
        const float h = (float)(i + 1) - (float)i;
        B[i] = (1 / h) * (A[i + 1] - A[i]) - (h / 3) * (2 * Cc[i] + Cc[i + 1]);
        D[i] = (Cc[i + 1] - Cc[i]) / (3 * h);
    }
    for (int k = 0; k < m; ++k) {
        const float xn = (float)k * (1.0f / 10);
        int seg = (int)(xn - 0.0f);
        if (seg < 0) seg = 0;
        if (seg >= n - 1) seg = n - 2;
        const float d = xn - (float)seg;
        out[k] = ((A[seg] + B[seg] * d) + (Cc[seg] * d) * d) + ((D[seg] * d) * d) * d;
    }
}

/* Peak of the interpolated profile within +-8 samples of the centre, then the
 * two half-profile areas over the peak value (Gaussian: area = sigma*sqrt(pi/2)). */
static void two_sided_width(const float *v, int m, float *left, float *right)
{
    const int span = (int)(10 * 0.8f);
    const int c = m / 2;
    int lo = c - span, hi = c + span;
    if (lo < 0) lo = 0;
    if (hi > m - 1) hi = m - 1;
    int best = m / 2;
    for (int k = lo; k <= hi; ++k)
        if (v[k] > v[best]) best = k;
    const float peak = v[best];
    const int ll = best, rl = m - best - 1;
    const int w = ll < rl ? ll : rl;
    float sl = 0, sr = 0;
    for (int k = best - w; k <= best; ++k) sl = sl + v[k];
    for (int k = best; k <= best + w; ++k) sr = sr + v[k];
    *left = ((sl * (1.0f / 10)) / peak) / 1.2533f;
    *right = ((sr * (1.0f / 10)) / peak) / 1.2533f;
}

static void psf_width(int R, const uint16_t *rec, float *out4)
{
    float mx[17], my[17], ix[161], iy[161];
    const int m = (R - 1) * 10 + 1;
    for (int k = 0; k < R; ++k) mx[k] = my[k] = 0;
    for (int r = 0; r < R; ++r)
        for (int c = 0; c < R; ++c) {
            mx[c] = mx[c] + (float)rec[r * R + c];
            my[r] = my[r] + (float)rec[r * R + c];
        }
    float minx = mx[0], miny = my[0];
    for (int k = 0; k < R; ++k) {
        minx = fminf(minx, mx[k]);
        miny = fminf(miny, my[k]);
    }
    for (int k = 0; k < R; ++k) {
        mx[k] = (mx[k] - minx) / (float)R;
        my[k] = (my[k] - miny) / (float)R;
    }
    spline_x10(R, mx, ix);
    spline_x10(R, my, iy);
    two_sided_width(ix, m, &out4[0], &out4[1]);
    two_sided_width(iy, m, &out4[2], &out4[3]);
}

static int cmp_key(const void *a, const void *b)
{
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : x > y;
}

/* Same-frame nearest-neighbour distance: for each ROI the minimum over other
 * ROIs of the same frame of dx^2+dy^2 (integer), capped at 1e8 (the
 * reference's "other frame / self" bias), then sqrt.  Grouped by frame here
 * instead of the reference's all-pairs loop; the integer minimum is the same. */
static void nearest_neighbour(int R, const uint16_t *rois, int n, float *wle)
{
    const int whole = R * (R + 1);
    int64_t *key = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        const uint16_t *h = rois + (size_t)i * whole + R * R;
        const int64_t frame = (int64_t)h[2] + 65536 * (int64_t)h[3];
        key[i] = (frame << 24) | i;
    }
    qsort(key, n, sizeof(int64_t), cmp_key);
    int s = 0;
    while (s < n) {
        int e = s;
        while (e < n && (key[e] >> 24) == (key[s] >> 24)) ++e;
#pragma omp parallel for schedule(dynamic, 16)
        for (int a = s; a < e; ++a) {
            const int i = (int)(key[a] & 0xFFFFFF);
            const uint16_t *hi = rois + (size_t)i * whole + R * R;
            float best = 100000000.0f;
            for (int b = s; b < e; ++b) {
                if (b == a) continue;
                const int j = (int)(key[b] & 0xFFFFFF);
                const uint16_t *hj = rois + (size_t)j * whole + R * R;
                const int dx = (int)hi[0] - (int)hj[0], dy = (int)hi[1] - (int)hj[1];
                const float d2 = (float)(int)((unsigned)(dx * dx) + (unsigned)(dy * dy));
                best = fminf(best, d2);
            }
            wle[(size_t)i * QCS_WLE_PARA_NUM + 0] = sqrtf(best);
        }
        s = e;
    }
    free(key);
}

int qcso_wle(const qcs_loc_para *p, const uint16_t *rois, int n, float *wle)
{
    if (!p || n < 0 || (n > 0 && (!rois || !wle))) return QCS_ERR_ARG;
    const int R = p->ROISize;
    if (R < 3 || R > 17) return QCS_ERR_ROISIZE;
    const int whole = R * (R + 1);
    apply_threads();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) psf_width(R, rois + (size_t)i * whole, wle + (size_t)i * QCS_WLE_PARA_NUM + 1);
    nearest_neighbour(R, rois, n, wle);
    const float th = (p->LocType == QCS_LOCTYPE_GS2D) ? (float)R / 2.1f / 2.35f : (float)R / 1.9f / 2.35f;
    for (int i = 0; i < n; ++i) {
        float *w = wle + (size_t)i * QCS_WLE_PARA_NUM;
        const int det = rois[(size_t)i * whole + R * R + 4];
        const float nn = w[0], sl = w[1], sr = w[2], su = w[3], sd = w[4];
        const float d1 = fabsf(sl - sr) / fminf(sl, sr);
        const float d2 = fabsf(su - sd) / fminf(su, sd);
        const int contaminated = (d1 >= 0.40f) || (d2 >= 0.40f);
        const float mean = (((sl + sr) + su) + sd) / 4;
        int type;
        if (det == QCS_ROITYPE_SINGLE && !contaminated && nn >= (float)R && mean <= th)
            type = QCS_MOLECULE_MLEFIT;
        else if (det == QCS_ROITYPE_MULTI || mean > th || nn < ((float)R / 2.0f + 1.0f))
            type = QCS_MOLECULE_MULTIFIT;
        else
            type = QCS_MOLECULE_WLEFIT;
        w[5] = (float)type;
    }
    return QCS_OK;
}

/* ---------------------------------------------------------- fit engine --- */
static inline float rabs_f32(float v) { return fabsf(v); }
static inline double rabs_f64(double v) { return fabs(v); }

static inline void write_row_f32(float *row, float pk, float x, float y, float z, float sx, float sy, float tot,
                                 float bkg, float snr, int frame)
{
    row[QCS_POS_PPHO] = pk;
    row[QCS_POS_XPOS] = x;
    row[QCS_POS_YPOS] = y;
    row[QCS_POS_ZPOS] = z;
    row[QCS_POS_SIGX] = sx;
    row[QCS_POS_SIGY] = sy;
    row[QCS_POS_TPHO] = tot;
    row[QCS_POS_BAKG] = bkg;
    row[QCS_POS_PSNR] = snr;
    row[QCS_POS_FRME] = (float)frame;
}

static inline void write_row_f64(float *row, double pk, double x, double y, double z, double sx, double sy,
                                 double tot, double bkg, double snr, int frame)
{
    write_row_f32(row, (float)pk, (float)x, (float)y, (float)z, (float)sx, (float)sy, (float)tot, (float)bkg,
                  (float)snr, frame);
}

#define REAL float
#define REAL_IS_DOUBLE 0
#define SFX _f32
#include "qcs_oracle_impl.h"
#undef REAL
#undef REAL_IS_DOUBLE
#undef SFX

#define REAL double
#define REAL_IS_DOUBLE 1
#define SFX _f64
#include "qcs_oracle_impl.h"
#undef REAL
#undef REAL_IS_DOUBLE
#undef SFX

static int check_common(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n, const float *out)
{
    if (!p || n < 0 || (n > 0 && (!rois || !wle || !out))) return QCS_ERR_ARG;
    if (p->ROISize < 5 || p->ROISize > 17 || (p->ROISize & 1) == 0) return QCS_ERR_ROISIZE;
    return QCS_OK;
}

int qcso_localize_f32(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n, float *out,
                      int out_cap, int *n_valid, float *ratios)
{
    int st = check_common(p, rois, wle, n, out);
    if (st) return st;
    apply_threads();
    return localize_f32(p, rois, wle, n, out, out_cap, n_valid, ratios);
}

int qcso_localize_f64(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n, float *out,
                      int out_cap, int *n_valid, float *ratios)
{
    int st = check_common(p, rois, wle, n, out);
    if (st) return st;
    apply_threads();
    return localize_f64(p, rois, wle, n, out, out_cap, n_valid, ratios);
}

int qcso_fit_single_f32(int kind, const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n,
                        float *out)
{
    int st = check_common(p, rois, wle, n, out);
    if (st) return st;
    apply_threads();
    return fit_single_f32(kind, p, rois, wle, n, out);
}

int qcso_fit_single_f64(int kind, const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n,
                        float *out)
{
    int st = check_common(p, rois, wle, n, out);
    if (st) return st;
    apply_threads();
    return fit_single_f64(kind, p, rois, wle, n, out);
}

/* ROI extraction: see qcs_oracle_extract.c */
