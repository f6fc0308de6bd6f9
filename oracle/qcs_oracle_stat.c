/*
 * TEST INFRASTRUCTURE ONLY -- localization statistics of the CPU oracle.
 *
 * Restates FluoStatisticData_TypeDef::GetStatisticalInf
 * (StatisticsInfo/statisticsInfo_top.cu:61-255) with its kernels
 * (statisticsInfo.cu:18-88, statisticsInfo_densityCalc.cu:17-103) and host
 * helpers (statisticsInfo_rc.cu:18-115, GetFirstFrame / GetLastFrame
 * bfgsMLE_Loc_top/bfgs_top.cu:345-381), one call per group of rows on one
 * state (ResetAllDat first), every CUDA thread run in turn in row order:
 *   - rows with total photons > 30, background > 2, SNR >= 3, mean width >=
 *     0.01 px and 0.01 < sqrt(CRLB_x^2 + CRLB_y^2) < 55 nm fill four
 *     histograms of StatInf_Hist_DatLenMax = 1600 bins (total photons / 25,
 *     precision / 0.15 nm, SNR / 0.125, width / 0.0125 px; truncated, clamped)
 *     and sums of precision, SNR, width and background;
 *   - activation density: in every frame between the first and last frame
 *     of the rows (without both ends when more than 3), the rows at least 5 px
 *     inside the image with no / one other such row of the frame within 10 px
 *     (2D) or 20 px (3D) give the neighbour ratios, turned into a density
 *     (molecules / um^2, GetActivationDensity) and corrected by the
 *     reference's polynomial (multi-emitter fitting on or off); kept from the
 *     previous call when 50 rows or fewer were counted;
 *   - means: total photons by centre of mass of the histogram bins above 10%
 *     of its maximum, the others as sums over the row count; each call's means
 *     appended to the time series, whose mean (without the first and last
 *     entries) is reported for photons, precision and SNR.
 * Float sums in row order with separate roundings: the reference built for
 * the host, bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "qcs_oracle.h"

#define ST_LEN 400
#define ST_LENMAX (ST_LEN * 4)
#define ST_GAP_PH (10000.0f / ST_LEN)
#define ST_GAP_PREC (60.0f / ST_LEN)
#define ST_GAP_SNR (50.0f / ST_LEN)
#define ST_GAP_PSF (5.0f / ST_LEN)

static int trunc_host(float v)
{
    if (v != v || v >= 2147483648.0f || v < -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
}

static int clamp_bin(int b)
{
    if (b < 0) b = 0;
    if (b >= ST_LENMAX) b = ST_LENMAX - 1;
    return b;
}

static int first_frame(const float *rows, int n)
{
    int cur = 0;
    for (int i = 0; i < n; ++i) {
        cur = trunc_host(rows[(size_t)i * 12 + 11]);
        if (cur != 0) break;
    }
    return cur;
}

static int last_frame(const float *rows, int n)
{
    int cur = 0;
    for (int i = n - 1; i > 0; --i) {
        cur = trunc_host(rows[(size_t)i * 12 + 11]);
        if (cur != 0) break;
    }
    return cur;
}

static float activation_density(float r0, float r1, float radius_um)
{
    const float PI = 3.14159f;
    if (r0 <= 0.001f) r0 = 0.001f;
    if (r1 <= 0.001f) r1 = 0.001f;
    if (r0 > 1) r0 = 1;
    if (r1 > 1) r1 = 1;
    const float ratio0 = logf(r0);
    const float ratio1 = logf(r1 / PI / radius_um / radius_um);
    const float density0 = -ratio0 / PI / radius_um / radius_um;
    const float density1 = -ratio1 / PI / radius_um / radius_um;
    return r0 * density0 + (1.0f - r0) * density1;
}

static float hist_mean(const int *h, int len, float pct)
{
    int mx = h[0];
    for (int i = 0; i < len; ++i) mx = h[i] > mx ? h[i] : mx;
    pct = pct * mx;
    float ws = 0, os = 0;
    for (int i = 0; i < len; ++i) {
        const float v = (float)h[i];
        if (v >= pct) {
            ws += v * (i + 0.5f);
            os += v;
        }
    }
    if (os == 0) os = 1;
    return ws / os;
}

static float series_mean(const float *v, int n)
{
    float mean = 0;
    if (n > 2) {
        float tot = 0;
        int k = 0;
        for (int i = 1; i < n - 1; ++i) {
            tot += v[i];
            k++;
        }
        if (k <= 0) k = 1;
        mean = tot / k;
    }
    return mean;
}

int qcso_stat(const qcs_loc_para *p, const float *rows, const int *sizes, int n_groups, int *hist, float *means)
{
    if (!p || !rows || !sizes || !hist || !means || n_groups < 0) return QCS_ERR_ARG;
    float *ts_ph = (float *)calloc((size_t)n_groups + 1, sizeof(float));
    float *ts_prec = (float *)calloc((size_t)n_groups + 1, sizeof(float));
    float *ts_snr = (float *)calloc((size_t)n_groups + 1, sizeof(float));
    int ts_n = 0;
    float m_ph = 0, m_prec = 0, m_snr = 0, m_bg = 0, m_psf = 0, m_ctl = 0, m_dens = 0;
    float tv_ph = 0, tv_prec = 0, tv_snr = 0;
    int h[4][ST_LENMAX];     /* the device histograms */
    int hout[4][ST_LENMAX];  /* their host copies, kept by a call with no rows */
    memset(h, 0, sizeof(h));
    memset(hout, 0, sizeof(hout));
    size_t off = 0;
    for (int g = 0; g < n_groups; ++g) {
        const int n = sizes[g];
        const float *r = rows + off * 12;
        off += (size_t)(n > 0 ? n : 0);
        if (n > 0) {
            /* CalcLocResultStatInf */
            float vnum = 0, sprec = 0, ssnr = 0, spsf = 0, sbg = 0;
            for (int i = 0; i < n; ++i) {
                const float *q = r + (size_t)i * 12;
                const float tp = q[6], bg = q[7];
                const float psf = (q[4] + q[5]) / 2;
                const float snr = q[8];
                const float px = q[9], py = q[10];
                const float pxy = sqrtf(px * px + py * py);
                if ((tp > 30.0f) && (bg > 2.0f) && (snr >= 3.0f) && (psf >= 0.01f) && (pxy > 0.01f) &&
                    ((double)pxy < 55.0)) {
                    h[0][clamp_bin(trunc_host(tp / ST_GAP_PH))]++;
                    h[1][clamp_bin(trunc_host(pxy / ST_GAP_PREC))]++;
                    h[2][clamp_bin(trunc_host(snr / ST_GAP_SNR))]++;
                    h[3][clamp_bin(trunc_host(psf / ST_GAP_PSF))]++;
                    vnum += 1.0f;
                    sprec += pxy;
                    ssnr += snr;
                    spsf += psf;
                    sbg += bg;
                }
            }
            if (vnum <= 0) vnum = 1;
            /* CalcLocalizationDensity2D */
            const float rad = (p->LocType == QCS_LOCTYPE_GS2D) ? 10.0f : 20.0f;
            const float rad_um = rad * p->PixelSize / 1000;
            const int sf = first_frame(r, n), ef = last_frame(r, n);
            int fs = sf, fe = ef;
            if (ef - sf + 1 > 3) {
                fs = sf + 1;
                fe = ef - 1;
            }
            float n0r = 0, n1r = 0;
            int total = 0;
            int *sel = (int *)malloc(sizeof(int) * (size_t)n);
            const float th2 = rad * rad;
            for (int f = fs; f <= fe; ++f) {
                int k = 0;
                for (int i = 0; i < n; ++i) {
                    const float *q = r + (size_t)i * 12;
                    const int xp = trunc_host(q[1]), yp = trunc_host(q[2]), fr = trunc_host(q[11]);
                    if (xp >= 5 && xp < p->ImageWidth - 5 && yp >= 5 && yp < p->ImageHigh - 5 && fr == f) sel[k++] = i;
                }
                int c0 = 0, c1 = 0;
                for (int a = 0; a < k; ++a) {
                    const float cx = r[(size_t)sel[a] * 12 + 1], cy = r[(size_t)sel[a] * 12 + 2];
                    int nb = 0;
                    for (int b = 0; b < k; ++b) {
                        const float ox = r[(size_t)sel[b] * 12 + 1], oy = r[(size_t)sel[b] * 12 + 2];
                        const float d2 = (ox - cx) * (ox - cx) + (oy - cy) * (oy - cy) + (b == a) * 1000000.0f;
                        nb += (d2 <= th2);
                    }
                    if (nb == 0) c0++;
                    if (nb == 1) c1++;
                }
                n0r += c0;
                n1r += c1;
                total += k;
            }
            free(sel);
            if (total > 50) {
                n0r /= total;
                n1r /= total;
                m_dens = activation_density(n0r, n1r, rad_um);
                if (p->MultiEmitterFitEn)
                    m_dens = m_dens * m_dens * 0.5098f + m_dens * 0.6364f;
                else
                    m_dens = m_dens * m_dens * 0.8082f + m_dens * 0.519f;
            }
            /* UpdateStatDat */
            memcpy(hout, h, sizeof(h));
            memset(h, 0, sizeof(h)); /* ResetDistribDat */
            m_ph = ST_GAP_PH * hist_mean(hout[0], ST_LENMAX, 0.1f);
            m_prec = sprec / vnum;
            m_snr = ssnr / vnum;
            m_bg = sbg / vnum;
            m_psf = spsf / vnum;
            m_ctl = m_psf * (-m_snr);
            ts_ph[ts_n] = m_ph;
            ts_prec[ts_n] = m_prec;
            ts_snr[ts_n] = m_snr;
            ts_n++;
            tv_ph = series_mean(ts_ph, ts_n);
            tv_prec = series_mean(ts_prec, ts_n);
            tv_snr = series_mean(ts_snr, ts_n);
        }
        int *ho = hist + (size_t)g * 4 * ST_LENMAX;
        memcpy(ho, hout, sizeof(hout));
        float *mo = means + (size_t)g * 10;
        mo[0] = m_ph;
        mo[1] = m_prec;
        mo[2] = m_snr;
        mo[3] = m_bg;
        mo[4] = m_psf;
        mo[5] = m_ctl;
        mo[6] = m_dens;
        mo[7] = tv_ph;
        mo[8] = tv_prec;
        mo[9] = tv_snr;
    }
    free(ts_ph);
    free(ts_prec);
    free(ts_snr);
    return QCS_OK;
}

/*
 * On-time fit: FluoStatisticData_TypeDef::UpdateOntimeRatio
 * (StatisticsInfo/statisticsInfo_top.cu:23-57) with the curve fit it runs,
 * BFGSOptimizer<float, 2, 4, 11> over ExpFit_PreFitting / ExpFit_TargerF
 * (BFGS for curve fitting/BFGSOptimizer.h:120-533, CurveFitting.cpp:27-58):
 * least squares of y = a * exp(b * i), i = 0..n-1, from a = y0,
 * b = log(y1 / y0) (0 unless y0, y1 > 0.01), in coordinates divided by
 * max(|start|, 1); 4 quasi-Newton steps, each along the direction normalised
 * to a mean |component| of 1 with the step length bracketed in [1e-5, 1] and
 * halved 11 times; gradients by central differences of 0.002; the inverse
 * Hessian updated by the BFGS formula.  Then the mean on time 2 / (k1 + k2),
 * k1 = -log(1 - a), k2 = -b, and the ratios of on times of 4 frames and more
 * summed into entry 3 and entries 0..3 clamped to [0, 1].  Every float
 * operation separately rounded in the reference's order.
 */
static float ot_sse(const float *u, const float *scale, const float *y, int n)
{
    const float a = u[0] * scale[0], b = u[1] * scale[1];
    float e = 0;
    for (int i = 0; i < n; ++i) {
        const float d = a * expf(b * i) - y[i];
        e += d * d;
    }
    return e;
}

static void ot_grad(const float *u, const float *scale, const float *y, int n, float *g)
{
    float t[2] = {u[0], u[1]};
    for (int k = 0; k < 2; ++k) {
        t[k] = t[k] - 0.002f;
        const float lo = ot_sse(t, scale, y, n);
        t[k] = t[k] + 0.004f;
        const float hi = ot_sse(t, scale, y, n);
        g[k] = (hi - lo) * 250.0f;
        t[k] = t[k] - 0.002f;
    }
}

int qcso_ontime(const float *ratios, int n, float *mean_ontime, float *out)
{
    if (!ratios || !mean_ontime || !out || n < 4) return QCS_ERR_ARG;
    float p[2], scale[2], g[2], d[2], H[4] = {1, 0, 0, 1};
    p[0] = ratios[0];
    p[1] = (ratios[0] > 0.01 && ratios[1] > 0.01) ? logf(ratios[1] / ratios[0]) : 0.0f;
    for (int k = 0; k < 2; ++k) {
        const float m = fabsf(p[k]);
        scale[k] = m > 1.0f ? m : 1.0f;
        p[k] = p[k] / scale[k];
    }
    ot_grad(p, scale, ratios, n, g);
    d[0] = -g[0];
    d[1] = -g[1];
    for (int it = 0; it < 4; ++it) {
        float tot = 0;
        for (int k = 0; k < 2; ++k) tot += fabsf(d[k]);
        tot = tot / 2;
        for (int k = 0; k < 2; ++k) d[k] = d[k] / tot;
        float pos[2] = {0.00001f, 1.0f}, x[4], f[2];
        for (int k = 0; k < 2; ++k) {
            x[k] = d[k] * 0.0001f + p[k];
            x[2 + k] = d[k] * 1.0f + p[k];
        }
        f[0] = ot_sse(x, scale, ratios, n);
        f[1] = ot_sse(x + 2, scale, ratios, n);
        for (int b = 0; b < 11; ++b) {
            const int sel = f[0] < f[1];
            pos[sel] = (pos[0] + pos[1]) * 0.5f;
            if (b < 10) {
                for (int k = 0; k < 2; ++k) x[sel * 2 + k] = d[k] * pos[sel] + p[k];
                f[sel] = ot_sse(x + sel * 2, scale, ratios, n);
            }
        }
        const float step = (pos[0] + pos[1]) * 0.5f;
        float s[2], yk[2], og[2];
        for (int k = 0; k < 2; ++k) {
            s[k] = d[k] * step;
            p[k] = p[k] + s[k];
        }
        if (it < 3) {
            og[0] = g[0];
            og[1] = g[1];
            ot_grad(p, scale, ratios, n, g);
            for (int k = 0; k < 2; ++k) yk[k] = g[k] - og[k];
            float sy = 0;
            for (int k = 0; k < 2; ++k) sy += s[k] * yk[k];
            sy = 1.0f / sy;
            float ty[2], ts[2], A[4], S[4], T[4];
            for (int k = 0; k < 2; ++k) {
                ty[k] = yk[k] * sy;
                ts[k] = s[k] * sy;
            }
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c) {
                    A[r * 2 + c] = (r == c ? 1.0f : 0.0f) - s[r] * ty[c];
                    S[r * 2 + c] = s[r] * ts[c];
                }
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c) {
                    T[r * 2 + c] = 0;
                    for (int k = 0; k < 2; ++k) T[r * 2 + c] += A[r * 2 + k] * H[k * 2 + c];
                }
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c) {
                    H[r * 2 + c] = 0;
                    for (int k = 0; k < 2; ++k) H[r * 2 + c] += T[r * 2 + k] * A[c * 2 + k];
                }
            for (int k = 0; k < 4; ++k) H[k] = H[k] + S[k];
            for (int r = 0; r < 2; ++r) {
                d[r] = 0;
                for (int c = 0; c < 2; ++c) d[r] -= H[r * 2 + c] * g[c];
            }
        }
    }
    const float a = p[0] * scale[0], b = p[1] * scale[1];
    const float k1 = -logf(1 - a), k2 = -b;
    *mean_ontime = 2 / (k1 + k2);
    for (int i = 0; i < n; ++i) out[i] = ratios[i];
    for (int i = 4; i < n; ++i) out[3] += out[i];
    for (int i = 0; i < 4; ++i) out[i] = fminf(fmaxf(out[i], 0.0f), 1.0f);
    return QCS_OK;
}
