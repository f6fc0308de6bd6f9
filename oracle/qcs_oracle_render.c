/*
 * TEST INFRASTRUCTURE ONLY -- CPU restatement of the super-resolution render
 * (ImageRenderData_TypeDef::FluoRenderTop's device part), the checker of
 * qc-storm_b200/csrc/qcs_render.cu.  Never called by the product library.
 *
 * Follows (paths under MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/):
 *   ImgRender/ImageRender_2d.cu:25-50   CreateRenderPSF (7x7 Gaussian, centre at the fractional position)
 *   ImgRender/ImageRender_2d.cu:55-155  FluoRenderWithPrec_2D (selection, weight, width, splat, max, histogram)
 *   ImgRender/ImageRender_3d.cu:60-148  FluoRenderWithPrec_3D (mean CRLB width, z-weighted colour map)
 *   ImgRender/ImageRender_top.cu:29-60  FluoRenderTop (2D for GS2D, 3D otherwise)
 * Rows are rendered one after another in row order, the order in which the
 * host build of the reference (one emulated thread at a time) adds them, so
 * with -ffp-contract=off and glibc expf the images, the maximum and the
 * histogram equal that build's bit for bit (tests/test_oracle_render_pin.py).
 * One guard is added: the histogram bin is (int)centre * 400 / max, and while
 * the running maximum is 0 (unit weights whose centre value is below 1) the
 * reference divides by zero; here, as in the product, the bin is skipped.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "qcs_oracle.h"

#define W 7
#define HALF 3

static void render_psf(float psf[W * W], float x, float y, float sigma) {
    sigma = -0.5f / (sigma * sigma);
    x = x - (int)x;
    y = y - (int)y;
    x = x + HALF;
    y = y + HALF;
    for (int yc = 0; yc < W; yc++)
        for (int xc = 0; xc < W; xc++) {
            const float dx = xc - x, dy = yc - y;
            psf[yc * W + xc] = expf((dx * dx + dy * dy) * sigma);
        }
}

static float fmaxf_ref(float a, float b) { return fmaxf(a, b); }

int qcso_render(const qcs_loc_para *p, const float *rows, int n, int mode, float fixed_prec, float *img,
                float *colormap, int *max_val, int *hist) {
    const int is2d = p->LocType == QCS_LOCTYPE_GS2D;
    const int SRW = p->SRImageWidth, SRH = p->SRImageHigh;
    const float zoom = p->PixelZoom, pixel = p->PixelSize;
    const float ZDepthTh = 5 * fmaxf(fabsf(p->MinZDepth), fabsf(p->MaxZDepth));
    float psf[W * W];
    for (int i = 0; i < n; i++) {
        const float *r = rows + (size_t)i * QCS_OUT_PARA_NUM;
        float PeakPhoton = r[QCS_POS_PPHO];
        const float X = r[QCS_POS_XPOS] * zoom;
        const float Y = r[QCS_POS_YPOS] * zoom;
        const float Z = r[QCS_POS_ZPOS];
        float CurSNR = r[QCS_POS_PSNR];
        float LocPrec = is2d ? r[QCS_POS_CRBX] : (r[QCS_POS_CRBX] + r[QCS_POS_CRBY]) / 2;
        CurSNR = isnan(LocPrec) ? 0 : CurSNR;
        PeakPhoton = isnan(LocPrec) ? 0 : PeakPhoton;
        PeakPhoton = (LocPrec <= 0) ? 0 : PeakPhoton;
        int valid = (CurSNR >= p->SNR_th) && (PeakPhoton > 1.0f) && (X > W) && (X < SRW - 1 - W) && (Y > W) &&
                    (Y < SRH - 1 - W);
        if (!is2d) valid = valid && (fabsf(Z) < ZDepthTh);
        if (!valid) continue;
        if (mode == QCS_RENDER_1PHOTON_CRLB || mode == QCS_RENDER_1PHOTON_FIXED) PeakPhoton = 1.0f;
        if (mode == QCS_RENDER_1PHOTON_FIXED) LocPrec = fixed_prec;
        if (is2d && LocPrec > 30.0f) {
            LocPrec = 30.0f;
            PeakPhoton = 0.0f;
        }
        LocPrec = fmaxf_ref(LocPrec, pixel / zoom / 2);
        const float sigma = LocPrec / (pixel / zoom);
        render_psf(psf, X, Y, sigma);
        if (is2d && mode == QCS_RENDER_FITTED_PHOTON_1PIXEL) {
            img[SRW * (int)Y + (int)X] += PeakPhoton;
        } else {
            for (int rc = 0; rc < W; rc++) {
                const int off = SRW * ((int)Y - HALF + rc) + (int)X - HALF;
                for (int cc = 0; cc < W; cc++) {
                    img[off + cc] += PeakPhoton * psf[rc * W + cc];
                    if (!is2d) colormap[off + cc] += Z * PeakPhoton * psf[rc * W + cc];
                }
            }
        }
        const int centre = SRW * (int)Y + (int)X;
        const int c = (int)img[centre];
        if (c > *max_val) *max_val = c;
        if (*max_val != 0) {
            const int pos = c * QCS_RENDER_HIST_LEN / *max_val;
            if (pos >= 0 && pos < QCS_RENDER_HIST_LEN) hist[pos] += 1;
        }
    }
    return 0;
}
