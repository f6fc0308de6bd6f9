/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle of the FP64 Fisher-matrix CRLB side
 * output (qcs_crlb_fisher_fp64 in the product library).  The product's bound
 * has no counterpart in the reference: the reference's CRLB columns are a
 * diagonal x / y estimate (bfgsMLE_Loc_top/LocPrecCalc_GaussianCRLB.h:65-243:
 * Fisher information of x alone, numerical second derivatives with step 0.02
 * on a fixed grid, emitter at the centre, read noise added to the
 * background).  For an emitter at the ROI centre the full bound of x
 * decouples from the other parameters by symmetry and equals that diagonal
 * estimate up to its numerical derivative; tests/test_oracle_fisher.py checks
 * this oracle against the reference's host build in that case, and against
 * closed forms.
 *
 * Same model, same parameters and same outputs as the product (see its
 * header comment in include/qcstorm_b200.h), everything in double, the
 * inverse by Gauss-Jordan elimination with partial pivoting (a different
 * method from the product's Cholesky, on purpose).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define QCSO_PI 3.14159265358979323846

#include "qcs_oracle.h"

static int invert(int P, double A[6][6], double X[6][6]) {
    double M[6][12];
    for (int r = 0; r < P; r++) {
        for (int c = 0; c < P; c++) {
            M[r][c] = A[r][c];
            M[r][P + c] = (r == c) ? 1.0 : 0.0;
        }
    }
    for (int c = 0; c < P; c++) {
        int piv = c;
        for (int r = c + 1; r < P; r++)
            if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
        if (!(fabs(M[piv][c]) > 0.0)) return 0;
        if (piv != c)
            for (int k = 0; k < 2 * P; k++) {
                double t = M[c][k];
                M[c][k] = M[piv][k];
                M[piv][k] = t;
            }
        const double d = M[c][c];
        for (int k = 0; k < 2 * P; k++) M[c][k] /= d;
        for (int r = 0; r < P; r++) {
            if (r == c) continue;
            const double f = M[r][c];
            if (f != 0.0)
                for (int k = 0; k < 2 * P; k++) M[r][k] -= f * M[c][k];
        }
    }
    for (int r = 0; r < P; r++)
        for (int c = 0; c < P; c++) X[r][c] = M[r][P + c];
    return 1;
}

int qcso_crlb_fisher_f64(const qcs_loc_para *p, const float *rows, int n, const uint16_t *rois, int n_rois,
                         float *out) {
    if (!p || n < 0 || !(p->QE > 0.0f)) return QCS_ERR_ARG;
    const int R = p->ROISize;
    const int P = p->LocType == QCS_LOCTYPE_AS3D ? 6 : 5;
    const double QE = p->QE, rn2 = (double)p->ReadNoise_e * p->ReadNoise_e;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float *row = rows + (size_t)i * 12;
        float *o = out + (size_t)i * QCS_FISHER_COLS;
        memset(o, 0, QCS_FISHER_COLS * sizeof(float));
        const double N = (double)row[6] * QE, B = (double)row[7] * QE;
        const double sx = row[4], sy = row[5];
        if (!(row[0] > 0.0f) || !(N > 1.0) || !(B >= 0.0) || !(sx > 0.1 && sx < 10.0) ||
            !(sy > 0.1 && sy < 10.0)) {
            o[QCS_FISHER_STATUS] = QCS_FISHER_INVALID;
            continue;
        }
        double x0 = R / 2.0, y0 = R / 2.0;
        if (rois && i < n_rois) {
            const uint16_t *hdr = rois + (size_t)i * R * (R + 1) + R * R;
            x0 = (double)row[1] - hdr[0] + R / 2;
            y0 = (double)row[2] - hdr[1] + R / 2;
        }
        const double amp = N / (2.0 * QCSO_PI * sx * sy);
        double I[6][6] = {{0}};
        for (int pr = 0; pr < R; pr++) {
            for (int pc = 0; pc < R; pc++) {
                const double dx = pc + 0.5 - x0, dy = pr + 0.5 - y0;
                const double g = exp(-(dx * dx / (2.0 * sx * sx) + dy * dy / (2.0 * sy * sy)));
                const double mu = amp * g + B;
                double d[6];
                d[0] = amp * g * dx / (sx * sx);                  /* d mu / d x0 */
                d[1] = amp * g * dy / (sy * sy);                  /* d mu / d y0 */
                d[2] = g / (2.0 * QCSO_PI * sx * sy);                /* d mu / d N  */
                d[3] = 1.0;                                       /* d mu / d B  */
                if (P == 5) {                                     /* d mu / d sigma (sx = sy) */
                    d[4] = amp * g * ((dx * dx + dy * dy) / (sx * sx * sx) - 2.0 / sx);
                } else {
                    d[4] = amp * g * (dx * dx / (sx * sx * sx) - 1.0 / sx);
                    d[5] = amp * g * (dy * dy / (sy * sy * sy) - 1.0 / sy);
                }
                for (int r = 0; r < P; r++)
                    for (int c = 0; c < P; c++) I[r][c] += d[r] * d[c] / (mu + rn2);
            }
        }
        double S[6][6];
        if (!invert(P, I, S) || !(S[0][0] > 0.0) || !(S[1][1] > 0.0)) {
            o[QCS_FISHER_STATUS] = QCS_FISHER_SINGULAR;
            continue;
        }
        o[QCS_FISHER_X] = (float)(sqrt(S[0][0]) * p->PixelSize);
        o[QCS_FISHER_Y] = (float)(sqrt(S[1][1]) * p->PixelSize);
        o[QCS_FISHER_PHOTONS] = (float)(sqrt(S[2][2]) / QE);
        o[QCS_FISHER_BACKGROUND] = (float)(sqrt(S[3][3]) / QE);
        if (P == 5) {
            o[QCS_FISHER_SIGMA_X] = o[QCS_FISHER_SIGMA_Y] = (float)sqrt(S[4][4]);
        } else {
            o[QCS_FISHER_SIGMA_X] = (float)sqrt(S[4][4]);
            o[QCS_FISHER_SIGMA_Y] = (float)sqrt(S[5][5]);
            const double s = sx * sx - sy * sy;
            double p4, p3, p2, p1;
            if (s >= 0.0) {
                p4 = p->p4_XGY; p3 = p->p3_XGY; p2 = p->p2_XGY; p1 = p->p1_XGY;
            } else {
                p4 = p->p4_XLY; p3 = p->p3_XLY; p2 = p->p2_XLY; p1 = p->p1_XLY;
            }
            const double dpoly = 4.0 * p4 * s * s * s + 3.0 * p3 * s * s + 2.0 * p2 * s + p1;
            const double jx = dpoly * 2.0 * sx * p->ZDepthCorrFactor;
            const double jy = -dpoly * 2.0 * sy * p->ZDepthCorrFactor;
            const double vz = jx * jx * S[4][4] + jx * jy * (S[4][5] + S[5][4]) + jy * jy * S[5][5];
            o[QCS_FISHER_Z] = (float)sqrt(vz > 0.0 ? vz : 0.0);
        }
        o[QCS_FISHER_STATUS] = QCS_FISHER_OK;
    }
    return QCS_OK;
}
