// Cramer-Rao lower bound of every fitted parameter from the full Fisher
// information matrix, built and inverted in FP64: a side output next to the
// 12-float localization rows, whose CRLB columns (9, 10) keep the
// reference's diagonal x / y estimate (LocPrecCalc_GaussianCRLB.h:65-243:
// Fisher information of x alone, numerical second derivatives, fixed 9x9 or
// 15x15 grid, emitter at its centre).  No counterpart in the reference.
//
// Model of a row (the fit's own model, expected photoelectrons at the pixel
// centres (col + 0.5, row + 0.5) of the R x R ROI):
//   mu_k = N / (2 pi sx sy) exp(-dx^2 / (2 sx^2) - dy^2 / (2 sy^2)) + B,
// parameters x, y, N (total photoelectrons), B (background per pixel),
// sigma (GS2D, DH3D: sx = sy) or sx, sy (AS3D).  Poisson counts with Gaussian
// read noise: I_ij = sum_k (dmu_k/dtheta_i)(dmu_k/dtheta_j) / (mu_k + rn^2),
// the reference's treatment of read noise as extra background.  I is
// inverted by Cholesky; CRLB_i = sqrt((I^-1)_ii), and for AS3D the z bound
// follows from sx, sy through the calibration polynomial's Jacobian.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"
#include "qcs_kernels.h"

namespace qcs {
namespace {

struct FisherArgs {
    const float *rows;
    const uint16_t *rois;
    const int *n_dev;
    int n, n_rois, R;
    float qe, rn2, pixel_nm, zcorr;
    float pg[5], pl[5];  // p4..p0 of the sigma_x^2 - sigma_y^2 >= 0 and < 0 branches
    float *out;
};

template <int P>
__device__ void fisher_row(const FisherArgs &a, int i) {
    const float *row = a.rows + (size_t)i * 12;
    float *o = a.out + (size_t)i * QCS_FISHER_COLS;
    const double QE = a.qe;
    const double N = (double)row[6] * QE, B = (double)row[7] * QE;
    const double sx = row[4], sy = row[5];
#pragma unroll
    for (int c = 0; c < QCS_FISHER_COLS; c++) o[c] = 0.0f;
    if (!(row[0] > 0.0f) || !(N > 1.0) || !(B >= 0.0) || !(sx > 0.1 && sx < 10.0) || !(sy > 0.1 && sy < 10.0)) {
        o[QCS_FISHER_STATUS] = (float)QCS_FISHER_INVALID;
        return;
    }
    const int R = a.R;
    double x0 = R / 2.0, y0 = R / 2.0;  // no record: the emitter at the ROI centre
    if (a.rois && i < a.n_rois) {
        const uint16_t *hdr = a.rois + (size_t)i * R * (R + 1) + R * R;
        x0 = (double)row[1] - hdr[0] + R / 2;
        y0 = (double)row[2] - hdr[1] + R / 2;
    }
    const double isx2 = 1.0 / (sx * sx), isy2 = 1.0 / (sy * sy);
    const double norm = 1.0 / (2.0 * 3.14159265358979323846 * sx * sy);
    const double amp = N * norm;
    double I[P][P];
#pragma unroll
    for (int r = 0; r < P; r++)
#pragma unroll
        for (int c = 0; c < P; c++) I[r][c] = 0.0;
    for (int pr = 0; pr < R; pr++) {
        const double dy = pr + 0.5 - y0;
        for (int pc = 0; pc < R; pc++) {
            const double dx = pc + 0.5 - x0;
            const double g = exp(-0.5 * (dx * dx * isx2 + dy * dy * isy2));
            const double ag = amp * g;
            const double w = 1.0 / (ag + B + a.rn2);
            double d[P];
            d[0] = ag * dx * isx2;
            d[1] = ag * dy * isy2;
            d[2] = g * norm;
            d[3] = 1.0;
            if (P == 5) {
                d[4] = ag * ((dx * dx + dy * dy) * isx2 - 2.0) / sx;
            } else {
                d[4] = ag * (dx * dx * isx2 - 1.0) / sx;
                d[P - 1] = ag * (dy * dy * isy2 - 1.0) / sy;
            }
#pragma unroll
            for (int r = 0; r < P; r++)
#pragma unroll
                for (int c = 0; c <= r; c++) I[r][c] += d[r] * d[c] * w;
        }
    }
    // Cholesky I = L L^T (lower triangle in place), then S = I^-1 = L^-T L^-1
    double L[P][P];
#pragma unroll
    for (int r = 0; r < P; r++) {
#pragma unroll
        for (int c = 0; c <= r; c++) {
            double s = I[r][c];
#pragma unroll
            for (int k = 0; k < c; k++) s -= L[r][k] * L[c][k];
            if (r == c) {
                if (!(s > 0.0)) {
                    o[QCS_FISHER_STATUS] = (float)QCS_FISHER_SINGULAR;
                    return;
                }
                L[r][r] = sqrt(s);
            } else {
                L[r][c] = s / L[c][c];
            }
        }
    }
    // M = L^-1 (lower triangular)
    double M[P][P];
#pragma unroll
    for (int r = 0; r < P; r++) {
#pragma unroll
        for (int c = 0; c < P; c++) M[r][c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < P; c++) {
        M[c][c] = 1.0 / L[c][c];
#pragma unroll
        for (int r = c + 1; r < P; r++) {
            double s = 0.0;
#pragma unroll
            for (int k = c; k < r; k++) s += L[r][k] * M[k][c];
            M[r][c] = -s / L[r][r];
        }
    }
    // S_ij = sum_k M_ki M_kj (k >= max(i, j))
    auto S = [&](int i2, int j2) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < P; k++) s += M[k][i2] * M[k][j2];
        return s;
    };
    o[QCS_FISHER_X] = (float)(sqrt(S(0, 0)) * a.pixel_nm);
    o[QCS_FISHER_Y] = (float)(sqrt(S(1, 1)) * a.pixel_nm);
    o[QCS_FISHER_PHOTONS] = (float)(sqrt(S(2, 2)) / QE);
    o[QCS_FISHER_BACKGROUND] = (float)(sqrt(S(3, 3)) / QE);
    if (P == 5) {
        o[QCS_FISHER_SIGMA_X] = o[QCS_FISHER_SIGMA_Y] = (float)sqrt(S(4, 4));
    } else {
        o[QCS_FISHER_SIGMA_X] = (float)sqrt(S(4, 4));
        o[QCS_FISHER_SIGMA_Y] = (float)sqrt(S(5, 5));
        // z = poly(sx^2 - sy^2) * corr: dz/dsx = poly' 2 sx corr, dz/dsy = -poly' 2 sy corr
        const double s = sx * sx - sy * sy;
        const float *p = s >= 0.0 ? a.pg : a.pl;
        const double dpoly = ((4.0 * p[0] * s + 3.0 * p[1]) * s + 2.0 * p[2]) * s + p[3];
        const double jx = dpoly * 2.0 * sx * a.zcorr, jy = -dpoly * 2.0 * sy * a.zcorr;
        const double vz = jx * jx * S(4, 4) + 2.0 * jx * jy * S(4, 5) + jy * jy * S(5, 5);
        o[QCS_FISHER_Z] = (float)sqrt(vz > 0.0 ? vz : 0.0);
    }
    o[QCS_FISHER_STATUS] = (float)QCS_FISHER_OK;
}

template <int P>
__global__ void __launch_bounds__(128) fisher_kernel(FisherArgs a) {
    const int n = a.n_dev ? min(*a.n_dev, a.n) : a.n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) fisher_row<P>(a, i);
}

}  // namespace

cudaError_t launch_crlb_fisher(const qcs_loc_para &p, const float *rows, int n, const int *n_dev,
                               const uint16_t *rois, int n_rois, float *out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    FisherArgs a;
    a.rows = rows;
    a.rois = rois;
    a.n_dev = n_dev;
    a.n = n;
    a.n_rois = rois ? n_rois : 0;
    a.R = p.ROISize;
    a.qe = p.QE;
    a.rn2 = p.ReadNoise_e * p.ReadNoise_e;
    a.pixel_nm = p.PixelSize;
    a.zcorr = p.ZDepthCorrFactor;
    const float pg[5] = {p.p4_XGY, p.p3_XGY, p.p2_XGY, p.p1_XGY, p.p0_XGY};
    const float pl[5] = {p.p4_XLY, p.p3_XLY, p.p2_XLY, p.p1_XLY, p.p0_XLY};
    for (int k = 0; k < 5; k++) {
        a.pg[k] = pg[k];
        a.pl[k] = pl[k];
    }
    a.out = out;
    const int threads = 128;
    const int blocks = (n + threads - 1) / threads;
    if (p.LocType == QCS_LOCTYPE_AS3D)
        fisher_kernel<6><<<blocks, threads, 0, s>>>(a);
    else
        fisher_kernel<5><<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace qcs

extern "C" int qcs_crlb_fisher_fp64(const qcs_loc_para *p, const float *d_rows, int n, const uint16_t *d_rois,
                                    int n_rois, float *d_out, void *stream) {
    if (!p || n < 0 || n_rois < 0) return qcs::fail(QCS_ERR_ARG, "null parameter struct or negative count");
    if (p->LocType < QCS_LOCTYPE_GS2D || p->LocType > QCS_LOCTYPE_DH3D) return qcs::fail(QCS_ERR_ARG, "LocType");
    const int R = p->ROISize;
    if (R < 5 || R > 17 || (R & 1) == 0) return qcs::fail(QCS_ERR_ROISIZE, "ROISize must be odd, 5..17");
    if (!(p->QE > 0.0f)) return qcs::fail(QCS_ERR_ARG, "QE must be positive");
    if (n == 0) return QCS_OK;
    if (!d_rows || !d_out) return qcs::fail(QCS_ERR_ARG, "null pointer");
    QCS_CUDA(qcs::launch_crlb_fisher(*p, d_rows, n, nullptr, d_rois, n_rois, d_out, static_cast<cudaStream_t>(stream)),
             "Fisher CRLB launch");
    return QCS_OK;
}
