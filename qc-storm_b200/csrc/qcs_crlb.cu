// CRLB of x and y for each localization: diagonal Fisher information from
// numerical second derivatives (dh = 0.02) of a Gaussian PSF model on a fixed
// 9x9 (2D) or 15x15 (astigmatic 3D) grid with the emitter at the centre, the
// fitted total photons, background (+ read noise^2) and sigma x/y;
// CRLB = PixelSize / sqrt(FI) in nm, 100 when the row is not fittable.
// Re-expressed from LocPrecCalc_GaussianCRLB.h:65-243 with every rounding
// step explicit (bit-identical results at 9 x 9); adds the bounds guard that
// the reference kernel lacks (:65-128) and reads the row count from the
// device.
#include <cuda_runtime.h>

#include "qcs_fit_math.cuh"
#include "qcs_kernels.h"

namespace qcs {
namespace {

// Contraction of the PSF exponent dx^2/(2 sx^2) + dy^2/(2 sy^2) at each of
// the reference's evaluation sites, as nvcc compiles GaussianPSF_generate2D
// inlined into them (found by comparing every combination against the
// reference's CUDA build; see SumMode in qcs_fit_math.cuh): CENTRE = the
// model and the base point of both derivatives (x0 = y0 = 0), SHIFT_X = the
// +-dh points of the x derivative, SHIFT_Y = those of the y derivative.
// PeakPn * exp(.) + background and d2 - model * d2log are fused
// multiply-adds at every site.
template <int G>
struct CrlbSites;
template <>
struct CrlbSites<9> {
    enum { CENTRE = kFuseSecond, SHIFT_X = kFuseFirst, SHIFT_Y = kFuseSecond };
};
template <>
struct CrlbSites<15> {
    enum { CENTRE = kFuseFirst, SHIFT_X = kFuseFirst, SHIFT_Y = kFuseSecond };
};

struct PsfPara {
    float peak, six, siy, bkg;
};

// Gaussian PSF value of the reference's model at offsets dx = CurX - x0,
// dy = CurY - y0 (LocPrecCalc_GaussianCRLB.h:131-173).
template <int MODE>
__device__ __forceinline__ float psf_value(const PsfPara &p, float dx, float dy) {
    const float e = __expf(-sum_of_products<MODE>(__fmul_rn(dx, dx), p.six, __fmul_rn(dy, dy), p.siy));
    return __fmaf_rn(p.peak, e, p.bkg);
}

// (f(+h) - 2 f(0) + f(-h)) / h / h with the reference's rounding
// (LocPrecCalc_GaussianCRLB.h:188-196; 2 f(0) is exact, so fusing it changes nothing).
__device__ __forceinline__ float second_diff(float fp, float f0, float fn) {
    const float dh = 0.02f;
    return __fdiv_rn(__fdiv_rn(__fadd_rn(__fmaf_rn(-2.0f, f0, fp), fn), dh), dh);
}

// One thread per row.  The reference evaluates the PSF on the full grid
// seven times per row (model, then base, +dh, -dh for each derivative) and
// sums d2 - model * d2log over every pixel.  The same values come from far
// fewer evaluations, exactly: the base points equal the model (same
// parameters, same rounding), the model is symmetric in x and y, the -dh
// evaluation is the +dh one mirrored (x - (-h) = -((-x) - h) exactly), and
// each derivative's terms are symmetric across the other axis.  So the
// model is evaluated on one quadrant, each +dh grid on half the rows
// (columns), each term on half the grid, and the Fisher sums still add every
// pixel's term in the reference's pixel order.  Per-thread tables live in
// shared memory, [entry][thread].
template <int G, int TPB>
__global__ void __launch_bounds__(TPB) crlb_kernel(float *__restrict__ loc, const int *__restrict__ n_dev, int n,
                                                   const int *__restrict__ ids, const uint8_t *__restrict__ skip,
                                                   float ReadNoise_e, float QE, float PixelSize) {
    enum { H = G / 2, Q = H + 1 };
    using S = CrlbSites<G>;
    __shared__ float sM[Q * Q][TPB], sLM[Q * Q][TPB], sTX[Q * G][TPB], sTY[G * Q][TPB];
    const int rows = n_dev ? *n_dev : n;
    const int slot = threadIdx.x + blockDim.x * blockIdx.x;
    if (slot >= rows) return;
    const int gid = ids ? ids[slot] : slot;
    if (skip && skip[gid]) return;
    const int t = threadIdx.x;
    float *r = loc + (size_t)gid * 12;
    const float TotalPhoton_e = __fmul_rn(r[QCS_POS_TPHO], QE);
    float Background_e = __fmul_rn(r[QCS_POS_BAKG], QE);
    const float sx = r[QCS_POS_SIGX], sy = r[QCS_POS_SIGY];
    float ParaStdX = 100.0f, ParaStdY = 100.0f;
    if ((TotalPhoton_e > 1) && (Background_e > 1) && (sx > 0.1) && (sy > 0.1) && (sx < 10) && (sy < 10)) {
        // read noise counted into the background (LocPrecCalc_GaussianCRLB.h:89-92)
        Background_e = __fdiv_rn(__fmaf_rn(ReadNoise_e, ReadNoise_e, __fmul_rn(Background_e, QE)), QE);
        const float pi = 3.141592654f;
        PsfPara p;
        p.peak = __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(__fmul_rn(__fmul_rn(2.0f, pi), sx), sy)), TotalPhoton_e);
        p.six = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sx), sx));
        p.siy = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sy), sy));
        p.bkg = Background_e;
        const float h = 0.02f;
        // model on one quadrant: sM[a][b] at |CurY| = a, |CurX| = b
#pragma unroll 1
        for (int a = 0; a < Q; ++a)
#pragma unroll
            for (int b = 0; b < Q; ++b) {
                const float v = psf_value<S::CENTRE>(p, (float)b, (float)a);
                sM[a * Q + b][t] = v;
                sLM[a * Q + b][t] = logf(v);
            }
        // x derivative: +dh row at |CurY| = a, terms for every column
#pragma unroll 1
        for (int a = 0; a < Q; ++a) {
            float tp[G], lp[G];
#pragma unroll
            for (int x = 0; x < G; ++x) {
                tp[x] = psf_value<S::SHIFT_X>(p, __fsub_rn((float)(x - H), h), (float)a);
                lp[x] = logf(tp[x]);
            }
#pragma unroll
            for (int x = 0; x < G; ++x) {
                const int b = x < H ? H - x : x - H;
                const float m = sM[a * Q + b][t];
                const float d2 = second_diff(tp[x], m, tp[G - 1 - x]);
                const float dl = second_diff(lp[x], sLM[a * Q + b][t], lp[G - 1 - x]);
                sTX[a * G + x][t] = __fmaf_rn(-m, dl, d2);
            }
        }
        // y derivative: +dh column at |CurX| = b, terms for every row
#pragma unroll 1
        for (int b = 0; b < Q; ++b) {
            float tp[G], lp[G];
#pragma unroll
            for (int y = 0; y < G; ++y) {
                tp[y] = psf_value<S::SHIFT_Y>(p, (float)b, __fsub_rn((float)(y - H), h));
                lp[y] = logf(tp[y]);
            }
#pragma unroll
            for (int y = 0; y < G; ++y) {
                const int a = y < H ? H - y : y - H;
                const float m = sM[a * Q + b][t];
                const float d2 = second_diff(tp[y], m, tp[G - 1 - y]);
                const float dl = second_diff(lp[y], sLM[a * Q + b][t], lp[G - 1 - y]);
                sTY[y * Q + b][t] = __fmaf_rn(-m, dl, d2);
            }
        }
        // Fisher information, pixel order (LocPrecCalc_GaussianCRLB.h:226-243)
        float FX = 0, FY = 0;
#pragma unroll 1
        for (int y = 0; y < G; ++y) {
            const int a = y < H ? H - y : y - H;
#pragma unroll
            for (int x = 0; x < G; ++x) {
                const int b = x < H ? H - x : x - H;
                FX = __fadd_rn(FX, sTX[a * G + x][t]);
                FY = __fadd_rn(FY, sTY[y * Q + b][t]);
            }
        }
        if (FX == 0.0f) FX = 1;
        if (FY == 0.0f) FY = 1;
        ParaStdX = __fmul_rn(__fsqrt_rn(__fdiv_rn(1.0f, FX)), PixelSize);
        ParaStdY = __fmul_rn(__fsqrt_rn(__fdiv_rn(1.0f, FY)), PixelSize);
    }
    r[QCS_POS_CRBX] = ParaStdX;
    r[QCS_POS_CRBY] = ParaStdY;
}

}  // namespace

cudaError_t launch_crlb(float *loc, const int *n_dev, int n, int max_rows, int loc_type, float ReadNoise_e, float QE,
                        float PixelSize, cudaStream_t s, const int *ids, const uint8_t *skip) {
    if (max_rows <= 0) return cudaSuccess;
    if (loc_type != QCS_LOCTYPE_AS3D) {
        constexpr int tpb = 64;
        crlb_kernel<9, tpb><<<(max_rows + tpb - 1) / tpb, tpb, 0, s>>>(loc, n_dev, n, ids, skip, ReadNoise_e, QE,
                                                                       PixelSize);
    } else {
        constexpr int tpb = 32;
        crlb_kernel<15, tpb><<<(max_rows + tpb - 1) / tpb, tpb, 0, s>>>(loc, n_dev, n, ids, skip, ReadNoise_e, QE,
                                                                        PixelSize);
    }
    return cudaGetLastError();
}

}  // namespace qcs
