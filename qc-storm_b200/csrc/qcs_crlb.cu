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

// Two lanes per row.  The reference evaluates the PSF on the full grid
// seven times per row (model, then base, +dh, -dh for each derivative) and
// sums d2 - model * d2log over every pixel.  The same values come from far
// fewer evaluations, exactly: the base points equal the model (same
// parameters, same rounding), the model is symmetric in x and y, the -dh
// evaluation is the +dh one mirrored (x - (-h) = -((-x) - h) exactly), and
// each derivative's terms are symmetric across the other axis.  So the
// model is evaluated on one quadrant, each +dh grid on half the rows
// (columns), each term on half the grid, and the Fisher sums still add every
// pixel's term in the reference's pixel order.  A 32-thread block takes 16
// rows: lane r (r < 16) computes row r's x-derivative terms and Fisher sum,
// lane r + 16 its y-derivative terms and sum, after the two have filled the
// row's model table together.  The y terms are the x terms' code with the
// axes exchanged (the reference's two sites contract mirror-image products),
// so the warp does not diverge; each sum still runs in pixel order.  Tables
// live in shared memory, [entry][row].
template <int G>
__global__ void __launch_bounds__(32) crlb_kernel(float *__restrict__ loc, const int *__restrict__ n_dev, int n,
                                                  const int *__restrict__ ids, const uint8_t *__restrict__ skip,
                                                  float ReadNoise_e, float QE, float PixelSize) {
    enum { H = G / 2, Q = H + 1, ROWS = 16, TT = Q * G * ROWS, TSTRIDE = TT + ((TT % 32) == 0 ? 16 : 0) };
    using S = CrlbSites<G>;
    // the x-derivative lane uses fma(dx^2, six, dy^2 siy), the y-derivative lane
    // fma(dy^2, siy, dx^2 six): one expression with its operands exchanged
    static_assert(S::SHIFT_X == kFuseFirst && S::SHIFT_Y == kFuseSecond, "mirrored derivative sites");
    // per row: model and its log on one quadrant (shared by the row's two
    // lanes); per lane: its derivative's terms T[l][k] (line l, position k)
    __shared__ float sM[Q * Q][ROWS], sLM[Q * Q][ROWS];
    __shared__ float sT[2 * TSTRIDE];
    const int lane = threadIdx.x, slot = lane & (ROWS - 1), role = lane >> 4;  // role 0: x, 1: y
    const int rows = n_dev ? *n_dev : n;
    const int k_slot = blockIdx.x * ROWS + slot;
    bool have = k_slot < rows;
    const int gid = have ? (ids ? ids[k_slot] : k_slot) : 0;
    if (have && skip && skip[gid]) have = false;
    float *r = loc + (size_t)gid * 12;
    bool valid = false;
    PsfPara p = {0.0f, 0.0f, 0.0f, 0.0f};
    if (have) {
        const float TotalPhoton_e = __fmul_rn(r[QCS_POS_TPHO], QE);
        float Background_e = __fmul_rn(r[QCS_POS_BAKG], QE);
        const float sx = r[QCS_POS_SIGX], sy = r[QCS_POS_SIGY];
        valid = (TotalPhoton_e > 1) && (Background_e > 1) && (sx > 0.1) && (sy > 0.1) && (sx < 10) && (sy < 10);
        if (valid) {
            // read noise counted into the background (LocPrecCalc_GaussianCRLB.h:89-92)
            Background_e = __fdiv_rn(__fmaf_rn(ReadNoise_e, ReadNoise_e, __fmul_rn(Background_e, QE)), QE);
            const float pi = 3.141592654f;
            p.peak = __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(__fmul_rn(__fmul_rn(2.0f, pi), sx), sy)), TotalPhoton_e);
            p.six = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sx), sx));
            p.siy = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sy), sy));
            p.bkg = Background_e;
            // model on one quadrant, sM[a][b] at |CurY| = a, |CurX| = b: the two
            // lanes of the row take alternate entries
            for (int e = role; e < Q * Q; e += 2) {
                const int a = e / Q, b = e - (e / Q) * Q;
                const float v = psf_value<S::CENTRE>(p, (float)b, (float)a);
                sM[e][slot] = v;
                sLM[e][slot] = logf(v);
            }
        }
    }
    __syncwarp();
    float std_dev = 100.0f;
    if (valid) {
        const float h = 0.02f;
        float *T = sT + role * TSTRIDE;
        const float su = role ? p.siy : p.six, sv = role ? p.six : p.siy;
        // x lane: the +dh row at |CurY| = l, every column k; y lane: the +dh
        // column at |CurX| = l, every row k
#pragma unroll 1
        for (int l = 0; l < Q; ++l) {
            float tp[G], lp[G];
            const float fl = (float)l;
            const float ll = __fmul_rn(__fmul_rn(fl, fl), sv);
#pragma unroll
            for (int k = 0; k < G; ++k) {
                const float sh = __fsub_rn((float)(k - H), h);
                tp[k] = __fmaf_rn(p.peak, __expf(-__fmaf_rn(__fmul_rn(sh, sh), su, ll)), p.bkg);
                lp[k] = logf(tp[k]);
            }
#pragma unroll
            for (int k = 0; k < G; ++k) {
                const int o = k < H ? H - k : k - H;  // |k - H|
                const int e = role ? o * Q + l : l * Q + o;
                const float m = sM[e][slot];
                const float d2 = second_diff(tp[k], m, tp[G - 1 - k]);
                const float dl = second_diff(lp[k], sLM[e][slot], lp[G - 1 - k]);
                T[(l * G + k) * ROWS + slot] = __fmaf_rn(-m, dl, d2);
            }
        }
        // Fisher information, pixel order (LocPrecCalc_GaussianCRLB.h:226-243)
        float F = 0;
#pragma unroll 1
        for (int y = 0; y < G; ++y) {
            const int ay = y < H ? H - y : y - H;
#pragma unroll
            for (int x = 0; x < G; ++x) {
                const int bx = x < H ? H - x : x - H;
                const int tl = role ? bx : ay, tk = role ? y : x;
                F = __fadd_rn(F, T[(tl * G + tk) * ROWS + slot]);
            }
        }
        if (F == 0.0f) F = 1;
        std_dev = __fmul_rn(__fsqrt_rn(__fdiv_rn(1.0f, F)), PixelSize);
    }
    if (have) r[role ? QCS_POS_CRBY : QCS_POS_CRBX] = std_dev;
}

}  // namespace

cudaError_t launch_crlb(float *loc, const int *n_dev, int n, int max_rows, int loc_type, float ReadNoise_e, float QE,
                        float PixelSize, cudaStream_t s, const int *ids, const uint8_t *skip) {
    if (max_rows <= 0) return cudaSuccess;
    const int blocks = (max_rows + 15) / 16;  // 16 rows per 32-thread block
    if (loc_type != QCS_LOCTYPE_AS3D)
        crlb_kernel<9><<<blocks, 32, 0, s>>>(loc, n_dev, n, ids, skip, ReadNoise_e, QE, PixelSize);
    else
        crlb_kernel<15><<<blocks, 32, 0, s>>>(loc, n_dev, n, ids, skip, ReadNoise_e, QE, PixelSize);
    return cudaGetLastError();
}

}  // namespace qcs
