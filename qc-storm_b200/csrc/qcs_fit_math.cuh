// Device arithmetic of the MLEbfgs fit: losses, numerical gradient, BFGS
// update and the fixed iteration schedule, one CUDA thread per ROI.
//
// Bit-level contract: the results equal the reference CUDA kernels' (QC-STORM
// bfgsMLE_dll, compiled by nvcc for sm_100a) bit for bit on the same records.
// The fixed-schedule optimiser with a numerical gradient amplifies any
// rounding difference (one fused multiply-add more or less moves most fits by
// more than 1e-3 px), so matching the reference's results rather than its
// statistics needs the same rounding sequence: every expression keeps the
// reference's operand order and its __expf/__logf intrinsics, and the sums of
// two products, whose fusion nvcc decides from the surrounding code, are
// spelled with explicit round-to-nearest intrinsics chosen per kind and ROI
// size (ArithSpec below).
// References (MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/):
//   loss        bfgsMLE_Loc_LD/bfgsMLE_GS2D_core.h:459-518, bfgsMLE_AS3D_core.h:485-544,
//               bfgsMLE_Loc_HD/bfgsMLE_GS2D_2Emitter_core.h:519-592,
//               bfgsMLE_GS2D_3Emitter_core.h:511-589, bfgsMLE_AS3D_2Emitter_core.h:570-644
//   gradient    bfgsMLE_GS2D_core.h:430-454 (same in the other kinds)
//   schedule    bfgsMLE_GS2D_core.h:313-426 (same in the other kinds)
//   BFGS update bfgsMLE_Loc_LD/bfgsMLE_core.h:65-204
#pragma once

#include <cstdint>

namespace qcs {

enum FitKind { kGS2D = 0, kAS3D = 1, k2E = 2, k3E = 3, kAS3D2E = 4 };

// parameters, iterations, loss clamp (0 or 0.01), weighted loss
template <int KIND> struct KindTraits;
template <> struct KindTraits<kGS2D> { enum { P = 5, IT = 8, CLAMP001 = 0, WEIGHTED = 1 }; };
template <> struct KindTraits<kAS3D> { enum { P = 6, IT = 11, CLAMP001 = 1, WEIGHTED = 1 }; };
template <> struct KindTraits<k2E> { enum { P = 8, IT = 13, CLAMP001 = 0, WEIGHTED = 1 }; };
template <> struct KindTraits<k3E> { enum { P = 11, IT = 16, CLAMP001 = 0, WEIGHTED = 0 }; };
template <> struct KindTraits<kAS3D2E> { enum { P = 11, IT = 16, CLAMP001 = 1, WEIGHTED = 0 }; };

constexpr int kBisections = 11;

// Scaled parameterisation: amplitude/128, background/64, 1/(2 sigma^2)/0.1
// (bfgsMLE_core.h:52-60).
#define QCS_ASCALE (128.0f)
#define QCS_BSCALE (64.0f)
#define QCS_SSCALE (0.1f)

// One ROI's pixels as seen by its thread: element k at img[k * ld].
// img holds pairs (photoelectrons max((adu - offset) * gain, 1), its __logf),
// element k at img[k * ld]; w the weighted-MLE mask, element k at w[k * ld].
struct RoiRef {
    const float2 *img;
    const float *w;    // read by the weighted kinds only
    int ld;
};

// Pixel rows are unrolled up to this ROI size; the row loop stays rolled.
// Without the unrolled row a thread's pixel terms form one dependent chain
// (exp -> model -> log -> deviance -> sum) with nothing to overlap it, which
// made 11x11 fits four times slower per pixel than 9x9 ones.  Up to 13 the
// roundings of the loss are fixed in the source (ArithSpec), so unrolling
// changes no result.
constexpr int kUnrollMaxR = 13;

// Contraction of a sum of two products a*b + c*d, the only operand shape
// whose fused multiply-add nvcc chooses from the surrounding code (use
// counts after unrolling) rather than from the expression itself:
//   kFuseFirst   fma(a, b, c*d)     kFuseSecond  fma(c, d, a*b)
//   kNoFuse      a*b + c*d          kCompiler    written as a*b + c*d and
//                                                left to the compiler
enum SumMode { kFuseFirst = 0, kFuseSecond = 1, kNoFuse = 2, kCompiler = 3 };

template <int MODE>
__device__ __forceinline__ float sum_of_products(float a, float b, float c, float d) {
    if (MODE == kFuseFirst) return __fmaf_rn(a, b, __fmul_rn(c, d));
    if (MODE == kFuseSecond) return __fmaf_rn(c, d, __fmul_rn(a, b));
    if (MODE == kNoFuse) return __fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d));
    return a * b + c * d;
}

// Per-kind, per-ROI-size contraction choices of the loss (the squared
// distance of each emitter) and of the weighted-MLE mask exponent.
// SUM2 is the sum of the first two emitters' model terms (multi-emitter kinds).
// The choices below are the ones the reference kernels get from nvcc 12.9 for
// sm_100a, found by running the reference's own kernels on a B200 next to
// each explicit variant of these kernels on the same records and keeping the
// variant whose every output bit matches (tests/test_gpu_reference_parity.py
// re-checks them).  They differ between ROI sizes because nvcc's unrolling,
// and with it the use count that decides each fusion, differs.  Sizes not
// listed keep the plain expression (kCompiler).
// MODEL is amplitude * exp + background of the single-emitter kinds: the
// amplitude product is fused (its only use), the background product is not.
template <int KIND, int R>
struct ArithSpec {
    enum { DIST = kCompiler, MASK = kCompiler, SUM2 = kCompiler };
};
constexpr int kModelSum = kFuseFirst;
template <> struct ArithSpec<kGS2D, 7> { enum { DIST = kFuseFirst, MASK = kNoFuse, SUM2 = kCompiler }; };
template <> struct ArithSpec<kGS2D, 9> { enum { DIST = kFuseSecond, MASK = kCompiler, SUM2 = kCompiler }; };
template <> struct ArithSpec<kGS2D, 11> { enum { DIST = kFuseSecond, MASK = kNoFuse, SUM2 = kCompiler }; };
template <> struct ArithSpec<kGS2D, 13> { enum { DIST = kFuseSecond, MASK = kCompiler, SUM2 = kCompiler }; };
template <> struct ArithSpec<kAS3D, 7> { enum { DIST = kFuseFirst, MASK = kFuseFirst, SUM2 = kCompiler }; };
template <> struct ArithSpec<kAS3D, 9> { enum { DIST = kFuseFirst, MASK = kFuseFirst, SUM2 = kCompiler }; };
template <> struct ArithSpec<kAS3D, 11> { enum { DIST = kFuseFirst, MASK = kFuseFirst, SUM2 = kCompiler }; };
template <> struct ArithSpec<k2E, 7> { enum { DIST = kFuseFirst, MASK = kCompiler, SUM2 = kFuseFirst }; };
template <> struct ArithSpec<k2E, 11> { enum { DIST = kFuseSecond, MASK = kCompiler, SUM2 = kFuseFirst }; };
template <> struct ArithSpec<k3E, 7> { enum { DIST = kFuseSecond, MASK = kCompiler, SUM2 = kFuseFirst }; };
template <> struct ArithSpec<k3E, 11> { enum { DIST = kFuseSecond, MASK = kCompiler, SUM2 = kFuseFirst }; };
template <> struct ArithSpec<kAS3D2E, 7> { enum { DIST = kFuseFirst, MASK = kCompiler, SUM2 = kFuseFirst }; };

// Model exponential of one single-emitter parameter vector v at the pixel
// centred on (cp, rp) (GS2D: v = A, x, y, S, B; AS3D: A, x, y, Sx, Sy, B).
template <int KIND, int DIST>
__device__ __forceinline__ float single_expo(float cp, float rp, const float *v) {
    const float dx = cp - v[1], dy = rp - v[2];
    if (KIND == kGS2D) return __expf(-(sum_of_products<DIST>(dx, dx, dy, dy)) * v[3] * QCS_SSCALE);
    return __expf(-(sum_of_products<DIST>(dx * dx * v[3], QCS_SSCALE, dy * dy * v[4], QCS_SSCALE)));
}

// Poisson deviance term of one pixel given the model exponential e.
template <int KIND>
__device__ __forceinline__ float single_term(float e, const float *v, float pixval, float logpix) {
    const float IVal = sum_of_products<kModelSum>(v[0] * QCS_ASCALE, e, v[KindTraits<KIND>::P - 1], QCS_BSCALE);
    return __fmaf_rn(-pixval, __logf(IVal) - logpix, __fsub_rn(IVal, pixval));
}

template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST, int SUM2 = ArithSpec<KIND, R>::SUM2>
__device__ __forceinline__ float loss(const RoiRef &roi, float *Ininf) {
    typedef KindTraits<KIND> T;
#pragma unroll
    for (int k = 0; k < T::P; k++) {
        if (T::CLAMP001) {
            if (Ininf[k] < 0.01f) Ininf[k] = 0.01f;
        } else {
            if (Ininf[k] < 0.0f) Ininf[k] = 0.0f;
        }
    }
    float TotalLoss = 0;
#pragma unroll 1
    for (int row = 0; row < R; row++) {
#pragma unroll(R <= kUnrollMaxR ? R : 1)
        for (int col = 0; col < R; col++) {
            const float2 pl = roi.img[(row * R + col) * roi.ld];
            const float pixval = pl.x, logpix = pl.y;
            const float rowpos = row + 0.5f;
            const float colpos = col + 0.5f;
            float Loss_t;
            if (KIND == kGS2D || KIND == kAS3D) {
                Loss_t = single_term<KIND>(single_expo<KIND, DIST>(colpos, rowpos, Ininf), Ininf, pixval, logpix);
            } else if (KIND == k2E) {
                const float dx0 = colpos - Ininf[1], dy0 = rowpos - Ininf[2];
                const float dx1 = colpos - Ininf[4], dy1 = rowpos - Ininf[5];
                const float A0 = Ininf[0] * QCS_ASCALE, A1 = Ininf[3] * QCS_ASCALE;
                const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * Ininf[6] * QCS_SSCALE);
                const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * Ininf[6] * QCS_SSCALE);
                float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + Ininf[7] * QCS_BSCALE;
                Loss_t = IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
            } else if (KIND == k3E) {
                const float dx0 = colpos - Ininf[1], dy0 = rowpos - Ininf[2];
                const float dx1 = colpos - Ininf[4], dy1 = rowpos - Ininf[5];
                const float dx2 = colpos - Ininf[7], dy2 = rowpos - Ininf[8];
                const float A0 = Ininf[0] * QCS_ASCALE, A1 = Ininf[3] * QCS_ASCALE, A2 = Ininf[6] * QCS_ASCALE;
                const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * Ininf[9] * QCS_SSCALE);
                const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * Ininf[9] * QCS_SSCALE);
                const float e2 = __expf(-(sum_of_products<DIST>(dx2, dx2, dy2, dy2)) * Ininf[9] * QCS_SSCALE);
                float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + A2 * e2 + Ininf[10] * QCS_BSCALE;
                Loss_t = IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
            } else {  // kAS3D2E
                const float dx0 = colpos - Ininf[1], dy0 = rowpos - Ininf[2];
                const float dx1 = colpos - Ininf[6], dy1 = rowpos - Ininf[7];
                const float A0 = Ininf[0] * QCS_ASCALE, A1 = Ininf[5] * QCS_ASCALE;
                const float e0 = __expf(-(sum_of_products<DIST>(dx0 * dx0 * Ininf[3], QCS_SSCALE, dy0 * dy0 * Ininf[4],
                                                                QCS_SSCALE)));
                const float e1 = __expf(-(sum_of_products<DIST>(dx1 * dx1 * Ininf[8], QCS_SSCALE, dy1 * dy1 * Ininf[9],
                                                                QCS_SSCALE)));
                float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + Ininf[10] * QCS_BSCALE;
                Loss_t = IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
            }
            if (T::WEIGHTED)
                TotalLoss = __fmaf_rn(roi.w[(row * R + col) * roi.ld], Loss_t, TotalLoss);
            else
                TotalLoss = __fadd_rn(TotalLoss, Loss_t);
        }
    }
    return TotalLoss;
}

// Central difference on a working copy; each loss call clamps the copy in
// place and later parameters see the clamped values, as in the reference.
template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST, int SUM2 = ArithSpec<KIND, R>::SUM2>
__device__ __forceinline__ void numerical_gradient(const RoiRef &roi, const float *Ininf, float *grad) {
    enum { P = KindTraits<KIND>::P };
    float tIninf[P];
#pragma unroll
    for (int cnt = 0; cnt < P; cnt++) tIninf[cnt] = Ininf[cnt];
    for (int cnt = 0; cnt < P; cnt++) {
        tIninf[cnt] = tIninf[cnt] - 0.002f;
        float tgradn = loss<R, KIND, DIST, SUM2>(roi, tIninf);
        tIninf[cnt] = tIninf[cnt] + 0.004f;
        float tgradp = loss<R, KIND, DIST, SUM2>(roi, tIninf);
        grad[cnt] = (tgradp - tgradn) * 250.0f;
        tIninf[cnt] = tIninf[cnt] - 0.002f;
    }
}

// The central-difference gradient of the single-emitter kinds in one sweep
// over the pixels: the 2P evaluation points are first replayed exactly as
// numerical_gradient produces them (with its in-place clamping), then every
// pixel is loaded once and each point's deviance accumulated in its own sum,
// in pixel order.  The amplitude and background points leave the exponent's
// inputs (x, y, widths) unchanged, so their exponential is the base point's;
// this is checked bit for bit per ROI, and a warp with any ROI where it does
// not hold falls back to the point-by-point gradient.  Each sum therefore
// equals the separate loss evaluation bit for bit.
template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST>
__device__ __forceinline__ void numerical_gradient_shared(const RoiRef &roi, const float *Ininf, float *grad) {
    typedef KindTraits<KIND> T;
    enum { P = T::P, NE = 2 * P };
    float v[NE][P];
    {
        float t[P];
#pragma unroll
        for (int k = 0; k < P; k++) t[k] = Ininf[k];
#pragma unroll
        for (int k = 0; k < P; k++) {
            t[k] = t[k] - 0.002f;
#pragma unroll
            for (int c = 0; c < P; c++) {
                if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                v[2 * k][c] = t[c];
            }
            t[k] = t[k] + 0.004f;
#pragma unroll
            for (int c = 0; c < P; c++) {
                if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                v[2 * k + 1][c] = t[c];
            }
            t[k] = t[k] - 0.002f;
        }
    }
    bool share = true;
#pragma unroll
    for (int c = 1; c < P - 1; c++) {
        const unsigned b = __float_as_uint(v[0][c]);
        share = share && (__float_as_uint(v[1][c]) == b) && (__float_as_uint(v[NE - 2][c]) == b) &&
                (__float_as_uint(v[NE - 1][c]) == b);
    }
    if (!__all_sync(__activemask(), share)) {
        numerical_gradient<R, KIND, DIST>(roi, Ininf, grad);
        return;
    }
    float tot[NE];
#pragma unroll
    for (int j = 0; j < NE; j++) tot[j] = 0;
#pragma unroll 1
    for (int row = 0; row < R; row++) {
#pragma unroll(R <= kUnrollMaxR ? R : 1)
        for (int col = 0; col < R; col++) {
            const float2 pl = roi.img[(row * R + col) * roi.ld];
            const float pixval = pl.x, logpix = pl.y;
            const float w = T::WEIGHTED ? roi.w[(row * R + col) * roi.ld] : 1.0f;
            const float rowpos = row + 0.5f;
            const float colpos = col + 0.5f;
            const float e_base = single_expo<KIND, DIST>(colpos, rowpos, v[0]);
#pragma unroll
            for (int j = 0; j < NE; j++) {
                const bool base = (j < 2) || (j >= NE - 2);
                const float e = base ? e_base : single_expo<KIND, DIST>(colpos, rowpos, v[j]);
                const float Lt = single_term<KIND>(e, v[j], pixval, logpix);
                tot[j] = T::WEIGHTED ? __fmaf_rn(w, Lt, tot[j]) : __fadd_rn(tot[j], Lt);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < P; k++) grad[k] = (tot[2 * k + 1] - tot[2 * k]) * 250.0f;
}

// D <- (I - s y'/(y's)) D (I - y s'/(y's)) + s s'/(y's); D is row-major P x P
// at D[(r * P + c) * ld].
template <int P>
__device__ __forceinline__ void bfgs_update(float *D, int ld, const float *sk, const float *yk) {
    float divdat = 0;
#pragma unroll
    for (int cnt = 0; cnt < P; cnt++) divdat += sk[cnt] * yk[cnt];
    divdat = 1.0f / divdat;
    float tdat10[P], tdat20[P];
#pragma unroll
    for (int cnt = 0; cnt < P; cnt++) {
        tdat10[cnt] = yk[cnt] * divdat;
        tdat20[cnt] = sk[cnt] * divdat;
    }
    float skyk[P][P], sksk[P][P], tD0[P][P];
#pragma unroll
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int col = 0; col < P; col++) {
            if (row == col)
                skyk[row][col] = 1.0f - sk[row] * tdat10[col];
            else
                skyk[row][col] = 0.0f - sk[row] * tdat10[col];
            sksk[row][col] = sk[row] * tdat20[col];
        }
    }
#pragma unroll
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int col = 0; col < P; col++) {
            tD0[row][col] = 0;
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) tD0[row][col] += skyk[row][cnt] * D[(cnt * P + col) * ld];
        }
    }
#pragma unroll
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int col = 0; col < P; col++) {
            float acc = 0;
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) acc += tD0[row][cnt] * skyk[col][cnt];
            D[(row * P + col) * ld] = acc;
        }
    }
#pragma unroll
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int cnt = 0; cnt < P; cnt++) D[(row * P + cnt) * ld] = D[(row * P + cnt) * ld] + sksk[row][cnt];
    }
}

template <int R, int KIND, int DIST, int SUM2>
__device__ __forceinline__ void gradient(const RoiRef &roi, const float *Ininf, float *grad) {
    if (KIND == kGS2D || KIND == kAS3D)
        numerical_gradient_shared<R, KIND, DIST>(roi, Ininf, grad);
    else
        numerical_gradient<R, KIND, DIST, SUM2>(roi, Ininf, grad);
}

// Loss and gradient of one ROI evaluated by its own thread.
template <int R, int KIND, int DIST, int SUM2>
struct ThreadEval {
    RoiRef roi;
    __device__ __forceinline__ float loss(float *x) const { return qcs::loss<R, KIND, DIST, SUM2>(roi, x); }
    __device__ __forceinline__ void gradient(const float *x, float *g) const {
        qcs::gradient<R, KIND, DIST, SUM2>(roi, x, g);
    }
};

// GS2D loss of ThreadEval with the analytic gradient in one pass over the
// pixels (learned-start fits; the reference's fits use the central
// difference).  With mu = 128 A e + 64 B, e = exp(-0.1 S r^2), r^2 = dx^2 +
// dy^2, dx = col + 0.5 - X, and the weighted deviance sum w (mu - n - n ln
// mu/n), each parameter's derivative is sum w (1 - n / mu) dmu/dtheta:
//   dmu/dA = 128 e, dmu/dX = 128 A e 0.2 S dx, dmu/dY = 128 A e 0.2 S dy,
//   dmu/dS = -128 A e 0.1 r^2, dmu/dB = 64,
// at the point clamped as the loss clamps it.  One exponential and one
// division per pixel instead of the central difference's ten losses.
template <int R, int DIST>
struct AnalyticEvalGS2D {
    RoiRef roi;
    __device__ __forceinline__ float loss(float *x) const {
        return qcs::loss<R, kGS2D, DIST, ArithSpec<kGS2D, R>::SUM2>(roi, x);
    }
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        float c[5];
#pragma unroll
        for (int k = 0; k < 5; k++) c[k] = v[k] < 0.0f ? 0.0f : v[k];
        const float A128 = c[0] * QCS_ASCALE, B64 = c[4] * QCS_BSCALE, S01 = c[3] * QCS_SSCALE;
        float gA = 0, gX = 0, gY = 0, gS = 0, gB = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
            const float dy = (row + 0.5f) - c[2];
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(row * R + col) * roi.ld];
                const float w = roi.w[(row * R + col) * roi.ld];
                const float dx = (col + 0.5f) - c[1];
                const float r2 = __fmaf_rn(dx, dx, dy * dy);
                const float e = __expf(-r2 * S01);
                const float mu = __fmaf_rn(A128, e, B64);
                const float q = w * (1.0f - __fdividef(pl.x, mu));
                const float qe = q * e;
                gA += qe;
                gX = __fmaf_rn(qe, dx, gX);
                gY = __fmaf_rn(qe, dy, gY);
                gS = __fmaf_rn(qe, r2, gS);
                gB += q;
            }
        }
        g[0] = QCS_ASCALE * gA;
        g[1] = A128 * 2.0f * S01 * gX;
        g[2] = A128 * 2.0f * S01 * gY;
        g[3] = -A128 * QCS_SSCALE * gS;
        g[4] = QCS_BSCALE * gB;
    }
};

// The same for AS3D (separate widths): with mu = 128 A e + 64 B,
// e = exp(-0.1 (Sx dx^2 + Sy dy^2)),
//   dmu/dA = 128 e, dmu/dX = 128 A e 0.2 Sx dx, dmu/dY = 128 A e 0.2 Sy dy,
//   dmu/dSx = -128 A e 0.1 dx^2, dmu/dSy = -128 A e 0.1 dy^2, dmu/dB = 64,
// at the point clamped as the AS3D loss clamps it (every parameter >= 0.01).
template <int R, int DIST>
struct AnalyticEvalAS3D {
    RoiRef roi;
    __device__ __forceinline__ float loss(float *x) const {
        return qcs::loss<R, kAS3D, DIST, ArithSpec<kAS3D, R>::SUM2>(roi, x);
    }
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        float c[6];
#pragma unroll
        for (int k = 0; k < 6; k++) c[k] = v[k] < 0.01f ? 0.01f : v[k];
        const float A128 = c[0] * QCS_ASCALE, B64 = c[5] * QCS_BSCALE;
        const float Sx = c[3] * QCS_SSCALE, Sy = c[4] * QCS_SSCALE;
        float gA = 0, gX = 0, gY = 0, gSx = 0, gSy = 0, gB = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
            const float dy = (row + 0.5f) - c[2];
            const float qy = dy * dy;
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(row * R + col) * roi.ld];
                const float w = roi.w[(row * R + col) * roi.ld];
                const float dx = (col + 0.5f) - c[1];
                const float qx = dx * dx;
                const float e = __expf(-__fmaf_rn(qx, Sx, qy * Sy));
                const float mu = __fmaf_rn(A128, e, B64);
                const float q = w * (1.0f - __fdividef(pl.x, mu));
                const float qe = q * e;
                gA += qe;
                gX = __fmaf_rn(qe, dx, gX);
                gY = __fmaf_rn(qe, dy, gY);
                gSx = __fmaf_rn(qe, qx, gSx);
                gSy = __fmaf_rn(qe, qy, gSy);
                gB += q;
            }
        }
        g[0] = QCS_ASCALE * gA;
        g[1] = A128 * 2.0f * Sx * gX;
        g[2] = A128 * 2.0f * Sy * gY;
        g[3] = -A128 * QCS_SSCALE * gSx;
        g[4] = -A128 * QCS_SSCALE * gSy;
        g[5] = QCS_BSCALE * gB;
    }
};


// The two-emitter GS2D loss (shared S and B, the loss the 2E fit minimises)
// with its analytic gradient: mu = 128 (A0 e0 + A1 e1) + 64 B,
// ek = exp(-0.1 S rk^2), and with q = w (1 - n / mu)
//   dA_k = 128 sum q ek, dX_k = 128 A_k 0.2 S sum q ek dx_k (same for Y),
//   dS = -12.8 sum q (A0 e0 r0^2 + A1 e1 r1^2), dB = 64 sum q,
// at the point clamped as the loss clamps it (parameters >= 0).
template <int R, int DIST>
struct AnalyticEval2E {
    RoiRef roi;
    __device__ __forceinline__ float loss(float *x) const {
        return qcs::loss<R, k2E, DIST, ArithSpec<k2E, R>::SUM2>(roi, x);
    }
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        float c[8];
#pragma unroll
        for (int k = 0; k < 8; k++) c[k] = v[k] < 0.0f ? 0.0f : v[k];
        const float A0 = c[0] * QCS_ASCALE, A1 = c[3] * QCS_ASCALE, S01 = c[6] * QCS_SSCALE, B64 = c[7] * QCS_BSCALE;
        float gA0 = 0, gX0 = 0, gY0 = 0, gA1 = 0, gX1 = 0, gY1 = 0, gS = 0, gB = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
            const float dy0 = (row + 0.5f) - c[2], dy1 = (row + 0.5f) - c[5];
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(row * R + col) * roi.ld];
                const float w = roi.w[(row * R + col) * roi.ld];
                const float dx0 = (col + 0.5f) - c[1], dx1 = (col + 0.5f) - c[4];
                const float r0 = __fmaf_rn(dx0, dx0, dy0 * dy0), r1 = __fmaf_rn(dx1, dx1, dy1 * dy1);
                const float e0 = __expf(-r0 * S01), e1 = __expf(-r1 * S01);
                const float mu = __fmaf_rn(A0, e0, __fmaf_rn(A1, e1, B64));
                const float q = w * (1.0f - __fdividef(pl.x, mu));
                const float q0 = q * e0, q1 = q * e1;
                gA0 += q0;
                gX0 = __fmaf_rn(q0, dx0, gX0);
                gY0 = __fmaf_rn(q0, dy0, gY0);
                gA1 += q1;
                gX1 = __fmaf_rn(q1, dx1, gX1);
                gY1 = __fmaf_rn(q1, dy1, gY1);
                gS = __fmaf_rn(A0 * q0, r0, __fmaf_rn(A1 * q1, r1, gS));
                gB += q;
            }
        }
        g[0] = QCS_ASCALE * gA0;
        g[1] = A0 * 2.0f * S01 * gX0;
        g[2] = A0 * 2.0f * S01 * gY0;
        g[3] = QCS_ASCALE * gA1;
        g[4] = A1 * 2.0f * S01 * gX1;
        g[5] = A1 * 2.0f * S01 * gY1;
        g[6] = -QCS_SSCALE * gS;
        g[7] = QCS_BSCALE * gB;
    }
};
// Loss of the GS2D three-emitter fit (the plain kernel's, unweighted) with
// the analytic gradient of that Poisson deviance: d/d mu = 1 - n / mu per
// pixel, chained through the three Gaussians sharing 1/(2 sigma^2) and the
// background (the learned-start three-emitter fit; no central differences).
template <int R, int DIST>
struct AnalyticEval3E {
    RoiRef roi;
    __device__ __forceinline__ float loss(float *x) const {
        return qcs::loss<R, k3E, DIST, ArithSpec<k3E, R>::SUM2>(roi, x);
    }
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        float c[11];
#pragma unroll
        for (int k = 0; k < 11; k++) c[k] = v[k] < 0.0f ? 0.0f : v[k];
        const float A0 = c[0] * QCS_ASCALE, A1 = c[3] * QCS_ASCALE, A2 = c[6] * QCS_ASCALE;
        const float S = c[9] * QCS_SSCALE, B64 = c[10] * QCS_BSCALE;
        float gA0 = 0, gX0 = 0, gY0 = 0, gA1 = 0, gX1 = 0, gY1 = 0, gA2 = 0, gX2 = 0, gY2 = 0, gS = 0, gB = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
            const float dy0 = (row + 0.5f) - c[2], dy1 = (row + 0.5f) - c[5], dy2 = (row + 0.5f) - c[8];
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(row * R + col) * roi.ld];
                const float dx0 = (col + 0.5f) - c[1], dx1 = (col + 0.5f) - c[4], dx2 = (col + 0.5f) - c[7];
                const float r0 = __fmaf_rn(dx0, dx0, dy0 * dy0), r1 = __fmaf_rn(dx1, dx1, dy1 * dy1);
                const float r2 = __fmaf_rn(dx2, dx2, dy2 * dy2);
                const float e0 = __expf(-r0 * S), e1 = __expf(-r1 * S), e2 = __expf(-r2 * S);
                const float mu = __fmaf_rn(A0, e0, __fmaf_rn(A1, e1, __fmaf_rn(A2, e2, B64)));
                const float q = 1.0f - __fdividef(pl.x, mu);
                const float q0 = q * e0, q1 = q * e1, q2 = q * e2;
                gA0 += q0;
                gX0 = __fmaf_rn(q0, dx0, gX0);
                gY0 = __fmaf_rn(q0, dy0, gY0);
                gA1 += q1;
                gX1 = __fmaf_rn(q1, dx1, gX1);
                gY1 = __fmaf_rn(q1, dy1, gY1);
                gA2 += q2;
                gX2 = __fmaf_rn(q2, dx2, gX2);
                gY2 = __fmaf_rn(q2, dy2, gY2);
                gS = __fmaf_rn(A0 * q0, r0, __fmaf_rn(A1 * q1, r1, __fmaf_rn(A2 * q2, r2, gS)));
                gB += q;
            }
        }
        g[0] = QCS_ASCALE * gA0;
        g[1] = A0 * 2.0f * S * gX0;
        g[2] = A0 * 2.0f * S * gY0;
        g[3] = QCS_ASCALE * gA1;
        g[4] = A1 * 2.0f * S * gX1;
        g[5] = A1 * 2.0f * S * gY1;
        g[6] = QCS_ASCALE * gA2;
        g[7] = A2 * 2.0f * S * gX2;
        g[8] = A2 * 2.0f * S * gY2;
        g[9] = -QCS_SSCALE * gS;
        g[10] = QCS_BSCALE * gB;
    }
};

// Loss and gradient of one single-emitter ROI (GS2D / AS3D) evaluated by a
// group of G consecutive lanes of a warp, bit for bit equal to ThreadEval:
//  - loss: the lanes compute the pixel terms k = lane, lane + G, ... (the
//    same expressions as loss()) into the ROI's scratch row; then every lane
//    accumulates the row in pixel order with the same fused multiply-adds,
//    so all lanes hold the serial sum;
//  - gradient: the 2P central-difference points are replayed as
//    numerical_gradient does (in-place clamping); lane l accumulates the
//    sums of points l, l + G, ... over all pixels in pixel order.  Each
//    point evaluates its own exponential, which equals the shared one of
//    numerical_gradient_shared whenever that one applies.
// img / w / part: the ROI's PIX (value, log) pairs, weights and scratch,
// contiguous and 16-byte aligned; mask: the group's lanes.  The sums equal
// the serial kernel's only where the pixel distance's contraction is fixed in
// the source (DIST != kCompiler).
template <int R, int KIND, int DIST, int G>
struct GroupEval {
    const float2 *img;
    const float *w;
    float *part;
    int lane;
    unsigned mask;

    __device__ __forceinline__ float loss(float *Ininf) const {
        typedef KindTraits<KIND> T;
        enum { PIX = R * R };
#pragma unroll
        for (int k = 0; k < T::P; k++) {
            if (T::CLAMP001) {
                if (Ininf[k] < 0.01f) Ininf[k] = 0.01f;
            } else {
                if (Ininf[k] < 0.0f) Ininf[k] = 0.0f;
            }
        }
#pragma unroll
        for (int i = 0; i < (PIX + G - 1) / G; i++) {
            const int k = lane + i * G;
            if (k < PIX) {
                const int row = k / R, col = k - (k / R) * R;
                const float2 pl = img[k];
                part[k] = single_term<KIND>(single_expo<KIND, DIST>(col + 0.5f, row + 0.5f, Ininf), Ininf, pl.x,
                                            pl.y);
            }
        }
        __syncwarp(mask);
        float TotalLoss = 0;
        const float4 *w4 = reinterpret_cast<const float4 *>(w);
        const float4 *p4 = reinterpret_cast<const float4 *>(part);
#pragma unroll
        for (int q = 0; q < PIX / 4; q++) {
            const float4 a = w4[q], t = p4[q];
            TotalLoss = __fmaf_rn(a.x, t.x, TotalLoss);
            TotalLoss = __fmaf_rn(a.y, t.y, TotalLoss);
            TotalLoss = __fmaf_rn(a.z, t.z, TotalLoss);
            TotalLoss = __fmaf_rn(a.w, t.w, TotalLoss);
        }
#pragma unroll
        for (int k = PIX / 4 * 4; k < PIX; k++) TotalLoss = __fmaf_rn(w[k], part[k], TotalLoss);
        __syncwarp(mask);
        return TotalLoss;
    }

    __device__ __forceinline__ void gradient(const float *Ininf, float *grad) const {
        typedef KindTraits<KIND> T;
        enum { P = T::P, NE = 2 * P, NC = (NE + G - 1) / G, PIX = R * R };
        float v[NC][P] = {};
        {
            float t[P];
#pragma unroll
            for (int k = 0; k < P; k++) t[k] = Ininf[k];
#pragma unroll
            for (int k = 0; k < P; k++) {
                t[k] = t[k] - 0.002f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                }
#pragma unroll
                for (int j = 0; j < NC; j++)
                    if (lane + j * G == 2 * k)
#pragma unroll
                        for (int c = 0; c < P; c++) v[j][c] = t[c];
                t[k] = t[k] + 0.004f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                }
#pragma unroll
                for (int j = 0; j < NC; j++)
                    if (lane + j * G == 2 * k + 1)
#pragma unroll
                        for (int c = 0; c < P; c++) v[j][c] = t[c];
                t[k] = t[k] - 0.002f;
            }
        }
        float tot[NC];
#pragma unroll
        for (int j = 0; j < NC; j++) tot[j] = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = img[row * R + col];
                const float wk = w[row * R + col];
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    if (lane + j * G < NE) {
                        const float e = single_expo<KIND, DIST>(col + 0.5f, row + 0.5f, v[j]);
                        tot[j] = __fmaf_rn(wk, single_term<KIND>(e, v[j], pl.x, pl.y), tot[j]);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < P; k++) {
            const float tn = __shfl_sync(mask, tot[(2 * k) / G], (2 * k) % G, G);
            const float tp = __shfl_sync(mask, tot[(2 * k + 1) / G], (2 * k + 1) % G, G);
            grad[k] = (tp - tn) * 250.0f;
        }
    }
};

// Poisson deviance term of one pixel of the multi-emitter kinds at the
// parameters v: the expressions of loss(), term for term.
template <int KIND, int DIST, int SUM2>
__device__ __forceinline__ float multi_term(float colpos, float rowpos, const float *v, float pixval, float logpix) {
    if (KIND == k2E) {
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[4], dy1 = rowpos - v[5];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * v[6] * QCS_SSCALE);
        const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * v[6] * QCS_SSCALE);
        float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + v[7] * QCS_BSCALE;
        return IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
    } else if (KIND == k3E) {
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[4], dy1 = rowpos - v[5];
        const float dx2 = colpos - v[7], dy2 = rowpos - v[8];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE, A2 = v[6] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * v[9] * QCS_SSCALE);
        const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * v[9] * QCS_SSCALE);
        const float e2 = __expf(-(sum_of_products<DIST>(dx2, dx2, dy2, dy2)) * v[9] * QCS_SSCALE);
        float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + A2 * e2 + v[10] * QCS_BSCALE;
        return IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
    } else {  // kAS3D2E
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[6], dy1 = rowpos - v[7];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[5] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0 * dx0 * v[3], QCS_SSCALE, dy0 * dy0 * v[4], QCS_SSCALE)));
        const float e1 = __expf(-(sum_of_products<DIST>(dx1 * dx1 * v[8], QCS_SSCALE, dy1 * dy1 * v[9], QCS_SSCALE)));
        float IVal_all = sum_of_products<SUM2>(A0, e0, A1, e1) + v[10] * QCS_BSCALE;
        return IVal_all - pixval - pixval * (__logf(IVal_all) - logpix);
    }
}

// The same loss and analytic gradient evaluated by one warp: lane l sums the
// pixels l, l + 32, ...; each sum is reduced by a shuffle tree and lane 0's
// total broadcast, so every lane holds the same value (the lanes' BFGS steps
// stay identical).  img: the ROI's PIX (value, log) pairs, contiguous.
template <int R>
struct AnalyticWarpEval3E {
    const float2 *img;
    int lane;
    unsigned mask;
    __device__ __forceinline__ float uniform_sum(float v) const {
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(mask, v, m);
        return __shfl_sync(mask, v, 0);
    }
    __device__ __forceinline__ float loss(float *x) const {
#pragma unroll
        for (int k = 0; k < 11; k++)
            if (x[k] < 0.0f) x[k] = 0.0f;
        float s = 0.0f;
        for (int k = lane; k < R * R; k += 32) {
            const int row = k / R, col = k - row * R;
            const float2 pl = img[k];
            s += multi_term<k3E, ArithSpec<k3E, R>::DIST, ArithSpec<k3E, R>::SUM2>(col + 0.5f, row + 0.5f, x, pl.x,
                                                                                  pl.y);
        }
        return uniform_sum(s);
    }
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        float c[11];
#pragma unroll
        for (int k = 0; k < 11; k++) c[k] = v[k] < 0.0f ? 0.0f : v[k];
        const float A[3] = {c[0] * QCS_ASCALE, c[3] * QCS_ASCALE, c[6] * QCS_ASCALE};
        const float S = c[9] * QCS_SSCALE, B64 = c[10] * QCS_BSCALE;
        float gA[3] = {0, 0, 0}, gX[3] = {0, 0, 0}, gY[3] = {0, 0, 0}, gS = 0, gB = 0;
        for (int k = lane; k < R * R; k += 32) {
            const int row = k / R, col = k - row * R;
            const float2 pl = img[k];
            float dx[3], dy[3], r[3], e[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                dx[j] = (col + 0.5f) - c[3 * j + 1];
                dy[j] = (row + 0.5f) - c[3 * j + 2];
                r[j] = __fmaf_rn(dx[j], dx[j], dy[j] * dy[j]);
                e[j] = __expf(-r[j] * S);
            }
            const float mu = __fmaf_rn(A[0], e[0], __fmaf_rn(A[1], e[1], __fmaf_rn(A[2], e[2], B64)));
            const float q = 1.0f - __fdividef(pl.x, mu);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const float qj = q * e[j];
                gA[j] += qj;
                gX[j] = __fmaf_rn(qj, dx[j], gX[j]);
                gY[j] = __fmaf_rn(qj, dy[j], gY[j]);
                gS = __fmaf_rn(A[j] * qj, r[j], gS);
            }
            gB += q;
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
            g[3 * j] = QCS_ASCALE * uniform_sum(gA[j]);
            g[3 * j + 1] = A[j] * 2.0f * S * uniform_sum(gX[j]);
            g[3 * j + 2] = A[j] * 2.0f * S * uniform_sum(gY[j]);
        }
        g[9] = -QCS_SSCALE * uniform_sum(gS);
        g[10] = QCS_BSCALE * uniform_sum(gB);
    }
};

// Loss and gradient of one multi-emitter ROI (2E, 3E, AS3D-2E) evaluated by
// a group of G consecutive lanes, bit for bit equal to ThreadEval:
//  - loss: lane l computes the pixel terms k = l, l + G, ... (multi_term)
//    into the ROI's scratch row; then every lane sums the row in pixel order
//    with the thread kernel's operations (the weighted 2E fit: fused
//    multiply-adds with the mask; 3E and AS3D-2E: plain adds);
//  - gradient: the 2P central-difference points are replayed as
//    numerical_gradient produces them (each loss call clamps its point in
//    place and the next point starts from the clamped values); lane l sums
//    points l, l + G, ... over all pixels in pixel order, and the lanes
//    exchange the sums.
// img / w / part: the ROI's pixels, mask and scratch, contiguous and 16-byte
// aligned; mask: the group's lanes.  Only for roundings fixed in the source
// (DIST, SUM2 != kCompiler).
template <int R, int KIND, int DIST, int SUM2, int G>
struct MultiGroupEval {
    const float2 *img;
    const float *w;
    float *part;
    int lane;
    unsigned mask;

    __device__ __forceinline__ float loss(float *Ininf) const {
        typedef KindTraits<KIND> T;
        enum { PIX = R * R };
#pragma unroll
        for (int k = 0; k < T::P; k++) {
            if (T::CLAMP001) {
                if (Ininf[k] < 0.01f) Ininf[k] = 0.01f;
            } else {
                if (Ininf[k] < 0.0f) Ininf[k] = 0.0f;
            }
        }
#pragma unroll
        for (int i = 0; i < (PIX + G - 1) / G; i++) {
            const int k = lane + i * G;
            if (k < PIX) {
                const int row = k / R, col = k - (k / R) * R;
                const float2 pl = img[k];
                part[k] = multi_term<KIND, DIST, SUM2>(col + 0.5f, row + 0.5f, Ininf, pl.x, pl.y);
            }
        }
        __syncwarp(mask);
        float TotalLoss = 0;
        const float4 *p4 = reinterpret_cast<const float4 *>(part);
        if (T::WEIGHTED) {
            const float4 *w4 = reinterpret_cast<const float4 *>(w);
#pragma unroll 8
            for (int q = 0; q < PIX / 4; q++) {
                const float4 a = w4[q], t = p4[q];
                TotalLoss = __fmaf_rn(a.x, t.x, TotalLoss);
                TotalLoss = __fmaf_rn(a.y, t.y, TotalLoss);
                TotalLoss = __fmaf_rn(a.z, t.z, TotalLoss);
                TotalLoss = __fmaf_rn(a.w, t.w, TotalLoss);
            }
#pragma unroll
            for (int k = PIX / 4 * 4; k < PIX; k++) TotalLoss = __fmaf_rn(w[k], part[k], TotalLoss);
        } else {
#pragma unroll 8
            for (int q = 0; q < PIX / 4; q++) {
                const float4 t = p4[q];
                TotalLoss = __fadd_rn(TotalLoss, t.x);
                TotalLoss = __fadd_rn(TotalLoss, t.y);
                TotalLoss = __fadd_rn(TotalLoss, t.z);
                TotalLoss = __fadd_rn(TotalLoss, t.w);
            }
#pragma unroll
            for (int k = PIX / 4 * 4; k < PIX; k++) TotalLoss = __fadd_rn(TotalLoss, part[k]);
        }
        __syncwarp(mask);
        return TotalLoss;
    }

    __device__ __forceinline__ void gradient(const float *Ininf, float *grad) const {
        typedef KindTraits<KIND> T;
        enum { P = T::P, NE = 2 * P, NC = (NE + G - 1) / G, PIX = R * R };
        float v[NC][P] = {};
        {
            float t[P];
#pragma unroll
            for (int k = 0; k < P; k++) t[k] = Ininf[k];
#pragma unroll
            for (int k = 0; k < P; k++) {
                t[k] = t[k] - 0.002f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                }
#pragma unroll
                for (int j = 0; j < NC; j++)
                    if (lane + j * G == 2 * k)
#pragma unroll
                        for (int c = 0; c < P; c++) v[j][c] = t[c];
                t[k] = t[k] + 0.004f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                }
#pragma unroll
                for (int j = 0; j < NC; j++)
                    if (lane + j * G == 2 * k + 1)
#pragma unroll
                        for (int c = 0; c < P; c++) v[j][c] = t[c];
                t[k] = t[k] - 0.002f;
            }
        }
        float tot[NC];
#pragma unroll
        for (int j = 0; j < NC; j++) tot[j] = 0;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
#pragma unroll(R <= kUnrollMaxR ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = img[row * R + col];
                const float wk = T::WEIGHTED ? w[row * R + col] : 1.0f;
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    if (lane + j * G < NE) {
                        const float Lt = multi_term<KIND, DIST, SUM2>(col + 0.5f, row + 0.5f, v[j], pl.x, pl.y);
                        tot[j] = T::WEIGHTED ? __fmaf_rn(wk, Lt, tot[j]) : __fadd_rn(tot[j], Lt);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < P; k++) {
            const float tn = __shfl_sync(mask, tot[(2 * k) / G], (2 * k) % G, G);
            const float tp = __shfl_sync(mask, tot[(2 * k + 1) / G], (2 * k + 1) % G, G);
            grad[k] = (tp - tn) * 250.0f;
        }
    }
};

// Expected photoelectrons of pixel (colpos, rowpos) under the model at the
// parameters v (fit units): the model value of loss(), expression for
// expression.
template <int KIND, int DIST, int SUM2>
__device__ __forceinline__ float model_value(float colpos, float rowpos, const float *v) {
    if (KIND == kGS2D || KIND == kAS3D) {
        const float e = single_expo<KIND, DIST>(colpos, rowpos, v);
        return sum_of_products<kModelSum>(v[0] * QCS_ASCALE, e, v[KindTraits<KIND>::P - 1], QCS_BSCALE);
    } else if (KIND == k2E) {
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[4], dy1 = rowpos - v[5];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * v[6] * QCS_SSCALE);
        const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * v[6] * QCS_SSCALE);
        return sum_of_products<SUM2>(A0, e0, A1, e1) + v[7] * QCS_BSCALE;
    } else if (KIND == k3E) {
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[4], dy1 = rowpos - v[5];
        const float dx2 = colpos - v[7], dy2 = rowpos - v[8];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE, A2 = v[6] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0, dx0, dy0, dy0)) * v[9] * QCS_SSCALE);
        const float e1 = __expf(-(sum_of_products<DIST>(dx1, dx1, dy1, dy1)) * v[9] * QCS_SSCALE);
        const float e2 = __expf(-(sum_of_products<DIST>(dx2, dx2, dy2, dy2)) * v[9] * QCS_SSCALE);
        return sum_of_products<SUM2>(A0, e0, A1, e1) + A2 * e2 + v[10] * QCS_BSCALE;
    } else {  // kAS3D2E
        const float dx0 = colpos - v[1], dy0 = rowpos - v[2];
        const float dx1 = colpos - v[6], dy1 = rowpos - v[7];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[5] * QCS_ASCALE;
        const float e0 = __expf(-(sum_of_products<DIST>(dx0 * dx0 * v[3], QCS_SSCALE, dy0 * dy0 * v[4], QCS_SSCALE)));
        const float e1 = __expf(-(sum_of_products<DIST>(dx1 * dx1 * v[8], QCS_SSCALE, dy1 * dy1 * v[9], QCS_SSCALE)));
        return sum_of_products<SUM2>(A0, e0, A1, e1) + v[10] * QCS_BSCALE;
    }
}

// Unweighted Poisson log-likelihood of the model at the fitted parameters Ininf
// over pixels k0, k0 + step, ... of the ROI (pixel k's (value, log) pair at
// img[k * ld]): sum n ln(mu) - mu, accumulated in FP64 (the data's ln n!
// term is common to every model of the ROI and left out).  The parameters are
// clamped as the loss clamps them.
template <int R, int KIND, int DIST, int SUM2>
__device__ __forceinline__ double model_loglik(const float2 *img, int ld, const float *Ininf, int k0, int step) {
    typedef KindTraits<KIND> T;
    float v[T::P];
#pragma unroll
    for (int k = 0; k < T::P; k++) v[k] = T::CLAMP001 ? fmaxf(Ininf[k], 0.01f) : fmaxf(Ininf[k], 0.0f);
    double s = 0.0;
    for (int k = k0; k < R * R; k += step) {
        const int row = k / R, col = k - (k / R) * R;
        const double mu = (double)model_value<KIND, DIST, SUM2>(col + 0.5f, row + 0.5f, v);
        s += (double)img[k * ld].x * log(mu) - mu;
    }
    return s;
}

// ------------------------------------------ staged single-emitter eval ---
// The weighted-MLE mask of an R x R ROI depends on |col - R/2| and
// |row - R/2| only: its exponent holds the squared distances of the pixel
// centre from the ROI centre, which are equal (exact small numbers) for
// mirrored pixels.  A thread therefore keeps U x U values (U = R/2 + 1);
// mask row ur is C4 float4 chunks, value (ur, uc) in chunk uc / 4, lane uc % 4.
// That holds where the mask's contraction is fixed in the source (MASK !=
// kCompiler).  Where nvcc chooses it, its choice differs between pixels (and
// with the surrounding code), so mirrored pixels need not agree bit for bit:
// there (FULL) the whole R x R mask of wle_weights is kept, pixel k at
// k * ld floats, which reproduces the reference's values.
template <int R, bool FULL = false>
struct MaskShape {
    enum { U = R / 2 + 1, C4 = (U + 3) / 4, FLOATS = FULL ? R * R : U * C4 * 4 };
};

__host__ __device__ constexpr int mirror_index(int k, int R) { return k < R / 2 ? R / 2 - k : k - R / 2; }

// wle_weights for the pixels col, row >= R/2 (same expressions, so the same
// values as at their mirror images), chunk c of mask row ur at wu[(ur * C4 + c) * ld].
template <int R, int MASK = kCompiler>
__device__ __forceinline__ void wle_weights_unique(float4 *wu, int ld, float WLE_SigmaX, float WLE_SigmaY,
                                                   int MoleculeType) {
    typedef MaskShape<R> M;
    const float ROICenter = R / 2.0f;
    const float WLE_SigmaX1 = 1.0f / (2.0f * WLE_SigmaX * WLE_SigmaX);
    const float WLE_SigmaY1 = 1.0f / (2.0f * WLE_SigmaY * WLE_SigmaY);
    for (int ur = 0; ur < M::U; ur++) {
        const float rowpos = (R / 2 + ur) + 0.5f;
        for (int c = 0; c < M::C4; c++) {
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int uc = c * 4 + j;
                const float colpos = (R / 2 + uc) + 0.5f;
                if (MoleculeType == 0 || uc >= M::U)
                    v[j] = 1.0f;
                else
                    v[j] = __expf(-sum_of_products<MASK>((colpos - ROICenter) * (colpos - ROICenter), WLE_SigmaX1,
                                                         (rowpos - ROICenter) * (rowpos - ROICenter), WLE_SigmaY1));
            }
            wu[(ur * M::C4 + c) * ld] = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
}

// Model exponential of single_expo from the pixel's offsets dx = col + 0.5 - x
// and dy = row + 0.5 - y (the same roundings).
template <int KIND, int DIST>
__device__ __forceinline__ float single_expo_d(float dx, float dy, const float *v) {
    if (KIND == kGS2D) return __expf(-(sum_of_products<DIST>(dx, dx, dy, dy)) * v[3] * QCS_SSCALE);
    return __expf(-(sum_of_products<DIST>(dx * dx * v[3], QCS_SSCALE, dy * dy * v[4], QCS_SSCALE)));
}

// Loss and gradient of one single-emitter ROI (GS2D / AS3D) evaluated by its
// own thread, with the pixels' (value, log) pairs at img[k * ld] and the
// mask's unique values (MaskShape) at wu[(ur * C4 + c) * ld].  Same terms,
// same order, same roundings as loss() / numerical_gradient_shared(), with
// fewer instructions: one 16-byte mask load per row, the column offsets of
// the position computed once per evaluation, the row centre kept as a float.
template <int R, int KIND, int DIST, bool FULL = false>
struct StagedEval {
    typedef KindTraits<KIND> T;
    typedef MaskShape<R> M;
    enum { P = T::P, UNROLL = R <= kUnrollMaxR };
    const float2 *img;
    // the mask: unique values as float4 chunks at ((const float4 *)mask)[(ur * C4 + c) * ld] (16-byte
    // aligned), or (FULL) the R x R values, pixel k at mask[k * ld]
    const float *mask;
    int ld;

    // the mask values of `row`, indexed by mirror_index(col) (FULL: by col)
    __device__ __forceinline__ void mask_row(int row, float (&w)[FULL ? R : M::C4 * 4]) const {
        if constexpr (FULL) {
#pragma unroll
            for (int c = 0; c < R; c++) w[c] = mask[(row * R + c) * ld];
        } else {
            const int ur = mirror_index(row, R);
            const float4 *wu = reinterpret_cast<const float4 *>(mask);
#pragma unroll
            for (int c = 0; c < M::C4; c++) {
                const float4 q = wu[(ur * M::C4 + c) * ld];
                w[4 * c] = q.x;
                w[4 * c + 1] = q.y;
                w[4 * c + 2] = q.z;
                w[4 * c + 3] = q.w;
            }
        }
    }
    __device__ __forceinline__ static constexpr int wcol(int col) { return FULL ? col : mirror_index(col, R); }
    __device__ __forceinline__ float mask_at(int row, int col) const {
        if constexpr (FULL) return mask[(row * R + col) * ld];
        const int ur = mirror_index(row, R), uc = mirror_index(col, R);
        return mask[((ur * M::C4 + uc / 4) * ld) * 4 + uc % 4];
    }

    __device__ __forceinline__ float loss(float *Ininf) const {
#pragma unroll
        for (int k = 0; k < P; k++) {
            if (T::CLAMP001) {
                if (Ininf[k] < 0.01f) Ininf[k] = 0.01f;
            } else {
                if (Ininf[k] < 0.0f) Ininf[k] = 0.0f;
            }
        }
        float TotalLoss = 0;
        if constexpr (UNROLL) {
            float dxs[R];
#pragma unroll
            for (int col = 0; col < R; col++) dxs[col] = (col + 0.5f) - Ininf[1];
            float rowpos = 0.5f;
            const float2 *pr = img;
#pragma unroll 1
            for (int row = 0; row < R; row++) {
                float w[FULL ? R : M::C4 * 4];
                mask_row(row, w);
                const float dy = rowpos - Ininf[2];
#pragma unroll
                for (int col = 0; col < R; col++) {
                    const float2 pl = pr[col * ld];
                    const float Lt = single_term<KIND>(single_expo_d<KIND, DIST>(dxs[col], dy, Ininf), Ininf, pl.x,
                                                       pl.y);
                    TotalLoss = __fmaf_rn(w[wcol(col)], Lt, TotalLoss);
                }
                rowpos += 1.0f;
                pr += R * ld;
            }
        } else {
#pragma unroll 1
            for (int row = 0; row < R; row++) {
#pragma unroll 1
                for (int col = 0; col < R; col++) {
                    const float2 pl = img[(row * R + col) * ld];
                    const float Lt = single_term<KIND>(
                        single_expo<KIND, DIST>(col + 0.5f, row + 0.5f, Ininf), Ininf, pl.x, pl.y);
                    TotalLoss = __fmaf_rn(mask_at(row, col), Lt, TotalLoss);
                }
            }
        }
        return TotalLoss;
    }

    // numerical_gradient_shared with this layout (and its point-by-point
    // fallback through loss()).
    __device__ __forceinline__ void gradient(const float *Ininf, float *grad) const {
        enum { NE = 2 * P };
        float v[NE][P];
        {
            float t[P];
#pragma unroll
            for (int k = 0; k < P; k++) t[k] = Ininf[k];
#pragma unroll
            for (int k = 0; k < P; k++) {
                t[k] = t[k] - 0.002f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                    v[2 * k][c] = t[c];
                }
                t[k] = t[k] + 0.004f;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (T::CLAMP001) { if (t[c] < 0.01f) t[c] = 0.01f; } else { if (t[c] < 0.0f) t[c] = 0.0f; }
                    v[2 * k + 1][c] = t[c];
                }
                t[k] = t[k] - 0.002f;
            }
        }
        bool share = true;
#pragma unroll
        for (int c = 1; c < P - 1; c++) {
            const unsigned b = __float_as_uint(v[0][c]);
            share = share && (__float_as_uint(v[1][c]) == b) && (__float_as_uint(v[NE - 2][c]) == b) &&
                    (__float_as_uint(v[NE - 1][c]) == b);
        }
        if (!__all_sync(__activemask(), share)) {
            float tI[P];
#pragma unroll
            for (int c = 0; c < P; c++) tI[c] = Ininf[c];
            for (int k = 0; k < P; k++) {
                tI[k] = tI[k] - 0.002f;
                const float tn = loss(tI);
                tI[k] = tI[k] + 0.004f;
                const float tp = loss(tI);
                grad[k] = (tp - tn) * 250.0f;
                tI[k] = tI[k] - 0.002f;
            }
            return;
        }
        float tot[NE];
#pragma unroll
        for (int j = 0; j < NE; j++) tot[j] = 0;
        float rowpos = 0.5f;
#pragma unroll 1
        for (int row = 0; row < R; row++) {
            float w[FULL ? R : M::C4 * 4];
            if constexpr (UNROLL) mask_row(row, w);
#pragma unroll(UNROLL ? R : 1)
            for (int col = 0; col < R; col++) {
                const float2 pl = img[(row * R + col) * ld];
                const float wk = UNROLL ? w[wcol(col)] : mask_at(row, col);
                const float colpos = col + 0.5f;
                const float e_base = single_expo<KIND, DIST>(colpos, rowpos, v[0]);
#pragma unroll
                for (int j = 0; j < NE; j++) {
                    const bool base = (j < 2) || (j >= NE - 2);
                    const float e = base ? e_base : single_expo<KIND, DIST>(colpos, rowpos, v[j]);
                    tot[j] = __fmaf_rn(wk, single_term<KIND>(e, v[j], pl.x, pl.y), tot[j]);
                }
            }
            rowpos += 1.0f;
        }
#pragma unroll
        for (int k = 0; k < P; k++) grad[k] = (tot[2 * k + 1] - tot[2 * k]) * 250.0f;
    }
};

// The learned-start single fit's loss and analytic gradient over the staged
// layout of fit_single_kernel (pixels as (value, log) pairs, the mask's unique
// values): StagedEval's loss, the gradient of AnalyticEvalGS2D /
// AnalyticEvalAS3D term for term (the mask values are the same, so the
// results are those of the full-mask evaluators).
template <int R, int KIND, int DIST, bool FULL = false>
struct StagedAnalyticEval : StagedEval<R, KIND, DIST, FULL> {
    typedef StagedEval<R, KIND, DIST, FULL> B;
    __device__ __forceinline__ void gradient(const float *v, float *g) const {
        enum { NW = FULL ? R : B::M::C4 * 4 };
        if constexpr (KIND == kGS2D) {
            float c[5];
#pragma unroll
            for (int k = 0; k < 5; k++) c[k] = v[k] < 0.0f ? 0.0f : v[k];
            const float A128 = c[0] * QCS_ASCALE, B64 = c[4] * QCS_BSCALE, S01 = c[3] * QCS_SSCALE;
            float gA = 0, gX = 0, gY = 0, gS = 0, gB = 0;
#pragma unroll 1
            for (int row = 0; row < R; row++) {
                float wr[NW];
                this->mask_row(row, wr);
                const float dy = (row + 0.5f) - c[2];
#pragma unroll(R <= kUnrollMaxR ? R : 1)
                for (int col = 0; col < R; col++) {
                    const float2 pl = this->img[(row * R + col) * this->ld];
                    const float w = wr[B::wcol(col)];
                    const float dx = (col + 0.5f) - c[1];
                    const float r2 = __fmaf_rn(dx, dx, dy * dy);
                    const float e = __expf(-r2 * S01);
                    const float mu = __fmaf_rn(A128, e, B64);
                    const float q = w * (1.0f - __fdividef(pl.x, mu));
                    const float qe = q * e;
                    gA += qe;
                    gX = __fmaf_rn(qe, dx, gX);
                    gY = __fmaf_rn(qe, dy, gY);
                    gS = __fmaf_rn(qe, r2, gS);
                    gB += q;
                }
            }
            g[0] = QCS_ASCALE * gA;
            g[1] = A128 * 2.0f * S01 * gX;
            g[2] = A128 * 2.0f * S01 * gY;
            g[3] = -A128 * QCS_SSCALE * gS;
            g[4] = QCS_BSCALE * gB;
        } else {
            float c[6];
#pragma unroll
            for (int k = 0; k < 6; k++) c[k] = v[k] < 0.01f ? 0.01f : v[k];
            const float A128 = c[0] * QCS_ASCALE, B64 = c[5] * QCS_BSCALE;
            const float Sx = c[3] * QCS_SSCALE, Sy = c[4] * QCS_SSCALE;
            float gA = 0, gX = 0, gY = 0, gSx = 0, gSy = 0, gB = 0;
#pragma unroll 1
            for (int row = 0; row < R; row++) {
                float wr[NW];
                this->mask_row(row, wr);
                const float dy = (row + 0.5f) - c[2];
                const float qy = dy * dy;
#pragma unroll(R <= kUnrollMaxR ? R : 1)
                for (int col = 0; col < R; col++) {
                    const float2 pl = this->img[(row * R + col) * this->ld];
                    const float w = wr[B::wcol(col)];
                    const float dx = (col + 0.5f) - c[1];
                    const float qx = dx * dx;
                    const float e = __expf(-__fmaf_rn(qx, Sx, qy * Sy));
                    const float mu = __fmaf_rn(A128, e, B64);
                    const float q = w * (1.0f - __fdividef(pl.x, mu));
                    const float qe = q * e;
                    gA += qe;
                    gX = __fmaf_rn(qe, dx, gX);
                    gY = __fmaf_rn(qe, dy, gY);
                    gSx = __fmaf_rn(qe, qx, gSx);
                    gSy = __fmaf_rn(qe, qy, gSy);
                    gB += q;
                }
            }
            g[0] = QCS_ASCALE * gA;
            g[1] = A128 * 2.0f * Sx * gX;
            g[2] = A128 * 2.0f * Sy * gY;
            g[3] = -A128 * QCS_SSCALE * gSx;
            g[4] = -A128 * QCS_SSCALE * gSy;
            g[5] = QCS_BSCALE * gB;
        }
    }
};

// Fixed schedule: IT quasi-Newton iterations, each with an NB-step bisection
// of the step length in [1e-5, 1] (the reference: 11); no convergence test.
// D: P x P scratch at D[(r * P + c) * ld]; ev evaluates the loss and the
// gradient.
template <int P, int IT, class Eval, int NB = kBisections>
__device__ __forceinline__ void bfgs_fit(const Eval &ev, float *Ininf, float *D, int ld) {
    float grad[P], d0[P], td0[P], sk[P], yk[P], tgrad[P];
    float ddat[2], dpos[2];  // two-element arrays indexed by constants only
#pragma unroll
    for (int r = 0; r < P; r++) {
#pragma unroll
        for (int c = 0; c < P; c++) D[(r * P + c) * ld] = (r == c) ? 1.0f : 0.0f;
    }
    ev.gradient(Ininf, grad);
#pragma unroll
    for (int rcnt = 0; rcnt < P; rcnt++) d0[rcnt] = -grad[rcnt];

    for (int itcnt = 0; itcnt < IT; itcnt++) {
        float td0_total = 0;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) {
            td0[rcnt] = fabsf(d0[rcnt]);
            td0_total += td0[rcnt];
        }
        td0_total = ((float)P) / td0_total;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) d0[rcnt] = d0[rcnt] * td0_total;

        dpos[0] = 0.00001f;
        dpos[1] = 1.0f;
        {
            float xlo[P], xhi[P];
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) xlo[cnt] = d0[cnt] * 0.0001f + Ininf[cnt];
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) xhi[cnt] = d0[cnt] * 1.0f + Ininf[cnt];
            ddat[0] = ev.loss(xlo);
            ddat[1] = ev.loss(xhi);
        }

        // Bisection: the half that moves is chosen per ROI; the moved point
        // is built with a select so that every thread of a warp runs the same
        // single loss evaluation (no divergent branches around the loss).
        for (int cnt = 0; cnt < NB; cnt++) {
            const int xdsel = (ddat[0] < ddat[1]);
            const float mid = (dpos[0] + dpos[1]) * 0.5f;
            dpos[0] = xdsel ? dpos[0] : mid;
            dpos[1] = xdsel ? mid : dpos[1];
            if (cnt < NB - 1) {
                const float dsel = xdsel ? dpos[1] : dpos[0];
                float xn[P];
#pragma unroll
                for (int k = 0; k < P; k++) xn[k] = d0[k] * dsel + Ininf[k];
                const float f = ev.loss(xn);
                ddat[0] = xdsel ? ddat[0] : f;
                ddat[1] = xdsel ? f : ddat[1];
            }
        }
        const float scale = (dpos[0] + dpos[1]) * 0.5f;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) {
            sk[rcnt] = d0[rcnt] * scale;
            Ininf[rcnt] = Ininf[rcnt] + sk[rcnt];
        }
#pragma unroll
        for (int cnt = 0; cnt < P; cnt++)
            if (Ininf[cnt] < 0.01f) Ininf[cnt] = 0.01f;

        if (itcnt < IT - 1) {
#pragma unroll
            for (int rcnt = 0; rcnt < P; rcnt++) tgrad[rcnt] = grad[rcnt];
            ev.gradient(Ininf, grad);
#pragma unroll
            for (int rcnt = 0; rcnt < P; rcnt++) yk[rcnt] = grad[rcnt] - tgrad[rcnt];
            bfgs_update<P>(D, ld, sk, yk);
#pragma unroll
            for (int row = 0; row < P; row++) {
                d0[row] = 0;
#pragma unroll
                for (int cnt = 0; cnt < P; cnt++) d0[row] -= D[(row * P + cnt) * ld] * grad[cnt];
            }
        }
    }
}

// bfgs_update with few live registers, for one lane that updates an inverse
// Hessian shared by a lane group: D (row-major P x P) and the scratch T
// (P x P) in shared memory.  The same values as bfgs_update, operation for
// operation: its P x P temporaries are recomputed from sk and the scaled
// vectors with the roundings nvcc gives their expressions (one fused
// multiply-add or separate product each), the left product kept in T.
// SKSK_FUSED: the final D + sk sk'/(y's) fused into one multiply-add (nvcc
// may contract the separately computed product into the sum).
template <int P, bool SKSK_FUSED>
__device__ __forceinline__ void bfgs_update_light(float *D, float *T, const float *sk, const float *yk) {
    float divdat = 0;
#pragma unroll
    for (int cnt = 0; cnt < P; cnt++) divdat = __fmaf_rn(sk[cnt], yk[cnt], divdat);
    divdat = 1.0f / divdat;
    float tdat10[P], tdat20[P];
#pragma unroll
    for (int cnt = 0; cnt < P; cnt++) {
        tdat10[cnt] = __fmul_rn(yk[cnt], divdat);
        tdat20[cnt] = __fmul_rn(sk[cnt], divdat);
    }
    // skyk(r, c) = [r == c] - sk[r] tdat10[c], one rounding
    auto skyk = [&](int r, int c) { return __fmaf_rn(-sk[r], tdat10[c], r == c ? 1.0f : 0.0f); };
#pragma unroll 1
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int col = 0; col < P; col++) {
            float acc = 0;
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) acc = __fmaf_rn(skyk(row, cnt), D[cnt * P + col], acc);
            T[row * P + col] = acc;
        }
    }
#pragma unroll 1
    for (int row = 0; row < P; row++) {
#pragma unroll
        for (int col = 0; col < P; col++) {
            float acc = 0;
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) acc = __fmaf_rn(T[row * P + cnt], skyk(col, cnt), acc);
            D[row * P + col] = SKSK_FUSED ? __fmaf_rn(sk[row], tdat20[col], acc)
                                          : __fadd_rn(acc, __fmul_rn(sk[row], tdat20[col]));
        }
    }
}

// bfgs_fit for a lane group that shares one inverse Hessian per ROI: every
// lane runs the line search and the evaluations (which need all lanes), the
// group's first lane alone updates D (bfgs_update_light) and the new search
// direction, which the others then read from dbuf.  D, T: P x P, dbuf: P
// floats of shared memory per ROI.  The same values as bfgs_fit.
template <int P, int IT, class Eval, bool SKSK_FUSED, int NB = kBisections>
__device__ __forceinline__ void bfgs_fit_shared(const Eval &ev, float *Ininf, float *D, float *T, float *dbuf,
                                                int lane, unsigned mask) {
    float grad[P], d0[P], td0[P], sk[P], yk[P], tgrad[P];
    float ddat[2], dpos[2];
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < P; r++) {
#pragma unroll
            for (int c = 0; c < P; c++) D[r * P + c] = (r == c) ? 1.0f : 0.0f;
        }
    }
    ev.gradient(Ininf, grad);
#pragma unroll
    for (int rcnt = 0; rcnt < P; rcnt++) d0[rcnt] = -grad[rcnt];

    for (int itcnt = 0; itcnt < IT; itcnt++) {
        float td0_total = 0;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) {
            td0[rcnt] = fabsf(d0[rcnt]);
            td0_total += td0[rcnt];
        }
        td0_total = ((float)P) / td0_total;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) d0[rcnt] = d0[rcnt] * td0_total;

        dpos[0] = 0.00001f;
        dpos[1] = 1.0f;
        {
            float xlo[P], xhi[P];
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) xlo[cnt] = d0[cnt] * 0.0001f + Ininf[cnt];
#pragma unroll
            for (int cnt = 0; cnt < P; cnt++) xhi[cnt] = d0[cnt] * 1.0f + Ininf[cnt];
            ddat[0] = ev.loss(xlo);
            ddat[1] = ev.loss(xhi);
        }
        for (int cnt = 0; cnt < NB; cnt++) {
            const int xdsel = (ddat[0] < ddat[1]);
            const float mid = (dpos[0] + dpos[1]) * 0.5f;
            dpos[0] = xdsel ? dpos[0] : mid;
            dpos[1] = xdsel ? mid : dpos[1];
            if (cnt < NB - 1) {
                const float dsel = xdsel ? dpos[1] : dpos[0];
                float xn[P];
#pragma unroll
                for (int k = 0; k < P; k++) xn[k] = d0[k] * dsel + Ininf[k];
                const float f = ev.loss(xn);
                ddat[0] = xdsel ? ddat[0] : f;
                ddat[1] = xdsel ? f : ddat[1];
            }
        }
        const float scale = (dpos[0] + dpos[1]) * 0.5f;
#pragma unroll
        for (int rcnt = 0; rcnt < P; rcnt++) {
            sk[rcnt] = d0[rcnt] * scale;
            Ininf[rcnt] = Ininf[rcnt] + sk[rcnt];
        }
#pragma unroll
        for (int cnt = 0; cnt < P; cnt++)
            if (Ininf[cnt] < 0.01f) Ininf[cnt] = 0.01f;

        if (itcnt < IT - 1) {
#pragma unroll
            for (int rcnt = 0; rcnt < P; rcnt++) tgrad[rcnt] = grad[rcnt];
            ev.gradient(Ininf, grad);
            if (lane == 0) {
#pragma unroll
                for (int rcnt = 0; rcnt < P; rcnt++) yk[rcnt] = grad[rcnt] - tgrad[rcnt];
                bfgs_update_light<P, SKSK_FUSED>(D, T, sk, yk);
#pragma unroll
                for (int row = 0; row < P; row++) {
                    float acc = 0;
#pragma unroll
                    for (int cnt = 0; cnt < P; cnt++) acc = __fmaf_rn(-D[row * P + cnt], grad[cnt], acc);
                    dbuf[row] = acc;
                }
            }
            __syncwarp(mask);
#pragma unroll
            for (int row = 0; row < P; row++) d0[row] = dbuf[row];
            __syncwarp(mask);
        }
    }
}

template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST, int SUM2 = ArithSpec<KIND, R>::SUM2,
          int ITERS = KindTraits<KIND>::IT>
__device__ __forceinline__ void mle_fit(const RoiRef &roi, float *Ininf, float *D, int ld) {
    bfgs_fit<KindTraits<KIND>::P, ITERS>(ThreadEval<R, KIND, DIST, SUM2>{roi}, Ininf, D, ld);
}

// Weighted-MLE mask (bfgsMLE_core.h:206-238).
template <int R, int MASK = kCompiler>
__device__ __forceinline__ void wle_weights(float *w, int ld, float WLE_SigmaX, float WLE_SigmaY, int MoleculeType) {
    const float ROICenter = R / 2.0f;
    const float WLE_SigmaX1 = 1.0f / (2.0f * WLE_SigmaX * WLE_SigmaX);
    const float WLE_SigmaY1 = 1.0f / (2.0f * WLE_SigmaY * WLE_SigmaY);
    for (int row = 0; row < R; row++) {
        for (int col = 0; col < R; col++) {
            const float rowpos = row + 0.5f;
            const float colpos = col + 0.5f;
            if (MoleculeType == 0)
                w[(row * R + col) * ld] = 1.0f;
            else
                w[(row * R + col) * ld] =
                    __expf(-sum_of_products<MASK>((colpos - ROICenter) * (colpos - ROICenter), WLE_SigmaX1,
                                                  (rowpos - ROICenter) * (rowpos - ROICenter), WLE_SigmaY1));
        }
    }
}

}  // namespace qcs
