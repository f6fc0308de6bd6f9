// CRLB of x and y for each localization: diagonal Fisher information from
// numerical second derivatives (dh = 0.02) of a Gaussian PSF model on a fixed
// 9x9 (2D) or 15x15 (astigmatic 3D) grid with the emitter at the centre, the
// fitted total photons, background (+ read noise^2) and sigma x/y;
// CRLB = PixelSize / sqrt(FI) in nm, 100 when the row is not fittable.
// Re-expressed from LocPrecCalc_GaussianCRLB.h:65-243 with the same
// expression shapes (bit-identical results); adds the bounds guard that the
// reference kernel lacks (:65-128) and reads the row count from the device.
#include <cuda_runtime.h>

#include "qcs_fit_math.cuh"
#include "qcs_kernels.h"

namespace qcs {
namespace {

enum { kParaTPhn = 0, kParaBkgn = 1, kParaXPos = 2, kParaYPos = 3, kParaSigX = 4, kParaSigY = 5 };

// Contraction of the PSF exponent x^2/(2 sx^2) + y^2/(2 sy^2) per grid size
// (see SumMode in qcs_fit_math.cuh).
// PEAK: peak * exp(.) + background; D2: f(+h) - 2 f(0) + f(-h);
// FI: FI + (d2 - model * d2log).  0 = fused multiply-add, 1 = separately
// rounded multiply and add, kCompiler = left to the compiler.
template <int G>
struct CrlbSpec {
    enum { MODE = kCompiler, PEAK = kCompiler, D2 = kCompiler, FI = kCompiler };
};

template <int S>
__device__ __forceinline__ float mul_add(float a, float b, float c) {
    if (S == 0) return __fmaf_rn(a, b, c);
    if (S == 1) return __fadd_rn(__fmul_rn(a, b), c);
    return a * b + c;
}

template <int G, int MODE = CrlbSpec<G>::MODE, int PEAK = CrlbSpec<G>::PEAK>
__device__ __forceinline__ void psf_generate(float *pPSFDat, const float *ParaArry) {
    enum { Half = G / 2 };
    const float TotalPhoton_e = ParaArry[kParaTPhn];
    const float Background_e = ParaArry[kParaBkgn];
    const float x0 = ParaArry[kParaXPos];
    const float y0 = ParaArry[kParaYPos];
    const float PSFSigmaX = ParaArry[kParaSigX];
    const float PSFSigmaY = ParaArry[kParaSigY];
    const float pi = 3.141592654f;
    const float PeakPn = 1 / (2 * pi * PSFSigmaX * PSFSigmaY) * TotalPhoton_e;
    const float PSFSigma_ix = 1 / (2 * PSFSigmaX * PSFSigmaX);
    const float PSFSigma_iy = 1 / (2 * PSFSigmaY * PSFSigmaY);
    float CurX, CurY;
    for (int ycnt = 0; ycnt < G; ycnt++) {
        CurY = ycnt - Half;
        for (int xcnt = 0; xcnt < G; xcnt++) {
            CurX = xcnt - Half;
            pPSFDat[ycnt * G + xcnt] =
                mul_add<PEAK>(PeakPn,
                              __expf(-sum_of_products<MODE>((CurX - x0) * (CurX - x0), PSFSigma_ix,
                                                            (CurY - y0) * (CurY - y0), PSFSigma_iy)),
                              Background_e);
        }
    }
}

template <int N>
__device__ __forceinline__ void log_calc(const float *d, float *l) {
#pragma unroll
    for (int cnt = 0; cnt < N; cnt++) l[cnt] = logf(d[cnt]);
}

template <int N, int D2>
__device__ __forceinline__ void deriv2(float *Deriv2, const float *dat_0, const float *dat_p, const float *dat_n,
                                       float dh) {
#pragma unroll
    for (int cnt = 0; cnt < N; cnt++) {
        if (D2 == kCompiler)
            Deriv2[cnt] = (dat_p[cnt] - 2 * dat_0[cnt] + dat_n[cnt]) / dh / dh;
        else
            Deriv2[cnt] = __fadd_rn(mul_add<D2>(-2.0f, dat_0[cnt], dat_p[cnt]), dat_n[cnt]) / dh / dh;
    }
}

template <int G, int N, int MODE, int PEAK, int D2>
__device__ __forceinline__ void derivative2(float *d2, float *d2log, float *ParaArry, int ParaID) {
    float t0[N], tl0[N], tp[N], tlp[N], tn[N], tln[N];
    const float dh = 0.02f;
    psf_generate<G, MODE, PEAK>(t0, ParaArry);
    log_calc<N>(t0, tl0);
    ParaArry[ParaID] += dh;
    psf_generate<G, MODE, PEAK>(tp, ParaArry);
    log_calc<N>(tp, tlp);
    ParaArry[ParaID] -= 2 * dh;
    psf_generate<G, MODE, PEAK>(tn, ParaArry);
    log_calc<N>(tn, tln);
    ParaArry[ParaID] += dh;
    deriv2<N, D2>(d2, t0, tp, tn, dh);
    deriv2<N, D2>(d2log, tl0, tlp, tln, dh);
}

template <int N, int FI>
__device__ __forceinline__ float crlb_std(const float *model, const float *d2, const float *d2log) {
    float FishirInf = 0;
    for (int cnt = 0; cnt < N; cnt++) {
        if (FI == kCompiler)
            FishirInf += (d2[cnt] - model[cnt] * d2log[cnt]);
        else
            FishirInf = __fadd_rn(FishirInf, mul_add<FI>(-model[cnt], d2log[cnt], d2[cnt]));
    }
    if (FishirInf == 0.0f) FishirInf = 1;
    return sqrtf(1 / FishirInf);
}

template <int G, int MODE = CrlbSpec<G>::MODE, int PEAK = CrlbSpec<G>::PEAK, int D2 = CrlbSpec<G>::D2,
          int FI = CrlbSpec<G>::FI>
__global__ void crlb_kernel(float *__restrict__ loc, const int *__restrict__ n_dev, int n, float ReadNoise_e, float QE,
                            float PixelSize) {
    enum { N = G * G };
    const int rows = n_dev ? *n_dev : n;
    const int gid = threadIdx.x + blockDim.x * blockIdx.x;
    if (gid >= rows) return;
    float *r = loc + (size_t)gid * 12;
    const float TotalPhoton_e = r[QCS_POS_TPHO] * QE;
    float Background_e = r[QCS_POS_BAKG] * QE;
    const float PSFSigmaX = r[QCS_POS_SIGX];
    const float PSFSigmaY = r[QCS_POS_SIGY];
    float ParaStdX = 100.0f;
    float ParaStdY = 100.0f;
    if ((TotalPhoton_e > 1) && (Background_e > 1) && (PSFSigmaX > 0.1) && (PSFSigmaY > 0.1) && (PSFSigmaX < 10) &&
        (PSFSigmaY < 10)) {
        float model[N], d2[N], d2log[N];
        float ParaArry[6];
        Background_e = (Background_e * QE + ReadNoise_e * ReadNoise_e) / QE;
        ParaArry[kParaTPhn] = TotalPhoton_e;
        ParaArry[kParaBkgn] = Background_e;
        ParaArry[kParaXPos] = 0;
        ParaArry[kParaYPos] = 0;
        ParaArry[kParaSigX] = PSFSigmaX;
        ParaArry[kParaSigY] = PSFSigmaY;
        psf_generate<G, MODE, PEAK>(model, ParaArry);
        derivative2<G, N, MODE, PEAK, D2>(d2, d2log, ParaArry, kParaXPos);
        ParaStdX = crlb_std<N, FI>(model, d2, d2log);
        derivative2<G, N, MODE, PEAK, D2>(d2, d2log, ParaArry, kParaYPos);
        ParaStdY = crlb_std<N, FI>(model, d2, d2log);
        ParaStdX = ParaStdX * PixelSize;
        ParaStdY = ParaStdY * PixelSize;
    }
    r[QCS_POS_CRBX] = ParaStdX;
    r[QCS_POS_CRBY] = ParaStdY;
}

}  // namespace

cudaError_t launch_crlb(float *loc, const int *n_dev, int n, int max_rows, int loc_type, float ReadNoise_e, float QE,
                        float PixelSize, cudaStream_t s) {
    const int tpb = 64;
    const int grid = (max_rows + tpb - 1) / tpb;
    if (grid == 0) return cudaSuccess;
    if (loc_type != QCS_LOCTYPE_AS3D)
        crlb_kernel<9><<<grid, tpb, 0, s>>>(loc, n_dev, n, ReadNoise_e, QE, PixelSize);
    else
        crlb_kernel<15><<<grid, tpb, 0, s>>>(loc, n_dev, n, ReadNoise_e, QE, PixelSize);
    return cudaGetLastError();
}

}  // namespace qcs
