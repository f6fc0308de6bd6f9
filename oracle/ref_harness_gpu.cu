// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" entry points over the reference QC-STORM library compiled with
// nvcc for sm_100a (oracle/build_ref.py --gpu -> oracle/_ref/libqcs_ref_gpu.so).
// Used on a GPU host as the bit-level checker of the product kernels: the
// reference's own CUDA code, run on the same inputs on the same device.
//   qcsrefg_localize    LDLocData_TypeDef::BFGS_MLELocalization (bfgs_top.cu:26-204)
//   qcsrefg_fit_kernel  bfgsMLELoc_Gauss2D<R,5> / bfgsMLELoc_AS3D<R,6> launched
//                       directly with the true ROI size (the reference dispatcher
//                       launches AS3D<8> for ROISize 9, bfgsMLE_Single_Emitter_Fit.cu:96)
//   qcsrefg_crlb        LocPrecCalc_GaussianCRLB (LocPrecCalc_GaussianCRLB.cu:23-40)
//   qcsrefg_wle         WLEParameterEstimation_TypeDef::WLEParameterEstimate
//   qcsrefg_extract     LDROIExtractData_TypeDef::ExtractMolecules
//   qcsrefg_zero_remove ZeroLocalizationsRemovel_TypeDef::RemoveZeroLocalizations
//   qcsrefg_consec     ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg over a sequence of groups
//   qcsrefg_stat       FluoStatisticData_TypeDef::GetStatisticalInf over a sequence of groups
// Every entry point returns 0, or the CUDA error code of the first failure.
#include <cstdio>
#include <cstring>
#include <vector>

#include "bfgs_top.h"
#include "LDROIExtraction.h"
#include "WLEParaEstimation.h"
#include "bfgsMLE_GS2D_core.h"
#include "bfgsMLE_AS3D_core.h"
#include "bfgsMLE_GS2D_2Emitter_core.h"
#include "bfgsMLE_GS2D_3Emitter_core.h"
#include "bfgsMLE_AS3D_2Emitter_core.h"
#include "LocPrecCalc_GaussianCRLB.h"
#include "ZeroLocalizationsRemove.h"
#include "ConsecutiveFit.h"
#include "statisticsInfo.h"
#include "ImageRender_2d.h"
#include "ImageRender_3d.h"

#include "../include/qcstorm_b200.h"

namespace {

void to_ref(const qcs_loc_para *p, LocalizationPara &r) {
    static_assert(sizeof(qcs_loc_para) == sizeof(LocalizationPara), "layout");
    memcpy(&r, p, sizeof(LocalizationPara));
}

// The reference launches its multi-emitter kernels even for empty queues
// (zero blocks), which only sets a non-sticky invalid-configuration error;
// that one is cleared and ignored here.
int check() {
    cudaError_t e = cudaDeviceSynchronize();
    cudaError_t l = cudaGetLastError();
    if (e == cudaSuccess && l != cudaErrorInvalidConfiguration) e = l;
    return (int)e;
}

}  // namespace

extern "C" {

// The reference sizes every buffer for MaxPointNum rows and does not bound
// appended second emitters or detected ROIs; inputs that could overflow those
// buffers (and so make the reference read or write past them) are refused here.
int qcsrefg_localize(const qcs_loc_para *p, const unsigned short *rois, const float *wle, int n,
                     float *out, int out_cap, int *n_valid, float *ratios) {
    LocalizationPara r;
    to_ref(p, r);
    if (n < 0 || n > MaxPointNum / 2) return -1;
    LDLocData_TypeDef loc;
    loc.Init(r);
    const int whole = r.ROISize * (r.ROISize + 1);
    int m = n < MaxPointNum ? n : MaxPointNum;
    unsigned short *h_roi = nullptr;
    float *h_wle = nullptr;
    cudaMallocHost((void **)&h_roi, sizeof(unsigned short) * whole * (size_t)(m > 0 ? m : 1));
    cudaMallocHost((void **)&h_wle, sizeof(float) * WLE_ParaNumber * (size_t)(m > 0 ? m : 1));
    memcpy(h_roi, rois, sizeof(unsigned short) * whole * (size_t)m);
    memcpy(h_wle, wle, sizeof(float) * WLE_ParaNumber * (size_t)m);
    cudaStream_t s;
    cudaStreamCreate(&s);
    loc.BFGS_MLELocalization(h_roi, h_wle, r, n, s);
    cudaStreamSynchronize(s);
    int st = check();
    int nv = loc.oValidFluoNum;
    if (nv > out_cap) nv = out_cap;
    memcpy(out, loc.h_LocArry, sizeof(float) * OutParaNumGS2D * (size_t)nv);
    *n_valid = loc.oValidFluoNum;
    if (ratios) {
        ratios[0] = loc.FitRatio_1E; ratios[1] = loc.FitRatio_2E; ratios[2] = loc.FitRatio_3E;
        ratios[3] = loc.FitRatio_Final_1E; ratios[4] = loc.FitRatio_Final_2E;
        ratios[5] = loc.FitRatio_Final_3E; ratios[6] = loc.FitRatio_Final_4E;
    }
    cudaStreamDestroy(s);
    cudaFreeHost(h_roi);
    cudaFreeHost(h_wle);
    loc.Deinit(r);
    return st;
}

// kind 0 = GS2D, 1 = AS3D; MultiEmitterFitEn forced to 0 (identity queue).
// out: n rows of 12 floats, zero-initialised before the launch.
int qcsrefg_fit_kernel(int kind, const qcs_loc_para *p, const unsigned short *rois, const float *wle,
                       int n, float *out, float *ms) {
    LocalizationPara r;
    to_ref(p, r);
    CoreFittingPara c;
    c.MultiEmitterFitEn = 0; c.WLEEn = r.WLEEn; c.Offset = r.Offset; c.KAdc = r.KAdc; c.QE = r.QE;
    c.ReadNoise_e = r.ReadNoise_e; c.ZDepthCorrFactor = r.ZDepthCorrFactor;
    c.p4_XGY = r.p4_XGY; c.p3_XGY = r.p3_XGY; c.p2_XGY = r.p2_XGY; c.p1_XGY = r.p1_XGY; c.p0_XGY = r.p0_XGY;
    c.p4_XLY = r.p4_XLY; c.p3_XLY = r.p3_XLY; c.p2_XLY = r.p2_XLY; c.p1_XLY = r.p1_XLY; c.p0_XLY = r.p0_XLY;
    const int whole = r.ROISize * (r.ROISize + 1);
    unsigned short *d_roi; float *d_wle, *d_loc; CoreFittingPara *d_c; FitPosInf_TypeDef *d_f;
    int *d_int;
    cudaMalloc((void **)&d_roi, sizeof(unsigned short) * whole * (size_t)n);
    cudaMalloc((void **)&d_wle, sizeof(float) * WLE_ParaNumber * (size_t)n);
    cudaMalloc((void **)&d_loc, sizeof(float) * OutParaNumGS2D * (size_t)n);
    cudaMalloc((void **)&d_c, sizeof(CoreFittingPara));
    cudaMalloc((void **)&d_f, sizeof(FitPosInf_TypeDef));
    cudaMalloc((void **)&d_int, sizeof(int) * (8 + 3 * (size_t)n));
    cudaMemcpy(d_roi, rois, sizeof(unsigned short) * whole * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_wle, wle, sizeof(float) * WLE_ParaNumber * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemset(d_loc, 0, sizeof(float) * OutParaNumGS2D * (size_t)n);
    cudaMemset(d_int, 0, sizeof(int) * (8 + 3 * (size_t)n));
    cudaMemcpy(d_c, &c, sizeof(c), cudaMemcpyHostToDevice);
    FitPosInf_TypeDef f;
    memset(&f, 0, sizeof(f));
    f.d_SingleFitFluoNum = d_int + 0;
    f.d_MultiFitFluoNum_2E = d_int + 1;
    f.d_MultiFitFluoNum_3E = d_int + 2;
    f.d_RejectedFluoNum = d_int + 3;
    f.d_MultiFit_AddedFluoNum = d_int + 4;
    f.d_SingleFitFluoPos = d_int + 8;
    f.d_MultiFitFluoPos_2E = d_int + 8 + n;
    f.d_MultiFitFluoPos_3E = d_int + 8 + 2 * (size_t)n;
    cudaMemcpy(d_f, &f, sizeof(f), cudaMemcpyHostToDevice);
    const int blocks = (n + ThreadsPerBlock - 1) / ThreadsPerBlock;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = 2;
#define QCSREFG_CASE(KIND, R, KERNEL)                                                    \
    if (kind == KIND && r.ROISize == R) {                                                \
        cudaEventRecord(e0);                                                             \
        KERNEL<<<blocks, ThreadsPerBlock>>>(d_loc, d_roi, d_wle, n, d_f, d_c);           \
        cudaEventRecord(e1);                                                             \
        st = check();                                                                    \
    }
    QCSREFG_CASE(0, 5, (bfgsMLELoc_Gauss2D<5, FitParaNum_2D>))
    QCSREFG_CASE(0, 7, (bfgsMLELoc_Gauss2D<7, FitParaNum_2D>))
    QCSREFG_CASE(0, 9, (bfgsMLELoc_Gauss2D<9, FitParaNum_2D>))
    QCSREFG_CASE(0, 11, (bfgsMLELoc_Gauss2D<11, FitParaNum_2D>))
    QCSREFG_CASE(0, 13, (bfgsMLELoc_Gauss2D<13, FitParaNum_2D>))
    QCSREFG_CASE(1, 5, (bfgsMLELoc_AS3D<5, FitParaNum_AS3D>))
    QCSREFG_CASE(1, 7, (bfgsMLELoc_AS3D<7, FitParaNum_AS3D>))
    QCSREFG_CASE(1, 9, (bfgsMLELoc_AS3D<9, FitParaNum_AS3D>))
    QCSREFG_CASE(1, 11, (bfgsMLELoc_AS3D<11, FitParaNum_AS3D>))
    QCSREFG_CASE(1, 13, (bfgsMLELoc_AS3D<13, FitParaNum_AS3D>))
#undef QCSREFG_CASE
    if (st == 0) {
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        if (ms) *ms = t;
        cudaMemcpy(out, d_loc, sizeof(float) * OutParaNumGS2D * (size_t)n, cudaMemcpyDeviceToHost);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_roi); cudaFree(d_wle); cudaFree(d_loc); cudaFree(d_c); cudaFree(d_f); cudaFree(d_int);
    return st;
}

// One multi-emitter fit kernel over all n records (queue 0..n-1): kind 2 =
// GS2D 2E, 3 = GS2D 3E, 4 = AS3D 2E.  out: out_cap rows; first emitters (or
// zero rows) at the record index, second emitters appended from row n in the
// order of the reference's atomic counter; *n_rows = n + appended.
int qcsrefg_fit_multi_kernel(int kind, const qcs_loc_para *p, const unsigned short *rois, const float *wle, int n,
                             float *out, int out_cap, int *n_rows) {
    LocalizationPara r;
    to_ref(p, r);
    if (n <= 0 || n > MaxPointNum / 2 || out_cap < 2 * n) return -1;
    CoreFittingPara c;
    c.MultiEmitterFitEn = 1; c.WLEEn = r.WLEEn; c.Offset = r.Offset; c.KAdc = r.KAdc; c.QE = r.QE;
    c.ReadNoise_e = r.ReadNoise_e; c.ZDepthCorrFactor = r.ZDepthCorrFactor;
    c.p4_XGY = r.p4_XGY; c.p3_XGY = r.p3_XGY; c.p2_XGY = r.p2_XGY; c.p1_XGY = r.p1_XGY; c.p0_XGY = r.p0_XGY;
    c.p4_XLY = r.p4_XLY; c.p3_XLY = r.p3_XLY; c.p2_XLY = r.p2_XLY; c.p1_XLY = r.p1_XLY; c.p0_XLY = r.p0_XLY;
    const int whole = r.ROISize * (r.ROISize + 1);
    unsigned short *d_roi; float *d_wle, *d_loc; CoreFittingPara *d_c; FitPosInf_TypeDef *d_f; int *d_int;
    cudaMalloc((void **)&d_roi, sizeof(unsigned short) * whole * (size_t)n);
    cudaMalloc((void **)&d_wle, sizeof(float) * WLE_ParaNumber * (size_t)n);
    cudaMalloc((void **)&d_loc, sizeof(float) * OutParaNumGS2D * (size_t)MaxPointNum);
    cudaMalloc((void **)&d_c, sizeof(CoreFittingPara));
    cudaMalloc((void **)&d_f, sizeof(FitPosInf_TypeDef));
    cudaMalloc((void **)&d_int, sizeof(int) * (8 + 3 * (size_t)MaxPointNum));
    cudaMemcpy(d_roi, rois, sizeof(unsigned short) * whole * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_wle, wle, sizeof(float) * WLE_ParaNumber * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemset(d_loc, 0, sizeof(float) * OutParaNumGS2D * (size_t)MaxPointNum);
    cudaMemset(d_int, 0, sizeof(int) * (8 + 3 * (size_t)MaxPointNum));
    cudaMemcpy(d_c, &c, sizeof(c), cudaMemcpyHostToDevice);
    std::vector<int> ident(n);
    for (int i = 0; i < n; ++i) ident[i] = i;
    FitPosInf_TypeDef f;
    memset(&f, 0, sizeof(f));
    f.d_SingleFitFluoNum = d_int + 0;
    f.d_MultiFitFluoNum_2E = d_int + 1;
    f.d_MultiFitFluoNum_3E = d_int + 2;
    f.d_RejectedFluoNum = d_int + 3;
    f.d_MultiFit_AddedFluoNum = d_int + 4;
    f.d_SingleFitFluoPos = d_int + 8;
    f.d_MultiFitFluoPos_2E = d_int + 8 + MaxPointNum;
    f.d_MultiFitFluoPos_3E = d_int + 8 + 2 * (size_t)MaxPointNum;
    cudaMemcpy(kind == 3 ? f.d_MultiFitFluoPos_3E : f.d_MultiFitFluoPos_2E, ident.data(), sizeof(int) * n,
               cudaMemcpyHostToDevice);
    cudaMemcpy(f.d_MultiFit_AddedFluoNum, &n, sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_f, &f, sizeof(f), cudaMemcpyHostToDevice);
    const int blocks = (n + ThreadsPerBlock - 1) / ThreadsPerBlock;
    int st = 2;
#define QCSREFG_MCASE(KIND, R, KERNEL)                                          \
    if (kind == KIND && r.ROISize == R) {                                       \
        KERNEL<<<blocks, ThreadsPerBlock>>>(d_loc, d_roi, d_wle, n, d_f, d_c);  \
        st = check();                                                           \
    }
    QCSREFG_MCASE(2, 5, (bfgsMLELoc_Gauss2D_2E<5, FitParaNum_2D_2E>))
    QCSREFG_MCASE(2, 7, (bfgsMLELoc_Gauss2D_2E<7, FitParaNum_2D_2E>))
    QCSREFG_MCASE(2, 9, (bfgsMLELoc_Gauss2D_2E<9, FitParaNum_2D_2E>))
    QCSREFG_MCASE(2, 11, (bfgsMLELoc_Gauss2D_2E<11, FitParaNum_2D_2E>))
    QCSREFG_MCASE(2, 13, (bfgsMLELoc_Gauss2D_2E<13, FitParaNum_2D_2E>))
    QCSREFG_MCASE(3, 5, (bfgsMLELoc_Gauss2D_3E<5, FitParaNum_2D_3E>))
    QCSREFG_MCASE(3, 7, (bfgsMLELoc_Gauss2D_3E<7, FitParaNum_2D_3E>))
    QCSREFG_MCASE(3, 9, (bfgsMLELoc_Gauss2D_3E<9, FitParaNum_2D_3E>))
    QCSREFG_MCASE(3, 11, (bfgsMLELoc_Gauss2D_3E<11, FitParaNum_2D_3E>))
    QCSREFG_MCASE(3, 13, (bfgsMLELoc_Gauss2D_3E<13, FitParaNum_2D_3E>))
    QCSREFG_MCASE(4, 5, (bfgsMLELoc_AS3D_2E<5, FitParaNum_AS3D_2E>))
    QCSREFG_MCASE(4, 7, (bfgsMLELoc_AS3D_2E<7, FitParaNum_AS3D_2E>))
    QCSREFG_MCASE(4, 9, (bfgsMLELoc_AS3D_2E<9, FitParaNum_AS3D_2E>))
    QCSREFG_MCASE(4, 11, (bfgsMLELoc_AS3D_2E<11, FitParaNum_AS3D_2E>))
    QCSREFG_MCASE(4, 13, (bfgsMLELoc_AS3D_2E<13, FitParaNum_AS3D_2E>))
#undef QCSREFG_MCASE
    if (st == 0) {
        int added = 0;
        cudaMemcpy(&added, f.d_MultiFit_AddedFluoNum, sizeof(int), cudaMemcpyDeviceToHost);
        if (added > out_cap) added = out_cap;
        *n_rows = added;
        cudaMemcpy(out, d_loc, sizeof(float) * OutParaNumGS2D * (size_t)added, cudaMemcpyDeviceToHost);
    }
    cudaFree(d_roi); cudaFree(d_wle); cudaFree(d_loc); cudaFree(d_c); cudaFree(d_f); cudaFree(d_int);
    return st;
}

// Element-level probes of two reference device functions, one thread each:
// the weighted-MLE mask WLEWeightsCalc<R> (bfgsMLE_core.h:206-238) and the
// CRLB model image GaussianPSF_generate2D<G> (LocPrecCalc_GaussianCRLB.h:130-166).
}  // extern "C"

template <int R>
__global__ void probe_weights_kernel(float *out, float sx, float sy, int type) {
    float w[R * R];
    WLEWeightsCalc<R>(w, sx, sy, type);
    for (int k = 0; k < R * R; k++) out[k] = w[k];
}

template <int G>
__global__ void probe_psf_kernel(float *out, const float *para) {
    float p[GaussianCRLB_ParaNum], img[G * G];
    for (int k = 0; k < GaussianCRLB_ParaNum; k++) p[k] = para[k];
    GaussianPSF_generate2D<G>(img, p);
    for (int k = 0; k < G * G; k++) out[k] = img[k];
}

extern "C" {

int qcsrefg_probe_weights(int R, float sx, float sy, int type, float *out) {
    float *d;
    cudaMalloc((void **)&d, sizeof(float) * 17 * 17);
    switch (R) {
    case 5: probe_weights_kernel<5><<<1, 1>>>(d, sx, sy, type); break;
    case 7: probe_weights_kernel<7><<<1, 1>>>(d, sx, sy, type); break;
    case 9: probe_weights_kernel<9><<<1, 1>>>(d, sx, sy, type); break;
    case 11: probe_weights_kernel<11><<<1, 1>>>(d, sx, sy, type); break;
    case 13: probe_weights_kernel<13><<<1, 1>>>(d, sx, sy, type); break;
    default: cudaFree(d); return -1;
    }
    int st = check();
    cudaMemcpy(out, d, sizeof(float) * R * R, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return st;
}

int qcsrefg_probe_psf(int G, const float *para6, float *out) {
    float *d, *dp;
    cudaMalloc((void **)&d, sizeof(float) * 15 * 15);
    cudaMalloc((void **)&dp, sizeof(float) * 6);
    cudaMemcpy(dp, para6, sizeof(float) * 6, cudaMemcpyHostToDevice);
    if (G == 9) probe_psf_kernel<9><<<1, 1>>>(d, dp);
    else probe_psf_kernel<15><<<1, 1>>>(d, dp);
    int st = check();
    cudaMemcpy(out, d, sizeof(float) * G * G, cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaFree(dp);
    return st;
}

// CRLB over n rows in place; rows padded to a multiple of 32 (no bounds guard
// in the reference kernel).
int qcsrefg_crlb(const qcs_loc_para *p, float *loc, int n) {
    LocalizationPara r;
    to_ref(p, r);
    const int padded = (n + ThreadsPerBlock - 1) / ThreadsPerBlock * ThreadsPerBlock;
    float *d_loc;
    cudaMalloc((void **)&d_loc, sizeof(float) * OutParaNumGS2D * (size_t)(padded > 0 ? padded : 1));
    cudaMemset(d_loc, 0, sizeof(float) * OutParaNumGS2D * (size_t)(padded > 0 ? padded : 1));
    cudaMemcpy(d_loc, loc, sizeof(float) * OutParaNumGS2D * (size_t)n, cudaMemcpyHostToDevice);
    if (n > 0) LDLocData_TypeDef::LocPrecCalc_GaussianCRLB(d_loc, r, n, 0);
    int st = check();
    cudaMemcpy(loc, d_loc, sizeof(float) * OutParaNumGS2D * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d_loc);
    return st;
}

int qcsrefg_wle(const qcs_loc_para *p, const unsigned short *rois, int n, float *wle_out) {
    // WLEParameterEstimation_TypeDef sizes its buffers for MaxPointNum records
    if (n < 0 || n > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    WLEParameterEstimation_TypeDef w;
    w.Init(r);
    const int whole = r.ROISize * (r.ROISize + 1);
    unsigned short *d_roi;
    cudaMalloc((void **)&d_roi, sizeof(unsigned short) * whole * (size_t)(n > 0 ? n : 1));
    cudaMemcpy(d_roi, rois, sizeof(unsigned short) * whole * (size_t)n, cudaMemcpyHostToDevice);
    cudaStream_t s;
    cudaStreamCreate(&s);
    if (n > 0) w.WLEParameterEstimate(d_roi, r.LocType, r.MultiEmitterFitEn, r.ROISize, n, s);
    cudaStreamSynchronize(s);
    int st = check();
    cudaMemcpy(wle_out, w.d_WLEPara, sizeof(float) * WLE_ParaNumber * (size_t)n, cudaMemcpyDeviceToHost);
    cudaStreamDestroy(s);
    cudaFree(d_roi);
    w.Deinit();
    return st;
}

int qcsrefg_extract(const qcs_loc_para *p, const unsigned short *frames, int n_frames, int batch,
                    int start_frame, unsigned short *rois_out, float *wle_out, int cap, int *n_roi,
                    int *first_frame, int *end_frame) {
    LocalizationPara r;
    to_ref(p, r);
    if ((size_t)r.ImageWidth * r.ImageHigh * batch > (size_t)512 * 512 * 4) return -1;
    LDROIExtractData_TypeDef ex;
    ex.Init(r);
    ex.ResetROINum();
    const size_t frame_px = (size_t)r.ImageWidth * r.ImageHigh;
    cudaStream_t s;
    cudaStreamCreate(&s);
    for (int f = 0; f < n_frames; f += batch) {
        int nb = (n_frames - f) < batch ? (n_frames - f) : batch;
        memcpy(ex.h_RawImg, frames + f * frame_px, sizeof(unsigned short) * frame_px * nb);
        ex.ExtractMolecules(ex.h_RawImg, ImageSource_CPU_Pinned, r, start_frame + f, nb, s);
        if (ex.GetAccumulatedROINum() > MaxPointNum / 2) break;
    }
    cudaStreamSynchronize(s);
    int st = check();
    int n = ex.GetAccumulatedROINum();
    *n_roi = n;
    if (n > cap) n = cap;
    const int whole = r.ROISize * (r.ROISize + 1);
    memcpy(rois_out, ex.h_ImageROI, sizeof(unsigned short) * whole * (size_t)n);
    memcpy(wle_out, ex.Get_h_WLEPara(), sizeof(float) * WLE_ParaNumber * (size_t)n);
    *first_frame = ex.FirstFrame;
    *end_frame = ex.EndFrame;
    cudaStreamDestroy(s);
    ex.Deinit();
    return st;
}

int qcsrefg_zero_remove(const float *rows, int n, int sort_frame, int first_frame, int end_frame, float *out,
                        int *n_out) {
    if (n < 0 || n > MaxPointNum) return -1;
    ZeroLocalizationsRemovel_TypeDef z;
    z.Init();
    float *pinned = nullptr;
    cudaMallocHost((void **)&pinned, sizeof(float) * 12 * (size_t)(n > 0 ? n : 1));
    memcpy(pinned, rows, sizeof(float) * 12 * (size_t)n);
    cudaStream_t s;
    cudaStreamCreate(&s);
    z.RemoveZeroLocalizations(pinned, n, sort_frame, first_frame, end_frame, s);
    cudaStreamSynchronize(s);
    int st = check();
    *n_out = z.ValidFluoNum;
    memcpy(out, z.h_LocArry, sizeof(float) * 12 * (size_t)z.ValidFluoNum);
    cudaStreamDestroy(s);
    cudaFreeHost(pinned);
    z.Deinit();
    return st;
}

// qcsref_consec on the GPU build.
int qcsrefg_consec(const qcs_loc_para *p, const float *rows, const int *sizes, const int *is_end, int n_groups,
                   float *out, int *out_n, float *ontime) {
    for (int g = 0; g < n_groups; ++g)
        if (sizes[g] < 0 || sizes[g] > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    ConsecutiveFit_TypeDef cf;
    cf.Init();
    float *pinned = nullptr;
    cudaMallocHost((void **)&pinned, sizeof(float) * 12 * (size_t)MaxPointNum);
    cudaStream_t s;
    cudaStreamCreate(&s);
    size_t off = 0, oo = 0;
    int st = 0;
    for (int g = 0; g < n_groups && st == 0; ++g) {
        memcpy(pinned, rows + off * 12, sizeof(float) * 12 * (size_t)sizes[g]);
        cf.ConsecutiveFit_WeightedAvg(pinned, sizes[g], is_end[g], r, s);
        cudaStreamSynchronize(s);
        st = check();
        out_n[g] = cf.OutFluoNum;
        memcpy(out + oo * 12, cf.h_OutLocArry, sizeof(float) * 12 * (size_t)cf.OutFluoNum);
        memcpy(ontime + (size_t)g * MaxOnTimeConsecutiveNum, cf.h_OntimeRatio, sizeof(float) * MaxOnTimeConsecutiveNum);
        oo += (size_t)cf.OutFluoNum;
        off += (size_t)sizes[g];
    }
    cudaStreamDestroy(s);
    cudaFreeHost(pinned);
    cf.Deinit();
    return st;
}

// copies the histograms and means of call g (see qcsref_stat)
static void stat_out(const FluoStatisticData_TypeDef &sd, int g, int *hist, float *means) {
    int *h = hist + (size_t)g * 4 * StatInf_Hist_DatLenMax;
    memcpy(h, sd.h_Hist_TotalPhoton, sizeof(int) * StatInf_Hist_DatLenMax);
    memcpy(h + StatInf_Hist_DatLenMax, sd.h_Hist_LocPrecisionXY, sizeof(int) * StatInf_Hist_DatLenMax);
    memcpy(h + 2 * StatInf_Hist_DatLenMax, sd.h_Hist_PeakSNR, sizeof(int) * StatInf_Hist_DatLenMax);
    memcpy(h + 3 * StatInf_Hist_DatLenMax, sd.h_Hist_PSFWidth, sizeof(int) * StatInf_Hist_DatLenMax);
    float *m = means + (size_t)g * 10;
    m[0] = sd.MeanTotalPhoton;
    m[1] = sd.MeanLocPrecisionXY;
    m[2] = sd.MeanPeakSNR;
    m[3] = sd.MeanBackground;
    m[4] = sd.MeanPSFWidth;
    m[5] = sd.MeanPSFWidth_Ctl;
    m[6] = sd.MeanLocDensity2D;
    m[7] = sd.TimeVaryMean_TotalPhoton;
    m[8] = sd.TimeVaryMean_LocPrecisionXY;
    m[9] = sd.TimeVaryMean_PeakSNR;
}

// qcsref_stat on the GPU build.
int qcsrefg_stat(const qcs_loc_para *p, const float *rows, const int *sizes, int n_groups, int *hist, float *means) {
    for (int g = 0; g < n_groups; ++g)
        if (sizes[g] < 0 || sizes[g] > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    FluoStatisticData_TypeDef sd;
    sd.Init();
    cudaStream_t s;
    cudaStreamCreate(&s);
    sd.ResetAllDat(s);
    float *pinned = nullptr;
    cudaMallocHost((void **)&pinned, sizeof(float) * 12 * (size_t)MaxPointNum);
    size_t off = 0;
    int st = 0;
    for (int g = 0; g < n_groups && st == 0; ++g) {
        memcpy(pinned, rows + off * 12, sizeof(float) * 12 * (size_t)sizes[g]);
        sd.GetStatisticalInf(pinned, r, sizes[g], s);
        cudaStreamSynchronize(s);
        st = check();
        stat_out(sd, g, hist, means);
        off += (size_t)sizes[g];
    }
    cudaFreeHost(pinned);
    cudaStreamDestroy(s);
    sd.Deinit();
    return st;
}

// ImageRenderData_TypeDef::FluoRenderTop's device part (ImageRender_top.cu:29-60):
// the reference's FluoRenderWithPrec_2D / _3D launchers (ImageRender_2d.cu:372,
// ImageRender_3d.cu:333) on a render object holding only the buffers they
// touch.  img, colormap (3D only; may be NULL for 2D), max_val and hist (400
// ints) are read as the starting state and written back.
int qcsrefg_render(const qcs_loc_para *p, const float *rows, int n, int mode, float fixed_prec, float *img, float *colormap,
            int *max_val, int *hist) {
    LocalizationPara r;
    to_ref(p, r);
    ImageRenderData_TypeDef d;
    memset(&d, 0, sizeof(d));
    const size_t px = (size_t)r.SRImageWidth * (size_t)r.SRImageHigh;
    const bool is2d = RendType_Is2D(r.LocType);
    const int padded = (n + 31) / 32 * 32 + 32;
    cudaMalloc((void **)&d.d_LocArry, sizeof(float) * OutParaNumGS2D * (size_t)padded);
    cudaMemset(d.d_LocArry, 0, sizeof(float) * OutParaNumGS2D * (size_t)padded);
    if (n > 0) cudaMemcpy(d.d_LocArry, rows, sizeof(float) * OutParaNumGS2D * (size_t)n, cudaMemcpyHostToDevice);
    cudaMalloc((void **)&d.d_SRIntensityImg, sizeof(float) * px);
    cudaMemcpy(d.d_SRIntensityImg, img, sizeof(float) * px, cudaMemcpyHostToDevice);
    if (!is2d) {
        cudaMalloc((void **)&d.d_SRColorMapImg, sizeof(float) * px);
        cudaMemcpy(d.d_SRColorMapImg, colormap, sizeof(float) * px, cudaMemcpyHostToDevice);
    }
    cudaMalloc((void **)&d.d_MaxImageVal, sizeof(int));
    cudaMemcpy(d.d_MaxImageVal, max_val, sizeof(int), cudaMemcpyHostToDevice);
    cudaMalloc((void **)&d.d_HistMaxDat, sizeof(int) * ImgRend_MaxDatHistLen);
    cudaMemcpy(d.d_HistMaxDat, hist, sizeof(int) * ImgRend_MaxDatHistLen, cudaMemcpyHostToDevice);
    if (n > 0) {
        if (is2d)
            ImgRender_FluoRenderWithPrec_2D(nullptr, &d, r, mode, fixed_prec, n, 0);
        else
            ImgRender_FluoRender_3D(nullptr, &d, r, mode, fixed_prec, n, 0);
    }
    int st = check();
    cudaMemcpy(img, d.d_SRIntensityImg, sizeof(float) * px, cudaMemcpyDeviceToHost);
    if (!is2d) cudaMemcpy(colormap, d.d_SRColorMapImg, sizeof(float) * px, cudaMemcpyDeviceToHost);
    cudaMemcpy(max_val, d.d_MaxImageVal, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(hist, d.d_HistMaxDat, sizeof(int) * ImgRend_MaxDatHistLen, cudaMemcpyDeviceToHost);
    cudaFree(d.d_LocArry);
    cudaFree(d.d_SRIntensityImg);
    if (!is2d) cudaFree(d.d_SRColorMapImg);
    cudaFree(d.d_MaxImageVal);
    cudaFree(d.d_HistMaxDat);
    return st;
}

}  // extern "C"

// cudaWrapper.cu is not compiled (it only prints); this is its quiet stand-in.
void HandleErr(cudaError_t, const char *) {}
