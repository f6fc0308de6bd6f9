// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" entry points over the reference QC-STORM library compiled for
// the host (oracle/build_ref.py).  Everything below calls the reference's own
// classes and kernels; this file only converts parameters and copies results.
//   qcsref_localize    LDLocData_TypeDef::BFGS_MLELocalization (bfgs_top.cu:26-204)
//   qcsref_fit_kernel  one fit kernel launched directly, e.g. bfgsMLELoc_AS3D<9,6>
//                      (the reference dispatcher launches <8> for ROISize 9,
//                      bfgsMLE_Single_Emitter_Fit.cu:96)
//   qcsref_crlb        GaussianCRLB_Calc_top (LocPrecCalc_GaussianCRLB.h:65-128)
//   qcsref_wle         WLEParameterEstimation_TypeDef::WLEParameterEstimate
//   qcsref_zero_remove ZeroLocalizationsRemovel_TypeDef::RemoveZeroLocalizations
//   qcsref_consec      ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg over a sequence of groups
//   qcsref_stat        FluoStatisticData_TypeDef::GetStatisticalInf over a sequence of groups
//   qcsref_ontime      FluoStatisticData_TypeDef::UpdateOntimeRatio over a sequence of calls
//                      (WLEParaEstimation.cpp:20-40)
//   qcsref_extract     LDROIExtractData_TypeDef::ExtractMolecules (LDROIExtraction.cu:30-80)
#include <cstdio>
#include <cstring>
#include <vector>

#include "bfgs_top.h"
#include "LDROIExtraction.h"
#include "WLEParaEstimation.h"
#include "bfgsMLE_GS2D_core.h"
#include "bfgsMLE_AS3D_core.h"
#include "LocPrecCalc_GaussianCRLB.h"
#include "ZeroLocalizationsRemove.h"
#include "ConsecutiveFit.h"
#include "statisticsInfo.h"
#include "ImageRender_2d.h"
#include "ImageRender_3d.h"

#include "../include/qcstorm_b200.h"

// cudaWrapper.cu is not compiled (it only prints); these are its quiet stand-ins.
void HandleErr(cudaError_t, const char *) {}

namespace {

void to_ref(const qcs_loc_para *p, LocalizationPara &r) {
    r.Offset = p->Offset;
    r.KAdc = p->KAdc;
    r.QE = p->QE;
    r.ReadNoise_e = p->ReadNoise_e;
    r.ROISize = p->ROISize;
    r.LocType = p->LocType;
    r.MultiEmitterFitEn = p->MultiEmitterFitEn;
    r.WLEEn = p->WLEEn;
    r.ConsecFit_DistanceTh_nm = p->ConsecFit_DistanceTh_nm;
    r.ConsecFitEn = p->ConsecFitEn;
    r.PixelSize = p->PixelSize;
    r.PixelZoom = p->PixelZoom;
    r.SNR_th = p->SNR_th;
    r.ColorMode_3D = p->ColorMode_3D;
    r.ImageWidth = p->ImageWidth;
    r.ImageHigh = p->ImageHigh;
    r.TotalFrameNum = p->TotalFrameNum;
    r.SRImageWidth = p->SRImageWidth;
    r.SRImageHigh = p->SRImageHigh;
    r.MinZDepth = p->MinZDepth;
    r.MaxZDepth = p->MaxZDepth;
    r.ZDepthCorrFactor = p->ZDepthCorrFactor;
    r.p4_XGY = p->p4_XGY; r.p3_XGY = p->p3_XGY; r.p2_XGY = p->p2_XGY; r.p1_XGY = p->p1_XGY; r.p0_XGY = p->p0_XGY;
    r.p4_XLY = p->p4_XLY; r.p3_XLY = p->p3_XLY; r.p2_XLY = p->p2_XLY; r.p1_XLY = p->p1_XLY; r.p0_XLY = p->p0_XLY;
    r.DH_RotateType = p->DH_RotateType;
    r.DH_MeanDistance = p->DH_MeanDistance;
    r.DH_DistanceTh = p->DH_DistanceTh;
    r.ImagesPerGroup = p->ImagesPerGroup;
    r.IsHollowTube = p->IsHollowTube;
    r.StrucuteSize_2D = p->StrucuteSize_2D;
    r.SpatialResolutionCalcEn = p->SpatialResolutionCalcEn;
}

CoreFittingPara core_para(const LocalizationPara &r) {
    CoreFittingPara c;
    c.MultiEmitterFitEn = r.MultiEmitterFitEn;
    c.WLEEn = r.WLEEn;
    c.Offset = r.Offset;
    c.KAdc = r.KAdc;
    c.QE = r.QE;
    c.ReadNoise_e = r.ReadNoise_e;
    c.ZDepthCorrFactor = r.ZDepthCorrFactor;
    c.p4_XGY = r.p4_XGY; c.p3_XGY = r.p3_XGY; c.p2_XGY = r.p2_XGY; c.p1_XGY = r.p1_XGY; c.p0_XGY = r.p0_XGY;
    c.p4_XLY = r.p4_XLY; c.p3_XLY = r.p3_XLY; c.p2_XLY = r.p2_XLY; c.p1_XLY = r.p1_XLY; c.p0_XLY = r.p0_XLY;
    return c;
}

}  // namespace

extern "C" {

// The reference's default LocalizationPara, field by field.
void qcsref_default_para(qcs_loc_para *p) {
    LocalizationPara r;
    p->Offset = r.Offset; p->KAdc = r.KAdc; p->QE = r.QE; p->ReadNoise_e = r.ReadNoise_e;
    p->ROISize = r.ROISize; p->LocType = r.LocType; p->MultiEmitterFitEn = r.MultiEmitterFitEn; p->WLEEn = r.WLEEn;
    p->ConsecFit_DistanceTh_nm = r.ConsecFit_DistanceTh_nm; p->ConsecFitEn = r.ConsecFitEn;
    p->PixelSize = r.PixelSize; p->PixelZoom = r.PixelZoom; p->SNR_th = r.SNR_th; p->ColorMode_3D = r.ColorMode_3D;
    p->ImageWidth = r.ImageWidth; p->ImageHigh = r.ImageHigh; p->TotalFrameNum = r.TotalFrameNum;
    p->SRImageWidth = r.SRImageWidth; p->SRImageHigh = r.SRImageHigh;
    p->MinZDepth = r.MinZDepth; p->MaxZDepth = r.MaxZDepth; p->ZDepthCorrFactor = r.ZDepthCorrFactor;
    p->p4_XGY = r.p4_XGY; p->p3_XGY = r.p3_XGY; p->p2_XGY = r.p2_XGY; p->p1_XGY = r.p1_XGY; p->p0_XGY = r.p0_XGY;
    p->p4_XLY = r.p4_XLY; p->p3_XLY = r.p3_XLY; p->p2_XLY = r.p2_XLY; p->p1_XLY = r.p1_XLY; p->p0_XLY = r.p0_XLY;
    p->DH_RotateType = r.DH_RotateType; p->DH_MeanDistance = r.DH_MeanDistance; p->DH_DistanceTh = r.DH_DistanceTh;
    p->ImagesPerGroup = r.ImagesPerGroup; p->IsHollowTube = r.IsHollowTube; p->StrucuteSize_2D = r.StrucuteSize_2D;
    p->SpatialResolutionCalcEn = r.SpatialResolutionCalcEn;
}

// LDLocData_TypeDef::BFGS_MLELocalization over n records.
// out: capacity out_cap rows of 12 floats; ratios: 7 floats
// [FitRatio_1E, 2E, 3E, Final_1E, Final_2E, Final_3E, Final_4E].
int qcsref_localize(const qcs_loc_para *p, const unsigned short *rois, const float *wle, int n,
                    float *out, int out_cap, int *n_valid, float *ratios) {
    LocalizationPara r;
    to_ref(p, r);
    LDLocData_TypeDef loc;
    loc.Init(r);
    const int whole = r.ROISize * (r.ROISize + 1);
    int m = n < MaxPointNum ? n : MaxPointNum;
    std::vector<unsigned short> h_roi(rois, rois + (size_t)m * whole);
    std::vector<float> h_wle(wle, wle + (size_t)m * WLE_ParaNumber);
    loc.BFGS_MLELocalization(h_roi.data(), h_wle.data(), r, n, nullptr);
    int nv = loc.oValidFluoNum;
    if (nv > out_cap) nv = out_cap;
    memcpy(out, loc.h_LocArry, sizeof(float) * OutParaNumGS2D * (size_t)nv);
    *n_valid = loc.oValidFluoNum;
    if (ratios) {
        ratios[0] = loc.FitRatio_1E; ratios[1] = loc.FitRatio_2E; ratios[2] = loc.FitRatio_3E;
        ratios[3] = loc.FitRatio_Final_1E; ratios[4] = loc.FitRatio_Final_2E;
        ratios[5] = loc.FitRatio_Final_3E; ratios[6] = loc.FitRatio_Final_4E;
    }
    loc.Deinit(r);
    return 0;
}

// One single-emitter fit kernel launched directly with MultiEmitterFitEn = 0
// semantics for the queue (identity map).  kind 0 = GS2D, 1 = AS3D.
// out: n rows of 12 floats (CRLB columns left as the kernel leaves them).
int qcsref_fit_kernel(int kind, const qcs_loc_para *p, const unsigned short *rois, const float *wle,
                      int n, float *out) {
    LocalizationPara r;
    to_ref(p, r);
    CoreFittingPara c = core_para(r);
    c.MultiEmitterFitEn = 0;
    std::vector<int> single(n), q2(MaxPointNum), q3(MaxPointNum);
    for (int i = 0; i < n; ++i) single[i] = i;
    int n_single = n, n2 = 0, n3 = 0, rej = 0, added = n;
    FitPosInf_TypeDef f;
    memset(&f, 0, sizeof(f));
    f.d_SingleFitFluoNum = &n_single;
    f.d_SingleFitFluoPos = single.data();
    f.d_MultiFitFluoNum_2E = &n2;
    f.d_MultiFitFluoPos_2E = q2.data();
    f.d_MultiFitFluoNum_3E = &n3;
    f.d_MultiFitFluoPos_3E = q3.data();
    f.d_RejectedFluoNum = &rej;
    f.d_MultiFit_AddedFluoNum = &added;
    const int whole = r.ROISize * (r.ROISize + 1);
    std::vector<unsigned short> d_roi(rois, rois + (size_t)n * whole);
    std::vector<float> d_wle(wle, wle + (size_t)n * WLE_ParaNumber);
    std::vector<float> d_loc((size_t)n * OutParaNumGS2D, 0.0f);
    qcs_emu_cfg cfg((n + ThreadsPerBlock - 1) / ThreadsPerBlock, ThreadsPerBlock);
#define QCSREF_CASE(KIND, R, KERNEL)                                                              \
    if (kind == KIND && r.ROISize == R) {                                                         \
        cfg.run((KERNEL), d_loc.data(), d_roi.data(), d_wle.data(), n, &f, &c);                    \
        memcpy(out, d_loc.data(), sizeof(float) * d_loc.size());                                  \
        return 0;                                                                                 \
    }
    QCSREF_CASE(0, 5, (bfgsMLELoc_Gauss2D<5, FitParaNum_2D>))
    QCSREF_CASE(0, 7, (bfgsMLELoc_Gauss2D<7, FitParaNum_2D>))
    QCSREF_CASE(0, 9, (bfgsMLELoc_Gauss2D<9, FitParaNum_2D>))
    QCSREF_CASE(0, 11, (bfgsMLELoc_Gauss2D<11, FitParaNum_2D>))
    QCSREF_CASE(0, 13, (bfgsMLELoc_Gauss2D<13, FitParaNum_2D>))
    QCSREF_CASE(1, 5, (bfgsMLELoc_AS3D<5, FitParaNum_AS3D>))
    QCSREF_CASE(1, 7, (bfgsMLELoc_AS3D<7, FitParaNum_AS3D>))
    QCSREF_CASE(1, 9, (bfgsMLELoc_AS3D<9, FitParaNum_AS3D>))
    QCSREF_CASE(1, 11, (bfgsMLELoc_AS3D<11, FitParaNum_AS3D>))
    QCSREF_CASE(1, 13, (bfgsMLELoc_AS3D<13, FitParaNum_AS3D>))
#undef QCSREF_CASE
    return 2;
}

// GaussianCRLB_Calc_top over n 12-float rows, in place.  The reference kernel
// has no bounds guard, so rows are padded to a multiple of 32 here.
int qcsref_crlb(const qcs_loc_para *p, float *loc, int n) {
    LocalizationPara r;
    to_ref(p, r);
    const int blocks = (n + ThreadsPerBlock - 1) / ThreadsPerBlock;
    std::vector<float> d_loc((size_t)blocks * ThreadsPerBlock * OutParaNumGS2D, 0.0f);
    memcpy(d_loc.data(), loc, sizeof(float) * OutParaNumGS2D * (size_t)n);
    LDLocData_TypeDef::LocPrecCalc_GaussianCRLB(d_loc.data(), r, n, nullptr);
    memcpy(loc, d_loc.data(), sizeof(float) * OutParaNumGS2D * (size_t)n);
    return 0;
}

// WLEParameterEstimate over n records; wle_out: n rows of 6 floats.
int qcsref_wle(const qcs_loc_para *p, const unsigned short *rois, int n, float *wle_out) {
    // WLEParameterEstimation_TypeDef sizes its buffers for MaxPointNum records
    if (n < 0 || n > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    WLEParameterEstimation_TypeDef w;
    w.Init(r);
    const int whole = r.ROISize * (r.ROISize + 1);
    std::vector<unsigned short> d_roi(rois, rois + (size_t)n * whole);
    w.WLEParameterEstimate(d_roi.data(), r.LocType, r.MultiEmitterFitEn, r.ROISize, n, nullptr);
    memcpy(wle_out, w.d_WLEPara, sizeof(float) * WLE_ParaNumber * (size_t)n);
    w.Deinit();
    return 0;
}

// ExtractMolecules over consecutive batches of frames (the JNI feeding
// pattern), accumulating ROI records and WLE rows.  batch: frames per call.
int qcsref_extract(const qcs_loc_para *p, const unsigned short *frames, int n_frames, int batch,
                   int start_frame, unsigned short *rois_out, float *wle_out, int cap, int *n_roi,
                   int *first_frame, int *end_frame) {
    LocalizationPara r;
    to_ref(p, r);
    LDROIExtractData_TypeDef ex;
    ex.Init(r);
    ex.ResetROINum();
    const size_t frame_px = (size_t)r.ImageWidth * r.ImageHigh;
    for (int f = 0; f < n_frames; f += batch) {
        int nb = (n_frames - f) < batch ? (n_frames - f) : batch;
        std::vector<unsigned short> buf(frames + f * frame_px, frames + (f + nb) * frame_px);
        ex.ExtractMolecules(buf.data(), ImageSource_CPU_Pinned, r, start_frame + f, nb, nullptr);
    }
    int n = ex.GetAccumulatedROINum();
    *n_roi = n;
    if (n > cap) n = cap;
    const int whole = r.ROISize * (r.ROISize + 1);
    memcpy(rois_out, ex.h_ImageROI, sizeof(unsigned short) * whole * (size_t)n);
    memcpy(wle_out, ex.Get_h_WLEPara(), sizeof(float) * WLE_ParaNumber * (size_t)n);
    *first_frame = ex.FirstFrame;
    *end_frame = ex.EndFrame;
    ex.Deinit();
    return 0;
}

// RemoveZeroLocalizations over n rows (ZeroLocalizationsRemove.cu:21-39);
// n must fit its MaxPointNum buffers.
int qcsref_zero_remove(const float *rows, int n, int sort_frame, int first_frame, int end_frame, float *out,
                       int *n_out) {
    if (n < 0 || n > MaxPointNum) return -1;
    ZeroLocalizationsRemovel_TypeDef z;
    z.Init();
    std::vector<float> in(rows, rows + (size_t)n * 12);
    z.RemoveZeroLocalizations(in.data(), n, sort_frame, first_frame, end_frame, nullptr);
    *n_out = z.ValidFluoNum;
    memcpy(out, z.h_LocArry, sizeof(float) * 12 * (size_t)z.ValidFluoNum);
    z.Deinit();
    return 0;
}

// ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg (ConsecutiveFit_top.cu:22-98)
// called once per group on one object: group g is sizes[g] rows (<= MaxPointNum)
// taken in turn from rows, the call's IsEndProc is is_end[g]; each call's
// OutFluoNum rows go to out back to back, their count to out_n[g] and the
// call's h_OntimeRatio (MaxOnTimeConsecutiveNum floats) to ontime[g * 10].
int qcsref_consec(const qcs_loc_para *p, const float *rows, const int *sizes, const int *is_end, int n_groups,
                  float *out, int *out_n, float *ontime) {
    for (int g = 0; g < n_groups; ++g)
        if (sizes[g] < 0 || sizes[g] > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    ConsecutiveFit_TypeDef cf;
    cf.Init();
    size_t off = 0, oo = 0;
    for (int g = 0; g < n_groups; ++g) {
        std::vector<float> in(rows + off * 12, rows + (off + (size_t)sizes[g]) * 12);
        cf.ConsecutiveFit_WeightedAvg(in.data(), sizes[g], is_end[g], r, nullptr);
        out_n[g] = cf.OutFluoNum;
        memcpy(out + oo * 12, cf.h_OutLocArry, sizeof(float) * 12 * (size_t)cf.OutFluoNum);
        memcpy(ontime + (size_t)g * MaxOnTimeConsecutiveNum, cf.h_OntimeRatio, sizeof(float) * MaxOnTimeConsecutiveNum);
        oo += (size_t)cf.OutFluoNum;
        off += (size_t)sizes[g];
    }
    cf.Deinit();
    return 0;
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

// FluoStatisticData_TypeDef (StatisticsInfo/statisticsInfo_top.cu:61-255): Init,
// ResetAllDat, then GetStatisticalInf once per group of sizes[g] rows (<=
// MaxPointNum) taken in turn from rows.  After call g: hist[g * 4 * 1600 ..]
// the four histograms (total photons, localization precision, peak SNR, PSF
// width; StatInf_Hist_DatLenMax bins each) and means[g * 10 ..] MeanTotalPhoton,
// MeanLocPrecisionXY, MeanPeakSNR, MeanBackground, MeanPSFWidth,
// MeanPSFWidth_Ctl, MeanLocDensity2D, TimeVaryMean_TotalPhoton,
// TimeVaryMean_LocPrecisionXY, TimeVaryMean_PeakSNR.
int qcsref_stat(const qcs_loc_para *p, const float *rows, const int *sizes, int n_groups, int *hist, float *means) {
    for (int g = 0; g < n_groups; ++g)
        if (sizes[g] < 0 || sizes[g] > MaxPointNum) return -1;
    LocalizationPara r;
    to_ref(p, r);
    FluoStatisticData_TypeDef sd;
    sd.Init();
    sd.ResetAllDat(nullptr);
    size_t off = 0;
    for (int g = 0; g < n_groups; ++g) {
        std::vector<float> in(rows + off * 12, rows + (off + (size_t)sizes[g]) * 12);
        sd.GetStatisticalInf(in.data(), r, sizes[g], nullptr);
        stat_out(sd, g, hist, means);
        off += (size_t)sizes[g];
    }
    sd.Deinit();
    return 0;
}

// FluoStatisticData_TypeDef::UpdateOntimeRatio (StatisticsInfo/statisticsInfo_top.cu:23-57)
// once per call c on ratios[c * MaxOnTimeConsecutiveNum ..] in turn, on one
// object: after call c, mean[c] = MeanOntime and out[c * 10 ..] = h_OntimeRatio.
// The function touches only h_OntimeRatio, MeanOntime and the four on-time time
// series, so the object's device buffers are not set up.
int qcsref_ontime(const float *ratios, int n_calls, float *mean, float *out) {
    FluoStatisticData_TypeDef sd;
    std::vector<float> buf(MaxOnTimeConsecutiveNum);
    sd.h_OntimeRatio = buf.data();
    for (int c = 0; c < n_calls; ++c) {
        std::vector<float> in(ratios + (size_t)c * MaxOnTimeConsecutiveNum,
                              ratios + (size_t)(c + 1) * MaxOnTimeConsecutiveNum);
        sd.UpdateOntimeRatio(in.data());
        mean[c] = sd.MeanOntime;
        memcpy(out + (size_t)c * MaxOnTimeConsecutiveNum, sd.h_OntimeRatio, sizeof(float) * MaxOnTimeConsecutiveNum);
    }
    if ((int)sd.TimeVary_OntimeF1Ratio.size() != n_calls) return -2;
    sd.h_OntimeRatio = nullptr;
    return 0;
}

// ImageRenderData_TypeDef::FluoRenderTop's device part (ImageRender_top.cu:29-60):
// the reference's FluoRenderWithPrec_2D / _3D launchers (ImageRender_2d.cu:372,
// ImageRender_3d.cu:333) on a render object holding only the buffers they
// touch.  img, colormap (3D only; may be NULL for 2D), max_val and hist (400
// ints) are read as the starting state and written back.
int qcsref_render(const qcs_loc_para *p, const float *rows, int n, int mode, float fixed_prec, float *img, float *colormap,
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
    int st = 0;
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
