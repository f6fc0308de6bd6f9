/*
 * qcstorm_b200 -- C++ façade with the class names, public members and member
 * signatures of the reference's exported localization classes
 * (MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/x64/Release/bfgs_MLE_dll.h:52-461), so
 * that code written against them (the ImageJ / Micro-Manager JNI workers,
 * the batch drivers) recompiles unchanged against this header and links
 * libqcstorm_b200.so.  Header-only: every member forwards to the C ABI in
 * qcstorm_b200.h.  A source-level drop-in: MSVC class layouts are not
 * binary-matched.
 *
 *   LocalizationPara                 (bfgs_MLE_dll.h:52-141)
 *   WLEParameterEstimation_TypeDef   (bfgs_MLE_dll.h:203-217)
 *   LDROIExtractData_TypeDef         (bfgs_MLE_dll.h:222-301)
 *   LDLocData_TypeDef                (bfgs_MLE_dll.h:308-373)
 *   ZeroLocalizationsRemovel_TypeDef (bfgs_MLE_dll.h:425-453)
 *
 * Like the reference, members return void and report CUDA failures by
 * printing (HandleErr); the C ABI's status codes are available through
 * qcs_last_error().  Calls that the reference makes synchronous
 * (ExtractMolecules, BFGS_MLELocalization, RemoveZeroLocalizations) are
 * synchronous here too, so public host pointers hold the results on return.
 */
#ifndef QCSTORM_B200_HPP
#define QCSTORM_B200_HPP

#include <cstdio>
#include <cuda_runtime_api.h>

#include "qcstorm_b200.h"

/* constants of bfgs_CommonPara.h:37-85 and WLEParaEstimation_Parameters.h:20-34 */
#ifndef LocType_GS2D
#define LocType_GS2D QCS_LOCTYPE_GS2D
#define LocType_AS3D QCS_LOCTYPE_AS3D
#define LocType_DH3D QCS_LOCTYPE_DH3D
#endif
#ifndef ImageSource_GPU
#define ImageSource_GPU QCS_IMAGE_SOURCE_GPU
#define ImageSource_CPU_Pinned QCS_IMAGE_SOURCE_CPU_PINNED
#define ImageSource_CPU_Normal QCS_IMAGE_SOURCE_CPU_NORMAL
#endif
#ifndef MaxPointNum
#define MaxPointNum QCS_MAX_POINT_NUM
#endif
#ifndef OutParaNumGS2D
#define OutParaNumGS2D QCS_OUT_PARA_NUM
#define Pos_PPho QCS_POS_PPHO
#define Pos_XPos QCS_POS_XPOS
#define Pos_YPos QCS_POS_YPOS
#define Pos_ZPos QCS_POS_ZPOS
#define Pos_SigX QCS_POS_SIGX
#define Pos_SigY QCS_POS_SIGY
#define Pos_TPho QCS_POS_TPHO
#define Pos_Bakg QCS_POS_BAKG
#define Pos_PSNR QCS_POS_PSNR
#define Pos_CrbX QCS_POS_CRBX
#define Pos_CrbY QCS_POS_CRBY
#define Pos_Frme QCS_POS_FRME

// ImgRender/ImageRender_base.h:27, 36-39
#define ImgRend_MaxDatHistLen QCS_RENDER_HIST_LEN
#define RenderingMode_FittedPhoton_CalculatedLocPrec QCS_RENDER_FITTED_PHOTON_CRLB
#define RenderingMode_1Photon_CalculatedLocPrec QCS_RENDER_1PHOTON_CRLB
#define RenderingMode_1Photon_FixedLocPrec QCS_RENDER_1PHOTON_FIXED
#define RenderingMode_FittedPhoton_1Pixel QCS_RENDER_FITTED_PHOTON_1PIXEL
#endif
#ifndef WLE_ParaNumber
#define WLE_ParaNumber QCS_WLE_PARA_NUM
#define MoleculeType_MLEFit QCS_MOLECULE_MLEFIT
#define MoleculeType_WLEFit QCS_MOLECULE_WLEFIT
#define MoleculeType_MultiFit QCS_MOLECULE_MULTIFIT
#endif

namespace qcs_facade {
inline void report(int status, const char *what) {
    if (status != QCS_OK) printf("qcstorm_b200 %s: %s\n", what, qcs_last_error());
}
}  // namespace qcs_facade

// The reference's parameter class: same fields in the same order (the C
// struct is its first and only base), same constructor defaults.
class LocalizationPara : public qcs_loc_para {
public:
    LocalizationPara() { qcs_loc_para_default(this); }
    // bfgs_base.cu:89-98
    void UpdateSRImageSize() {
        SRImageWidth = ((int)(ImageWidth * PixelZoom) + 3) / 4 * 4;
        SRImageHigh = ((int)(ImageHigh * PixelZoom) + 3) / 4 * 4;
    }
    // bfgs_base.cu:100-175: every field equal
    bool IsEqual(LocalizationPara &o) {
        const qcs_loc_para &a = *this, &b = o;
        return a.Offset == b.Offset && a.KAdc == b.KAdc && a.QE == b.QE && a.ReadNoise_e == b.ReadNoise_e &&
               a.ROISize == b.ROISize && a.LocType == b.LocType && a.MultiEmitterFitEn == b.MultiEmitterFitEn &&
               a.WLEEn == b.WLEEn && a.ConsecFit_DistanceTh_nm == b.ConsecFit_DistanceTh_nm &&
               a.ConsecFitEn == b.ConsecFitEn && a.PixelSize == b.PixelSize && a.PixelZoom == b.PixelZoom &&
               a.SNR_th == b.SNR_th && a.ColorMode_3D == b.ColorMode_3D && a.ImageWidth == b.ImageWidth &&
               a.ImageHigh == b.ImageHigh && a.TotalFrameNum == b.TotalFrameNum && a.SRImageWidth == b.SRImageWidth &&
               a.SRImageHigh == b.SRImageHigh && a.MinZDepth == b.MinZDepth && a.MaxZDepth == b.MaxZDepth &&
               a.ZDepthCorrFactor == b.ZDepthCorrFactor && a.p4_XGY == b.p4_XGY && a.p3_XGY == b.p3_XGY &&
               a.p2_XGY == b.p2_XGY && a.p1_XGY == b.p1_XGY && a.p0_XGY == b.p0_XGY && a.p4_XLY == b.p4_XLY &&
               a.p3_XLY == b.p3_XLY && a.p2_XLY == b.p2_XLY && a.p1_XLY == b.p1_XLY && a.p0_XLY == b.p0_XLY &&
               a.DH_RotateType == b.DH_RotateType && a.DH_MeanDistance == b.DH_MeanDistance &&
               a.DH_DistanceTh == b.DH_DistanceTh && a.ImagesPerGroup == b.ImagesPerGroup &&
               a.IsHollowTube == b.IsHollowTube && a.StrucuteSize_2D == b.StrucuteSize_2D &&
               a.SpatialResolutionCalcEn == b.SpatialResolutionCalcEn;
    }
};

// WLE pre-pass on device records (bfgs_MLE_dll.h:203-217).
class WLEParameterEstimation_TypeDef {
public:
    float *h_WLEPara = nullptr;
    float *d_WLEPara = nullptr;

    void Init(LocalizationPara &LocPara) {
        qcs_facade::report(qcs_loc_init(&LocPara, &ctx_), "WLEParameterEstimation_TypeDef::Init");
        if (ctx_) {
            d_WLEPara = qcs_loc_device_wle_buffer(ctx_);
            cudaMallocHost((void **)&h_WLEPara, sizeof(float) * WLE_ParaNumber * MaxPointNum);
        }
        para_ = LocPara;
    }
    void Deinit() {
        if (h_WLEPara) cudaFreeHost(h_WLEPara);
        qcs_loc_deinit(ctx_);
        ctx_ = nullptr;
        h_WLEPara = d_WLEPara = nullptr;
    }
    // d_ImageROI: device records; results in d_WLEPara (WLEParaEstimation.cpp:20-40)
    void WLEParameterEstimate(unsigned short *d_ImageROI, int LocType, int MultiEmitterFitEn, int ROISize, int FluoNum,
                              cudaStream_t cstream) {
        qcs_loc_para p = para_;
        p.LocType = LocType;
        p.MultiEmitterFitEn = MultiEmitterFitEn;
        p.ROISize = ROISize;
        qcs_facade::report(qcs_wle_estimate_device(ctx_, d_ImageROI, FluoNum, &p, d_WLEPara, cstream),
                           "WLEParameterEstimate");
        cudaStreamSynchronize(cstream);
    }

private:
    qcs_loc_data *ctx_ = nullptr;
    qcs_loc_para para_{};
};

// ROI extraction (bfgs_MLE_dll.h:222-301).  h_ImageROI / Get_h_WLEPara()
// hold the accumulated records and WLE rows after every ExtractMolecules;
// d_ImageROI is the device accumulation buffer (the reference's holds only
// the last batch).
class LDROIExtractData_TypeDef {
public:
    unsigned short *h_RawImg = nullptr;
    unsigned short *d_RawImg = nullptr;
    unsigned short *h_ImageROI = nullptr;
    unsigned short *d_ImageROI = nullptr;
    int FirstFrame = -1;
    int EndFrame = -1;
    WLEParameterEstimation_TypeDef *WLEParameterEstimator = nullptr;

    void Init(LocalizationPara &LocPara) {
        qcs_facade::report(qcs_extract_init(&LocPara, &ex_), "LDROIExtractData_TypeDef::Init");
        if (!ex_) return;
        d_ImageROI = const_cast<unsigned short *>(qcs_extract_d_image_roi(ex_));
        WLEParameterEstimator = &wle_view_;
        wle_view_.d_WLEPara = const_cast<float *>(qcs_extract_d_wle_para(ex_));
        refresh();
    }
    void Deinit() {
        qcs_extract_deinit(ex_);
        ex_ = nullptr;
        h_ImageROI = d_ImageROI = nullptr;
        WLEParameterEstimator = nullptr;
    }
    void ExtractMolecules(unsigned short *pImgData, int ImageSource, LocalizationPara &LocPara, int StartFrame_CurBatch,
                          int BatchedImageNum, cudaStream_t cstream) {
        qcs_facade::report(
            qcs_extract_molecules(ex_, pImgData, ImageSource, &LocPara, StartFrame_CurBatch, BatchedImageNum, cstream),
            "ExtractMolecules");
        refresh();
    }
    int GetAccumulatedROINum() {
        int n = 0;
        qcs_facade::report(qcs_extract_accumulated_roi_num(ex_, &n), "GetAccumulatedROINum");
        return n;
    }
    void ResetROINum() {
        qcs_facade::report(qcs_extract_reset_roi_num(ex_, nullptr), "ResetROINum");
        FirstFrame = -1;
        EndFrame = -1;
    }
    float *Get_h_WLEPara() { return const_cast<float *>(qcs_extract_h_wle_para(ex_)); }
    float *Get_d_WLEPara() { return const_cast<float *>(qcs_extract_d_wle_para(ex_)); }
    static int GetMaxBatchedNumForCurrentImageSize(int ImageWidth, int ImageHigh) {
        return qcs_extract_max_batched_num(ImageWidth, ImageHigh);
    }

private:
    void refresh() {
        h_ImageROI = const_cast<unsigned short *>(qcs_extract_h_image_roi(ex_));
        wle_view_.h_WLEPara = const_cast<float *>(qcs_extract_h_wle_para(ex_));
        qcs_extract_frame_range(ex_, &FirstFrame, &EndFrame);
    }
    qcs_extract_data *ex_ = nullptr;
    WLEParameterEstimation_TypeDef wle_view_;
};

// Localization (bfgs_MLE_dll.h:308-373).
class LDLocData_TypeDef {
public:
    unsigned short *h_ImageROI = nullptr;
    unsigned short *d_ImageROI = nullptr;
    float *d_WLEPara = nullptr;
    float *h_LocArry = nullptr;
    float *d_LocArry = nullptr;
    int oValidFluoNum = 0;
    float FitRatio_1E = 0, FitRatio_2E = 0, FitRatio_3E = 0;
    float FitRatio_Final_1E = 0, FitRatio_Final_2E = 0, FitRatio_Final_3E = 0, FitRatio_Final_4E = 0;

    void Init(LocalizationPara &LocPara) {
        qcs_facade::report(qcs_loc_init(&LocPara, &ctx_), "LDLocData_TypeDef::Init");
        if (!ctx_) return;
        d_ImageROI = qcs_loc_device_roi_buffer(ctx_);
        d_WLEPara = qcs_loc_device_wle_buffer(ctx_);
        d_LocArry = const_cast<float *>(qcs_loc_device_rows(ctx_));
        h_LocArry = const_cast<float *>(qcs_loc_h_loc_arry(ctx_));
    }
    void Deinit(LocalizationPara &) {
        qcs_loc_deinit(ctx_);
        ctx_ = nullptr;
        h_LocArry = d_LocArry = nullptr;
        d_ImageROI = nullptr;
        d_WLEPara = nullptr;
    }
    void BFGS_MLELocalization(unsigned short *h_ImageROI_in, float *h_WLEPara, LocalizationPara &LocPara, int FluoNum,
                              cudaStream_t cstream) {
        // the reference clamps FluoNum to MaxPointNum (bfgs_top.cu:36)
        if (FluoNum > MaxPointNum) FluoNum = MaxPointNum;
        qcs_facade::report(qcs_loc_bfgs_mle_localization(ctx_, h_ImageROI_in, h_WLEPara, &LocPara, FluoNum, cstream),
                           "BFGS_MLELocalization");
        oValidFluoNum = qcs_loc_valid_num(ctx_);
        float r[7] = {0, 0, 0, 0, 0, 0, 0};
        qcs_loc_fit_ratios(ctx_, r);
        FitRatio_1E = r[0];
        FitRatio_2E = r[1];
        FitRatio_3E = r[2];
        FitRatio_Final_1E = r[3];
        FitRatio_Final_2E = r[4];
        FitRatio_Final_3E = r[5];
        FitRatio_Final_4E = r[6];
    }
    // bfgs_top.cu:345-380: first / last nonzero frame of rows sorted by frame
    static int GetFirstFrame(float *h_LocArry_in, int FluoNum) {
        int f = 0;
        for (int i = 0; i < FluoNum; i++) {
            f = (int)h_LocArry_in[i * OutParaNumGS2D + Pos_Frme];
            if (f != 0) break;
        }
        return f;
    }
    static int GetLastFrame(float *h_LocArry_in, int FluoNum) {
        int f = 0;
        for (int i = FluoNum - 1; i > 0; i--) {
            f = (int)h_LocArry_in[i * OutParaNumGS2D + Pos_Frme];
            if (f != 0) break;
        }
        return f;
    }
    // LocPrecCalc_GaussianCRLB.cu:23-40: CRLB columns of FluoNum device rows
    static void LocPrecCalc_GaussianCRLB(float *d_LocArry_in, LocalizationPara &LocPara, int FluoNum,
                                         cudaStream_t cstream) {
        qcs_facade::report(qcs_crlb_device(&LocPara, d_LocArry_in, FluoNum, cstream), "LocPrecCalc_GaussianCRLB");
        cudaStreamSynchronize(cstream);
    }

private:
    qcs_loc_data *ctx_ = nullptr;
};

// Zero-row removal (bfgs_MLE_dll.h:425-453).
class ZeroLocalizationsRemovel_TypeDef {
public:
    int ValidFluoNum = 0;
    float *h_LocArry = nullptr;

    void RemoveZeroLocalizations(float *ih_LocArry, int iFluoNum, int SortFrameEn, int FirstFrame, int EndFrame,
                                 cudaStream_t cstream) {
        qcs_facade::report(qcs_zero_remove(z_, ih_LocArry, iFluoNum, SortFrameEn, FirstFrame, EndFrame, cstream),
                           "RemoveZeroLocalizations");
        ValidFluoNum = qcs_zero_valid_num(z_);
        h_LocArry = const_cast<float *>(qcs_zero_h_loc_arry(z_));
    }
    void Init() {
        qcs_facade::report(qcs_zero_init(0, &z_), "ZeroLocalizationsRemovel_TypeDef::Init");
        ValidFluoNum = 0;
        h_LocArry = z_ ? const_cast<float *>(qcs_zero_h_loc_arry(z_)) : nullptr;
    }
    void Deinit() {
        qcs_zero_deinit(z_);
        z_ = nullptr;
        h_LocArry = nullptr;
    }

private:
    qcs_zero_data *z_ = nullptr;
};

// ImgRender/ImageRender_top.h: the super-resolution render of localization
// rows.  d_SRIntensityImg / d_SRColorMapImg point at the device images; the
// display-image helpers (GetDispImgTop, GetSaveImgTop) are not provided.
class ImageRenderData_TypeDef {
public:
    float *d_SRIntensityImg = nullptr;
    float *d_SRColorMapImg = nullptr;

    void Init(LocalizationPara &LocPara, int /*MaxDispImgWidth*/ = 0, int /*MaxDispImgHigh*/ = 0) {
        qcs_facade::report(qcs_render_init(&LocPara, 0, &r_), "ImageRenderData_TypeDef::Init");
        d_SRIntensityImg = r_ ? qcs_render_d_image(r_) : nullptr;
        d_SRColorMapImg = r_ ? qcs_render_d_colormap(r_) : nullptr;
    }
    void Deinit(LocalizationPara & /*LocPara*/) {
        qcs_render_deinit(r_);
        r_ = nullptr;
        d_SRIntensityImg = d_SRColorMapImg = nullptr;
    }
    void FluoRenderTop(float *h_LocArry, LocalizationPara &LocPara, int RenderingMode, float FixedlocPrec, int FluoNum,
                       cudaStream_t cstream) {
        qcs_facade::report(qcs_render_rows(r_, h_LocArry, &LocPara, RenderingMode, FixedlocPrec, FluoNum, cstream),
                           "FluoRenderTop");
    }
    void ResetFillImgTop(LocalizationPara & /*LocPara*/) {
        qcs_facade::report(qcs_render_reset(r_, nullptr), "ResetFillImgTop");
    }
    // Mode 0: maximum and histogram to zero (the rescale, mode 1, runs on the
    // device inside FluoRenderTop)
    void ResetFillMaxVal(int Mode) {
        if (Mode == 0) qcs_facade::report(qcs_render_reset_max(r_, nullptr), "ResetFillMaxVal");
    }
    qcs_render_data *handle() { return r_; }

private:
    qcs_render_data *r_ = nullptr;
};

#endif /* QCSTORM_B200_HPP */
