/*
 * qcstorm_b200 -- C ABI of the B200-native QC-STORM MLEbfgs localization path.
 *
 * This is the drop-in boundary for the path that the QC-STORM JNI layers
 * (ImageJ "QC-STORM_ CPPDLL", Micro-Manager "QC-STORM CPPDLL") and the batch
 * drivers drive through the reference's exported C++ classes
 * (MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/x64/Release/bfgs_MLE_dll.h):
 *
 *   reference                                            this ABI
 *   -------------------------------------------------    -------------------------------
 *   LocalizationPara (bfgs_base.h:26-110)                 qcs_loc_para (same fields, order)
 *   LocalizationPara::LocalizationPara() (bfgs_base.cu:18) qcs_loc_para_default
 *   LDROIExtractData_TypeDef (LDROIExtraction.h)          qcs_extract_*
 *   LDLocData_TypeDef (bfgs_top.h)                         qcs_loc_*
 *   WLEParameterEstimation_TypeDef (WLEParaEstimation.h)  qcs_wle_estimate
 *
 * Every function returns a status code (QCS_OK == 0); the reference returns
 * void and only prints CUDA errors, so a caller that ignores the status sees
 * the reference's behaviour.  Plain pointers and sizes only; no C++ types.
 *
 * Record formats (identical to the reference):
 *   ROI record   ROISize*(ROISize+1) uint16: ROISize^2 pixels (row-major, ADU)
 *                then header words [x, y, frame%65536, frame/65536, detector
 *                type] (LDROIExtraction_ROIExtraction.cu:280-298).
 *   WLE record   6 float: [nearest-neighbour distance, sigmaL, sigmaR, sigmaU,
 *                sigmaD, molecule type] (WLEParaEstimation_Parameters.h:20-28).
 *   Loc record   12 float: [peak photon, x, y, z nm, sigma x, sigma y, total
 *                photon, background, SNR, CRLB x nm, CRLB y nm, frame]
 *                (bfgs_CommonPara.h:296-309).
 */
#ifndef QCSTORM_B200_H
#define QCSTORM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define QCS_OK 0
#define QCS_ERR_ARG 1          /* null pointer, negative count, bad enum      */
#define QCS_ERR_ROISIZE 2      /* ROI size not supported by the fit kind      */
#define QCS_ERR_CAPACITY 3     /* count above the context's capacity          */
#define QCS_ERR_CUDA 4         /* CUDA runtime error (see qcs_last_error)     */
#define QCS_ERR_NOMEM 5        /* host or device allocation failed            */
#define QCS_ERR_STATE 6        /* context used after deinit / wrong order     */
#define QCS_ERR_NOT_BUILT 7    /* library built without CUDA support          */

/* ---- constants, same values as the reference ----------------------------- */
/* localization type (bfgs_CommonPara.h:275-277) */
#define QCS_LOCTYPE_GS2D 0
#define QCS_LOCTYPE_AS3D 1
#define QCS_LOCTYPE_DH3D 2
/* image source of qcs_extract_molecules (bfgs_CommonPara.h:319-323) */
#define QCS_IMAGE_SOURCE_GPU 0
#define QCS_IMAGE_SOURCE_CPU_PINNED 1
#define QCS_IMAGE_SOURCE_CPU_NORMAL 2
/* record sizes and capacity (bfgs_CommonPara.h:292-316, WLEParaEstimation_Parameters.h:20) */
#define QCS_OUT_PARA_NUM 12
#define QCS_WLE_PARA_NUM 6
#define QCS_MAX_POINT_NUM (20480 * 5)
/* output columns (bfgs_CommonPara.h:298-309) */
#define QCS_POS_PPHO 0
#define QCS_POS_XPOS 1
#define QCS_POS_YPOS 2
#define QCS_POS_ZPOS 3
#define QCS_POS_SIGX 4
#define QCS_POS_SIGY 5
#define QCS_POS_TPHO 6
#define QCS_POS_BAKG 7
#define QCS_POS_PSNR 8
#define QCS_POS_CRBX 9
#define QCS_POS_CRBY 10
#define QCS_POS_FRME 11

/* Super-resolution rendering modes (ImgRender/ImageRender_base.h:36-39) and
 * the length of the display-intensity histogram (:27). */
#define QCS_RENDER_FITTED_PHOTON_CRLB 0   /* weight peak photons, width from the CRLB */
#define QCS_RENDER_1PHOTON_CRLB 1         /* weight 1, width from the CRLB */
#define QCS_RENDER_1PHOTON_FIXED 2        /* weight 1, fixed width */
#define QCS_RENDER_FITTED_PHOTON_1PIXEL 3 /* weight peak photons, one pixel (2D) */
#define QCS_RENDER_HIST_LEN 400
/* molecule type in WLE record column 5 (WLEParaEstimation_Parameters.h:32-34) */
#define QCS_MOLECULE_MLEFIT 0
#define QCS_MOLECULE_WLEFIT 1
#define QCS_MOLECULE_MULTIFIT 2
/* detector ROI type in record header word 4 (LDROIExtraction_Param.h:53-54) */
#define QCS_ROITYPE_SINGLE 0
#define QCS_ROITYPE_MULTI 1

/*
 * Localization parameters.  Field names, types and order are those of the
 * reference's LocalizationPara (bfgs_base.h:26-99), so a JNI layer that fills
 * LocalizationPara field by field (QC_STORM_CPPDLL.cpp:33-143) fills this
 * struct the same way.  Fields outside the localization path (rendering,
 * consecutive fit, double helix, spatial resolution) are carried, not used.
 */
typedef struct qcs_loc_para {
    /* camera */
    float Offset;       /* ADU */
    float KAdc;         /* e-/ADU */
    float QE;           /* e-/photon */
    float ReadNoise_e;  /* e- */
    /* localization */
    int ROISize;
    int LocType;
    int MultiEmitterFitEn;
    int WLEEn;
    /* consecutive molecule filter (carried) */
    float ConsecFit_DistanceTh_nm;
    int ConsecFitEn;
    /* rendering (PixelSize is used by the CRLB, the rest is carried) */
    float PixelSize;
    float PixelZoom;
    float SNR_th;
    int ColorMode_3D;
    /* raw image size */
    int ImageWidth;
    int ImageHigh;
    int TotalFrameNum;
    int SRImageWidth;
    int SRImageHigh;
    /* astigmatic 3D calibration */
    float MinZDepth;
    float MaxZDepth;
    float ZDepthCorrFactor;
    float p4_XGY, p3_XGY, p2_XGY, p1_XGY, p0_XGY; /* sigma x >= sigma y */
    float p4_XLY, p3_XLY, p2_XLY, p1_XLY, p0_XLY; /* sigma x <  sigma y */
    /* double helix (carried) */
    int DH_RotateType;
    float DH_MeanDistance;
    float DH_DistanceTh;
    /* spatial resolution (carried) */
    int ImagesPerGroup;
    int IsHollowTube;
    float StrucuteSize_2D;
    int SpatialResolutionCalcEn;
} qcs_loc_para;

/* Fill with the reference's defaults (bfgs_base.cu:18-86). */
void qcs_loc_para_default(qcs_loc_para *p);

/* Text of the last error on the calling thread ("" if none). */
const char *qcs_last_error(void);

/* 1 if the library found a usable CUDA device, else 0. */
int qcs_device_available(void);

/* ---- ROI extraction: LDROIExtractData_TypeDef --------------------------- */
/*
 * Molecule detection and ROI cutting on batches of raw frames
 * (SubregionExtraction/LDROIExtraction.h:35-93): background removal, image
 * variance, 5-tap Gaussian smoothing, 3x3 local-maximum detection,
 * single/multi classification, ROI records with header, and the WLE pre-pass
 * of the new records.  Records and WLE rows accumulate in device memory
 * across calls until qcs_extract_reset_roi_num, like TotalROINumber.
 * Differences a caller can see: a batch's records come in pixel order
 * (y * width + x over the stacked batch) instead of GPU arrival order; the
 * variance comes from exact integer sums (the reference's float atomics
 * vary run to run); detections beyond QCS_MAX_POINT_NUM per batch or beyond
 * the context capacity are dropped and counted (qcs_extract_dropped_num)
 * instead of overrunning buffers; frames already in device memory
 * (QCS_IMAGE_SOURCE_GPU) are read in place, which the reference rejects.
 */
typedef struct qcs_extract_data qcs_extract_data;

/* LDROIExtractData_TypeDef::GetMaxBatchedNumForCurrentImageSize
 * (LDROIExtraction.h:86, LDROIExtraction.cu:207-216). */
int qcs_extract_max_batched_num(int image_width, int image_high);
/* LDROIExtractData_TypeDef::Init(LocalizationPara&) (LDROIExtraction.cu:219-286):
 * frame buffers for qcs_extract_max_batched_num frames of ImageWidth x
 * ImageHigh, QCS_MAX_POINT_NUM accumulated records of ROISize, smoothing taps
 * from ROISize / LocType / MultiEmitterFitEn (FilterInit). */
int qcs_extract_init(const qcs_loc_para *p, qcs_extract_data **out);
/* Same with explicit frames per batch and record capacity (<= 0: defaults). */
int qcs_extract_init_ex(const qcs_loc_para *p, int max_batched_num, int capacity, qcs_extract_data **out);
/* LDROIExtractData_TypeDef::Deinit (LDROIExtraction.cu:289). */
int qcs_extract_deinit(qcs_extract_data *c);
/*
 * LDROIExtractData_TypeDef::ExtractMolecules(unsigned short *pImgData,
 * int ImageSource, LocalizationPara&, int StartFrame_CurBatch,
 * int BatchedImageNum, cudaStream_t) (LDROIExtraction.cu:30-80).
 * img: batched_num stacked frames, host memory (QCS_IMAGE_SOURCE_CPU_PINNED /
 * _CPU_NORMAL) or device memory (QCS_IMAGE_SOURCE_GPU, read in place, must
 * stay valid until the stream reaches this work).  Asynchronous on `stream`
 * (NULL: the context's own stream); the reference synchronises twice per call.
 * Host frames are copied on the context's copy stream into one of two device
 * buffers used in turn, so one call's copy runs while the previous call's
 * kernels do (inside a stream capture the copy stays on `stream`); host
 * frames must stay unchanged until this call's work has run.
 */
int qcs_extract_molecules(qcs_extract_data *c, const uint16_t *img, int image_source, const qcs_loc_para *p,
                          int start_frame, int batched_num, void *stream);
/* GetAccumulatedROINum (LDROIExtraction.cu:181): waits for the last call. */
int qcs_extract_accumulated_roi_num(qcs_extract_data *c, int *n);
/* ResetROINum (LDROIExtraction.cu:187-194): count 0, frame range (-1, -1).
 * The device count is cleared in stream order on `stream` (NULL: the stream
 * of the last call), with no host synchronisation. */
int qcs_extract_reset_roi_num(qcs_extract_data *c, void *stream);
/* h_ImageROI and Get_h_WLEPara() (LDROIExtraction.h:43, .cu:196): host copies
 * of the accumulated records / WLE rows, brought up to date on each call
 * (waits for the last extraction); NULL on error. */
const uint16_t *qcs_extract_h_image_roi(qcs_extract_data *c);
const float *qcs_extract_h_wle_para(qcs_extract_data *c);
/* d_ImageROI-equivalent accumulation buffer and Get_d_WLEPara()
 * (LDROIExtraction.cu:201), device memory, to feed qcs_loc_localize_device
 * without a host round trip; qcs_extract_device_roi_num: device int holding
 * the accumulated count. */
const uint16_t *qcs_extract_d_image_roi(const qcs_extract_data *c);
const float *qcs_extract_d_wle_para(const qcs_extract_data *c);
const int *qcs_extract_device_roi_num(const qcs_extract_data *c);
/* FirstFrame / EndFrame (LDROIExtraction.h:46-47). */
int qcs_extract_frame_range(const qcs_extract_data *c, int *first_frame, int *end_frame);
/* Detections dropped for capacity since the last reset (no counterpart). */
int qcs_extract_dropped_num(qcs_extract_data *c, int *n);

/* ---- localization context: LDLocData_TypeDef --------------------------- */
/*
 * One context owns every buffer of the localization path for records of one
 * ROI size, like LDLocData_TypeDef::Init (bfgs_top.cu:234-293).  Capacity is
 * the largest record count one call accepts; the reference fixes it at
 * MaxPointNum = 102400 (bfgs_CommonPara.h:316) and silently truncates larger
 * calls (bfgs_top.cu:36), this ABI rejects them with QCS_ERR_CAPACITY.  Row
 * capacity is 2 x capacity (records + appended second emitters).
 */
typedef struct qcs_loc_data qcs_loc_data;

/* LDLocData_TypeDef::Init(LocalizationPara&) (bfgs_top.h:75, bfgs_top.cu:234). */
int qcs_loc_init(const qcs_loc_para *p, qcs_loc_data **out);
/* Same with an explicit record capacity (<= 0: QCS_MAX_POINT_NUM). */
int qcs_loc_init_capacity(const qcs_loc_para *p, int capacity, qcs_loc_data **out);
/* LDLocData_TypeDef::Deinit (bfgs_top.h:76, bfgs_top.cu:295). */
int qcs_loc_deinit(qcs_loc_data *c);
int qcs_loc_capacity(const qcs_loc_data *c);

/*
 * LDLocData_TypeDef::BFGS_MLELocalization(unsigned short *h_ImageROI,
 * float *h_WLEPara, LocalizationPara&, int FluoNum, cudaStream_t)
 * (bfgs_top.h:78, bfgs_top.cu:26-204).  Host records in; on return the rows
 * are in qcs_loc_h_loc_arry() (h_LocArry), their count in
 * qcs_loc_valid_num() (oValidFluoNum) and the fit ratios in
 * qcs_loc_fit_ratios() (FitRatio_*).  Synchronous, like the reference.
 * h_wle may be NULL: the WLE pre-pass then runs on the device from the
 * records (the reference computes it during ROI extraction).  stream: a
 * cudaStream_t or NULL for the context's own stream.
 */
int qcs_loc_bfgs_mle_localization(qcs_loc_data *c, const uint16_t *h_rois, const float *h_wle,
                                  const qcs_loc_para *p, int n, void *stream);
/* After qcs_loc_localize_device / _device_n: wait for `stream` (NULL: the
 * context's stream) and bring the rows, their count and the fit ratios to
 * the host, as qcs_loc_bfgs_mle_localization leaves them. */
int qcs_loc_read_rows(qcs_loc_data *c, const qcs_loc_para *p, void *stream);
/* Asynchronous form of qcs_loc_bfgs_mle_localization (bfgs_top.cu:26): enqueues
 * the copy of n host records (and WLE rows, or NULL) to the device, the
 * localization, and the copy of the counters and of every row slot the call
 * can fill (n, or 3n with multi-emitter fitting) into the context's host
 * buffers on `stream` (NULL: the context's stream), and returns without
 * waiting.  With records in pinned memory the copies overlap kernels of other
 * streams: two contexts used in turn keep the copy engines and the SMs busy
 * at once.  qcs_loc_finish waits for the call and sets h_LocArry,
 * oValidFluoNum and the fit ratios; until then the context refuses other
 * calls and the host buffers must not be read. */
int qcs_loc_localize_async(qcs_loc_data *c, const uint16_t *h_rois, const float *h_wle, const qcs_loc_para *p, int n,
                           void *stream);
/* Waits for the context's pending asynchronous call (qcs_loc_localize_async,
 * qcs_learned_localize_async) and publishes its rows, count and ratios. */
int qcs_loc_finish(qcs_loc_data *c, const qcs_loc_para *p);
/* h_LocArry: valid until the next call on the context (bfgs_top.h:38). */
const float *qcs_loc_h_loc_arry(const qcs_loc_data *c);
/* oValidFluoNum (bfgs_top.h:42). */
int qcs_loc_valid_num(const qcs_loc_data *c);
/* [FitRatio_1E, FitRatio_2E, FitRatio_3E, FitRatio_Final_1E, FitRatio_Final_2E,
 *  FitRatio_Final_3E, FitRatio_Final_4E] (bfgs_top.h:46-58). */
int qcs_loc_fit_ratios(const qcs_loc_data *c, float *out7);

/*
 * Device-resident form of the same call: records (and optionally WLE rows)
 * already in device memory, rows left in device memory
 * (qcs_loc_device_rows, count at qcs_loc_device_valid_num), asynchronous on
 * `stream` with no host synchronisation, so whole pipelines can be captured
 * in a CUDA graph.  No counterpart in the reference (it always copies
 * through pinned host memory, bfgs_top.cu:42-47, 201-202).
 */
int qcs_loc_localize_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle,
                            const qcs_loc_para *p, int n, void *stream);
/* Several device-resident calls of different ROI sizes at once (a stream
 * of 7x7, 9x9 and 11x11 records): entry i is qcs_loc_localize_device(ctx[i],
 * d_rois[i], d_wle[i], &p[i], n[i], stream) with the same rows, counters and
 * 2E / 3E stages in ctx[i], but the single-emitter fits of all entries run in
 * one persistent launch whose blocks take tiles of any size from one work
 * list (the larger ROIs first).  count 1..QCS_MIXED_MAX, distinct contexts;
 * LocType GS2D, AS3D or DH3D with ROISize 7, 9 or 11 (else QCS_ERR_ROISIZE);
 * records on a 4-byte boundary and no likelihood-ratio selection on any
 * context (else QCS_ERR_ARG).  d_wle[i] may be NULL (the WLE pre-pass runs
 * into ctx[i]); the stream NULL means ctx[0]'s.  No counterpart in the
 * reference, which launches one kernel per ROI size and fit stage
 * (bfgsMLE_Single_Emitter_Fit.cu:40-67). */
#define QCS_MIXED_MAX 6
int qcs_loc_localize_mixed_device(qcs_loc_data *const *ctx, const uint16_t *const *d_rois,
                                  const float *const *d_wle, const qcs_loc_para *p, const int *n, int count,
                                  void *stream);
/* The same with the record count read on the device: *d_n (clamped to
 * [0, max_n], max_n <= capacity), e.g. qcs_extract_device_roi_num, so that
 * frames -> extraction -> localization runs with no host round trip.  d_wle is
 * required (the extraction writes it).  No counterpart in the reference. */
int qcs_loc_localize_device_n(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p,
                              const int *d_n, int max_n, void *stream);
const float *qcs_loc_device_rows(const qcs_loc_data *c);
const int *qcs_loc_device_valid_num(const qcs_loc_data *c);
/* The context's own device record / WLE buffers (capacity records). */
uint16_t *qcs_loc_device_roi_buffer(qcs_loc_data *c);
float *qcs_loc_device_wle_buffer(qcs_loc_data *c);

/* ---- zero-row removal: ZeroLocalizationsRemovel_TypeDef ------------------ */
/*
 * Drops rejected rows (peak photons <= 1) and optionally orders the rest by
 * frame (bfgsMLE_Loc_top/ZeroLocalizationsRemove.cu:21-186).  The reference
 * launches one kernel per frame and appends through an atomic counter; here
 * one stable sort orders rows by frame, row order within a frame.
 */
typedef struct qcs_zero_data qcs_zero_data;
/* ZeroLocalizationsRemovel_TypeDef::Init (:104-122); capacity in rows (<= 0: 2 x QCS_MAX_POINT_NUM). */
int qcs_zero_init(int capacity, qcs_zero_data **out);
int qcs_zero_deinit(qcs_zero_data *c);
/* RemoveZeroLocalizations(ih_LocArry, iFluoNum, SortFrameEn, FirstFrame, EndFrame, cstream) (:21-39):
 * host rows in; kept rows in qcs_zero_h_loc_arry (h_LocArry), count in qcs_zero_valid_num (ValidFluoNum). */
int qcs_zero_remove(qcs_zero_data *c, const float *h_rows, int n, int sort_frame_en, int first_frame, int end_frame,
                    void *stream);
const float *qcs_zero_h_loc_arry(const qcs_zero_data *c);
int qcs_zero_valid_num(const qcs_zero_data *c);
/* Device form, asynchronous: d_rows (n rows, or *d_n of them when d_n is set,
 * e.g. qcs_loc_device_valid_num) -> d_out, kept count -> *d_nvalid (may be
 * NULL).  Both row arrays 16-byte aligned.  No counterpart in the reference. */
int qcs_zero_remove_device(qcs_zero_data *c, const float *d_rows, int n, const int *d_n, int sort_frame_en,
                           int first_frame, int end_frame, float *d_out, int *d_nvalid, void *stream);

/* ---- consecutive-frame merging: ConsecutiveFit_TypeDef -------------------- */
#define QCS_ONTIME_BINS 10 /* MaxOnTimeConsecutiveNum (StatisticsInfo/statisticsInfo.h:53) */
typedef struct qcs_consec qcs_consec;
/* ConsecutiveFit_TypeDef::Init (ConsecutiveFit/ConsecutiveFit_top.cu:101-131):
 * groups of at most `capacity` rows (<= 0: 2 x QCS_MAX_POINT_NUM). */
int qcs_consec_init(int capacity, qcs_consec **out);
int qcs_consec_deinit(qcs_consec *c);
/* ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg (ConsecutiveFit_top.cu:22-98):
 * merges the n frame-sorted host rows of this group (RemoveZeroLocalizations
 * with frame sorting leaves them so) with the previous call's group: rows in
 * consecutive frames whose integer positions are closer than
 * ConsecFit_DistanceTh_nm / PixelSize pixels form chains; each chain's first
 * row takes the summed photons and background and the averages of x, y, z and
 * the widths weighted by 10 / CRLB_x, the other rows are zeroed; CRLB
 * recomputed for the rows that leave.  Output (qcs_consec_h_out_loc_arry,
 * qcs_consec_out_num rows): the previous group, or with is_end everything.
 * QCS_ERR_CAPACITY above the capacity.  Synchronous, like the reference. */
int qcs_consec_fit(qcs_consec *c, const float *h_rows, int n, int is_end, const qcs_loc_para *p, void *stream);
/* The same with the group's rows in device memory; the output rows stay on
 * the device (qcs_consec_d_out_loc_arry). */
int qcs_consec_fit_device(qcs_consec *c, const float *d_rows, int n, int is_end, const qcs_loc_para *p,
                          void *stream);
int qcs_consec_out_num(const qcs_consec *c);                 /* OutFluoNum */
const float *qcs_consec_h_out_loc_arry(const qcs_consec *c); /* h_OutLocArry (pinned, valid until the next call) */
const float *qcs_consec_d_out_loc_arry(const qcs_consec *c);
/* Copies the last call's qcs_consec_out_num output rows from the device into h_out. */
int qcs_consec_read_rows(qcs_consec *c, float *h_out);
/* h_OntimeRatio of the last call: chains starting in the new group by length
 * 1..10 frames (the last bin: 10 or more), over their number. */
int qcs_consec_ontime_ratio(const qcs_consec *c, float *out10);

/* ---- localization statistics: FluoStatisticData_TypeDef ------------------ */
#define QCS_STAT_HIST_LEN 1600 /* StatInf_Hist_DatLenMax (StatisticsInfo/statisticsInfo.h:37) */
/* qcs_stat_means: MeanTotalPhoton, MeanLocPrecisionXY, MeanPeakSNR, MeanBackground,
 * MeanPSFWidth, MeanPSFWidth_Ctl, MeanLocDensity2D, TimeVaryMean_TotalPhoton,
 * TimeVaryMean_LocPrecisionXY, TimeVaryMean_PeakSNR (statisticsInfo.h:63-86) */
#define QCS_STAT_MEANS 10
#define QCS_STAT_MEAN_PHOTON 0
#define QCS_STAT_MEAN_PREC 1
#define QCS_STAT_MEAN_SNR 2
#define QCS_STAT_MEAN_BKG 3
#define QCS_STAT_MEAN_PSF 4
#define QCS_STAT_MEAN_PSF_CTL 5
#define QCS_STAT_MEAN_DENSITY 6
#define QCS_STAT_TV_PHOTON 7
#define QCS_STAT_TV_PREC 8
#define QCS_STAT_TV_SNR 9
/* qcs_stat_series: TimeVary_TotalPhoton, _LocPrecisionXY, _PeakSNR, _Background,
 * _PSFWidth, _PSFWidth_Ctl, _LocDensity2D (statisticsInfo.h:89-96), then
 * TimeVary_OntimeF1Ratio .. F4Ratio (statisticsInfo.h:116-119) */
#define QCS_STAT_SERIES 11
#define QCS_STAT_SERIES_PHOTON 0
#define QCS_STAT_SERIES_PREC 1
#define QCS_STAT_SERIES_SNR 2
#define QCS_STAT_SERIES_BKG 3
#define QCS_STAT_SERIES_PSF 4
#define QCS_STAT_SERIES_PSF_CTL 5
#define QCS_STAT_SERIES_DENSITY 6
#define QCS_STAT_SERIES_ONTIME_F1 7 /* ratios of on times of 1, 2, 3 and >= 4 frames */
#define QCS_STAT_SERIES_ONTIME_F2 8
#define QCS_STAT_SERIES_ONTIME_F3 9
#define QCS_STAT_SERIES_ONTIME_F4 10
typedef struct qcs_stat qcs_stat;
/* FluoStatisticData_TypeDef::Init (statisticsInfo_top.cu:258): calls of at
 * most `capacity` rows (<= 0: 2 x QCS_MAX_POINT_NUM); starts reset. */
int qcs_stat_init(int capacity, qcs_stat **out);
int qcs_stat_deinit(qcs_stat *st);
/* ResetAllDat (statisticsInfo_top.cu:391): histograms, means and time series
 * cleared (the mean on time is kept, as the reference keeps MeanOntime). */
int qcs_stat_reset_all(qcs_stat *st);
/* GetStatisticalInf (statisticsInfo_top.cu:61) over n host rows: the four
 * histograms (qcs_stat_histograms), the means and the activation density
 * (qcs_stat_means), one more entry in each time series (qcs_stat_series).
 * Synchronous, like the reference; n <= 0 changes nothing. */
int qcs_stat_get_statistical_inf(qcs_stat *st, const float *h_rows, int n, const qcs_loc_para *p, void *stream);
/* The same over n rows in device memory. */
int qcs_stat_get_statistical_inf_device(qcs_stat *st, const float *d_rows, int n, const qcs_loc_para *p,
                                        void *stream);
/* The last call's histograms: total photons (bins of 25 photons), precision
 * (0.15 nm), peak SNR (0.125), PSF width (0.0125 px), QCS_STAT_HIST_LEN each, in that order. */
int qcs_stat_histograms(const qcs_stat *st, int *out4x1600);
int qcs_stat_means(const qcs_stat *st, float *out10);
/* Copies up to max_n entries of time series `which` into out (may be NULL); returns its length. */
int qcs_stat_series(const qcs_stat *st, int which, float *out, int max_n);
/* UpdateOntimeRatio (statisticsInfo_top.cu:23-57): takes the QCS_ONTIME_BINS
 * on-time ratios of a consecutive-frame merge (qcs_consec_ontime_ratio), fits
 * y = a * exp(b * i) to them by the reference's 2-parameter BFGS curve fit (BFGS
 * for curve fitting/BFGSOptimizer.h, CurveFitting.cpp:27-58: 4 iterations, 11
 * bisections), sets the mean on time 2 / (-log(1 - a) - b) frames, sums the
 * ratios of 4 frames and more into entry 3, clamps entries 0..3 to [0, 1] and
 * appends them to the series QCS_STAT_SERIES_ONTIME_F1..F4.  Host arithmetic,
 * as in the reference: results equal its host build bit for bit. */
int qcs_stat_update_ontime_ratio(qcs_stat *st, const float *ratios10);
/* The mean on time (frames; 0 before the first update) and the QCS_ONTIME_BINS
 * ratios of the last update as shown (entries 0..3 folded and clamped). */
int qcs_stat_ontime(const qcs_stat *st, float *mean_ontime, float *ratios10);

/* ---- WLE pre-pass: WLEParameterEstimation_TypeDef ---------------------- */
/* WLEParameterEstimation_TypeDef::WLEParameterEstimate (WLEParaEstimation.h:41,
 * WLEParaEstimation.cpp:20-40): PSF width, same-frame nearest neighbour and
 * molecule type of n records; host in, host out. */
int qcs_wle_estimate(qcs_loc_data *c, const uint16_t *h_rois, int n, const qcs_loc_para *p, float *h_wle);
/* Same on device pointers, asynchronous on `stream`. */
int qcs_wle_estimate_device(qcs_loc_data *c, const uint16_t *d_rois, int n, const qcs_loc_para *p, float *d_wle,
                            void *stream);

/* ---- kernel-level entry points ----------------------------------------- */
/* One single-emitter fit pass over n device records, identity queue, no
 * cascade and no CRLB: LDLoc_BFGS_MLELocalizationGS2D / ...AS3D
 * (bfgsMLE_Single_Emitter_Fit.h:10-13, .cu:31-119), dispatching the true ROI
 * size (the reference launches the 8x8 kernel for ROISize 9 in AS3D, .cu:96).
 * loc_type: QCS_LOCTYPE_*; rows: n x 12 in d_loc, CRLB columns left 0. */
int qcs_fit_single_device(int loc_type, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n,
                          float *d_loc, void *stream);
/* The fit of qcs_fit_single_device with `lanes` lanes per ROI (8; also 4 or
 * 16 for GS2D 7x7): the same rows bit for bit, with about half the latency
 * per ROI, for short batches.  ROI sizes: GS2D 7, 9, 11, 13 and AS3D 7, 9, 11
 * (the sizes whose pixel-distance rounding is fixed in the source);
 * QCS_ERR_ARG otherwise. */
int qcs_fit_single_group_device(int loc_type, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle,
                                int n, float *d_loc, int lanes, void *stream);
/* Autotuner (no counterpart in the reference): times the single-emitter fit of
 * the first m records of d_rois / d_wle (device, WLE rows given) for m = 256,
 * 1,024, 4,096, ... up to n with one thread per ROI and with 8 lanes per ROI
 * (also 4 and 16 for GS2D 7x7), and keeps in the context, per batch size,
 * the fastest; qcs_loc_localize_device then fits a batch of n records with
 * the lanes of the first entry whose size is >= n (larger batches: one
 * thread per ROI).  Every choice gives the same rows bit for bit.  n >= 64
 * records; overwrites the context's rows. */
int qcs_loc_autotune(qcs_loc_data *c, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n,
                     void *stream);
/* The tuning table (returns its length; sizes / lanes may be NULL), or sets it
 * (count 0..8 entries of (largest batch, lanes 1 / 4 / 8 / 16); 0 clears it). */
int qcs_loc_tuning(const qcs_loc_data *c, int *sizes, int *lanes, int max_entries);
int qcs_loc_set_tuning(qcs_loc_data *c, const int *sizes, const int *lanes, int count);
/* With multi-emitter fitting, qcs_loc_autotune also times each multi-emitter
 * stage (2E or AS3D-2E, and 3E) on queues of the caller's first 64, 128,
 * 256, ... records with the lane-group kernel and with one thread per ROI,
 * and keeps the longest queue for which the lane groups are faster: a stage
 * whose queue (read on the device) is at most that long uses them.  The
 * limits (-1: one thread per ROI always; 0: the built-in default, about three
 * waves of the lane-group kernel), read or set here.  The rows are the same
 * either way. */
int qcs_loc_tuning_multi(const qcs_loc_data *c, int *limit_2e, int *limit_3e);
int qcs_loc_set_tuning_multi(qcs_loc_data *c, int limit_2e, int limit_3e);
/* Per-GPU tuning cache: writes the context's tuning (lanes table and
 * multi-emitter limits) to a text file tagged with the GPU's name, ROI size,
 * localization type and multi-emitter setting; loading sets the context's
 * tuning from such a file and refuses (QCS_ERR_STATE) one written for another
 * GPU model or shape, so a caller tunes once per machine and reloads. */
int qcs_loc_save_tuning(const qcs_loc_data *c, const char *path);
int qcs_loc_load_tuning(qcs_loc_data *c, const char *path);
/* Model selection of multi-emitter calls (no counterpart in the reference,
 * whose selection is its SNR / validity cascade, bfgsMLE_GS2D_core.h:279-298,
 * bfgsMLE_GS2D_2Emitter_core.h:296-348; QCS_SELECT_CASCADE, the default and
 * the parity mode).  QCS_SELECT_LR, for GS2D and DH3D calls with
 * MultiEmitterFitEn: every record is fitted with one, two and three emitters
 * (the reference's fits, schedules and accept rules), each fitted model's
 * unweighted Poisson log-likelihood sum(n ln mu - mu) is accumulated in FP64,
 * and a record keeps the smallest accepted model unless a larger accepted one
 * raises 2 ln L by more than `threshold` per added emitter (three parameters
 * per emitter; 0 picks QCS_SELECT_LR_DEFAULT_TH).  The rows are the chosen
 * model's, at most two emitters per record as the reference writes them, in
 * the cascade's layout (records, then appended second emitters) with CRLB.
 * Fit ratios: 1, 2, 3 = all records; 4, 5, 6 = fractions keeping one, two,
 * three emitters; 7 = no model accepted.  About three times the fitting work
 * of the cascade.  Allocates the mode's scratch (capacity x 108 bytes) once. */
#define QCS_SELECT_CASCADE 0
#define QCS_SELECT_LR 1
#define QCS_SELECT_LR_DEFAULT_TH 10.0f
int qcs_loc_set_model_selection(qcs_loc_data *c, int mode, float threshold);
int qcs_loc_model_selection(const qcs_loc_data *c, int *mode, float *threshold);
/* LDLocData_TypeDef::LocPrecCalc_GaussianCRLB (bfgs_top.h:90,
 * LocPrecCalc_GaussianCRLB.cu:23-40): CRLB columns of n device rows. */
int qcs_crlb_device(const qcs_loc_para *p, float *d_loc, int n, void *stream);

/* ---- learned start points (no counterpart in the reference) ------------- */
/*
 * A small network (K features -> 128 -> 128 -> 8, ReLU, BF16 tensor-core
 * GEMMs with FP32 accumulation; K = 64 for 7x7 ROIs, 128 for 9x9 and 11x11)
 * predicts each ROI's start point for the BFGS fit (GS2D: x, y, sigma, peak
 * photons, background; AS3D: x, y, sigma_x, sigma_y, peak photons,
 * background) and, for GS2D, from three logits its emitter-count class (0:
 * one emitter; 1: the stage of the two-emitter fit; 2: the stage of the
 * three-emitter fit), trained on the GPU by these entry points on ROIs
 * labelled by converged plain fits and by the plain multi-emitter cascade's
 * outcome.  One network per localization type and ROI size.
 * Parameters: W1 Kx128, b1, W2 128x128, b2, W3 128x8, b3, row-major [in][out]
 * (qcs_learned_shape gives the count).
 * Every `stream` argument of these entry points is a cudaStream_t, NULL for
 * the default stream; the calls are asynchronous on it unless they return a
 * host value (a loss).
 */
typedef struct qcs_learned_net qcs_learned_net;
/* Parameter count of the GS2D 7x7 network (K = 64). */
int qcs_learned_param_count(void);
/* A network for loc_type (QCS_LOCTYPE_GS2D or QCS_LOCTYPE_AS3D) and ROISize 7,
 * 9 or 11 (else QCS_ERR_ROISIZE); batch: training batch size and inference
 * chunk (<= 0: 4096); seed of the initial weights. */
/* Network kind for the start points of the GS2D two-emitter fit (the
 * multi-emitter cascade's 2E stage): 8 outputs, dx, dy of emitter 0 and of
 * emitter 1, log(peak / range) of each, sigma - 1.3, (background - min) / range. */
#define QCS_LEARNED_GS2D_2E 16
/* Network kind for the start points of the GS2D three-emitter fit (the
 * cascade's 3E stage): 16 outputs, of which 11 are used: dx, dy of emitters 0,
 * 1, 2, log(peak / range) of each, sigma - 1.3, (background - min) / range;
 * W3 128x16, b3 16.  MLP networks only. */
#define QCS_LEARNED_GS2D_3E 17
int qcs_learned_create_for(int loc_type, int roi_size, int batch, unsigned long long seed, qcs_learned_net **out);
/* Network architectures: the MLP above, and a convolutional network
 * (3x3 conv, 32 channels, zero 'same' padding, ReLU -> 3x3 conv, 64 channels,
 * ReLU -> fully connected 256 over the flattened 64 x R x R map (position
 * major, channel minor) and the two scale features, ReLU -> the same eight
 * outputs) on the first R*R features taken as the R x R image.  Same
 * features, targets, loss, training and start-point entry points; its
 * parameters, row-major [in][out]: W1 [9][32] (tap 3 (dy + 1) + (dx + 1)),
 * b1, W2 [9 * 32][64] (row tap * 32 + input channel), b2, W3 [R*R*64 + 2][256],
 * b3, W4 [256][8], b4.  Inference runs two tensor-core kernels per chunk of
 * 65,536 records (0.4-1 GB of device memory per conv network for the
 * flattened maps). */
#define QCS_LEARNED_ARCH_MLP 0
#define QCS_LEARNED_ARCH_CONV 1
int qcs_learned_create_arch(int arch, int loc_type, int roi_size, int batch, unsigned long long seed,
                            qcs_learned_net **out);
/* QCS_LEARNED_ARCH_MLP or QCS_LEARNED_ARCH_CONV (-1 for NULL). */
int qcs_learned_arch(const qcs_learned_net *net);
/* qcs_learned_create_for(QCS_LOCTYPE_GS2D, 7, batch, seed, out). */
int qcs_learned_create(int batch, unsigned long long seed, qcs_learned_net **out);
/* The network's localization type, ROI size and parameter count (any may be NULL). */
int qcs_learned_shape(const qcs_learned_net *net, int *loc_type, int *roi_size, int *params);
/* Frees the network.  A QCS_LEARNED_GS2D_2E network that is attached to a
 * GS2D network (qcs_learned_set_two_emitter) is refused with QCS_ERR_STATE
 * and left intact: detach it or destroy its owner first.  Destroying an owner
 * detaches its two-emitter network. */
int qcs_learned_destroy(qcs_learned_net *net);
int qcs_learned_get_params(qcs_learned_net *net, float *h_params);
int qcs_learned_set_params(qcs_learned_net *net, const float *h_params);
/* Features (n x K: 64 for 7x7, 128 for 9x9 and 11x11) and per-record (min,
 * range) of n device records of p->ROISize (GS2D or AS3D). */
int qcs_learned_features_device(const qcs_loc_para *p, const uint16_t *d_rois, int n, float *d_feat, float *d_scale,
                                void *stream);
/* Training targets (n x 5 for GS2D, n x 6 for AS3D) and validity (n) from
 * plain-fit rows of the same records. */
int qcs_learned_targets_device(const qcs_loc_para *p, const uint16_t *d_rois, const float *d_rows,
                               const float *d_scale, int n, float *d_targets, float *d_valid, void *stream);
/* Network outputs (n x 8; n x 16 for QCS_LEARNED_GS2D_3E networks) of n feature rows. */
int qcs_learned_forward_device(qcs_learned_net *net, const float *d_feat, int n, float *d_out, void *stream);
/* Loss and parameter gradient of one batch (n <= batch); gradients via qcs_learned_get_grads. */
int qcs_learned_gradient_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                const float *d_valid, int n, float *h_loss, void *stream);
/* The same with emitter-count labels d_classes (n floats: 0, 1, 2, or -1 for
 * none; NULL: none): the loss adds 0.5 x the softmax cross-entropy of the
 * count logits (outputs 5..7) per labelled row, over the batch. */
int qcs_learned_gradient_counts_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                       const float *d_valid, const float *d_classes, int n, float *h_loss,
                                       void *stream);
int qcs_learned_get_grads(qcs_learned_net *net, float *h_grads);
/* Adam training over n rows for `epochs` epochs; h_epoch_loss (epochs floats, may be NULL). */
int qcs_learned_train_device(qcs_learned_net *net, const float *d_feat, const float *d_targets, const float *d_valid,
                             int n, int epochs, float lr, unsigned long long seed, float *h_epoch_loss, void *stream);
/* The same with emitter-count labels (as qcs_learned_gradient_counts_device). */
int qcs_learned_train_counts_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                    const float *d_valid, const float *d_classes, int n, int epochs, float lr,
                                    unsigned long long seed, float *h_epoch_loss, void *stream);
/* Emitter-count labels of the n records of the last multi-emitter call on c
 * (d_labels: n floats): 0 where the plain cascade did not send the record to
 * the two-emitter fit, 1 where that fit kept it, 2 where it passed it on to
 * the three-emitter fit. */
int qcs_loc_count_labels_device(qcs_loc_data *c, int n, float *d_labels, void *stream);
/* Routing threshold th of the count classes: with multi-emitter fitting on,
 * qcs_learned_localize_device sends a record straight to the three-emitter
 * fit when p(class 2) >= th, else to the two-emitter fit when p(class 1) +
 * p(class 2) >= th (softmax probabilities); th = 0 (the default) routes by
 * the WLE classes alone, as the reference does.  QCS_ERR_ARG outside [0, 1]. */
int qcs_learned_set_count_threshold(qcs_learned_net *net, float th);
float qcs_learned_count_threshold(const qcs_learned_net *net);
/* Attaches a QCS_LEARNED_GS2D_2E network `two` of the same ROI size to the
 * GS2D network `net` (NULL detaches).  `net` keeps a pointer to `two`, so
 * `two` must stay alive while attached: qcs_learned_destroy(two) refuses
 * (QCS_ERR_STATE) until it is detached or `net` is destroyed.  Learned
 * localization calls with
 * multi-emitter fitting on then start the cascade's two-emitter fits from
 * its start points with `iters` BFGS iterations of `bisections` line-search
 * steps (3 or 4 of 6, or the reference's 13 of 11) and the analytic gradient.
 * A fit is poor when no emitter is kept or when the two-emitter model's
 * Poisson deviance exceeds dev_th (0: 2 ROISize^2 + 2); poor fits go on to the
 * three-emitter fit, as the reference's rejected two-emitter fits do
 * (fallback QCS_TWO_FALLBACK_3E), are fitted again by the reference's
 * two-emitter fit (QCS_TWO_FALLBACK_PLAIN: one more pass of that fit), or
 * keep their own result under the reference's accept rules
 * (QCS_TWO_FALLBACK_NONE: no refit; a plain refit pass, even of a few ROIs,
 * costs the plain two-emitter schedule's latency). */
/* Attaches a QCS_LEARNED_GS2D_3E network `three` of the same ROI size to the
 * GS2D network `net` (NULL detaches): learned multi-emitter calls with `net`
 * then start the three-emitter stage's fits from its start points, with
 * `iters` BFGS iterations of `bisections` line-search steps (4 or 6 of 6, or
 * 16 of 11; bisections <= 0: 6), and refit plainly every fit that keeps no
 * emitter or whose unweighted Poisson deviance exceeds dev_th (0: 2 R^2 + 2;
 * negative: no plain refits, the learned fits' results stand).  A plain refit
 * pass, even of a few ROIs, costs the plain three-emitter schedule's latency.
 * `three` stays owned by the caller and must outlive the attachment
 * (qcs_learned_destroy refuses it while attached).  The context allocates
 * 97 bytes per record of capacity for the three-emitter stage on the first
 * such call, which must not be inside a stream capture. */
int qcs_learned_set_three_emitter(qcs_learned_net *net, qcs_learned_net *three, int iters, int bisections,
                                  float dev_th);
/* Three-emitter fits of the last learned call redone by the plain three-emitter fit. */
int qcs_learned_refit_3e_num(qcs_loc_data *ctx, int *n);
/* Training data of a QCS_LEARNED_GS2D_3E network.  With capture on, each
 * plain multi-emitter call of the context also keeps the final fitted
 * parameters of its three-emitter fits (11 floats per 3E-queue slot, fit
 * units; qcs_loc_device_three_emitter_params); the rows are unchanged.  Turning
 * it on allocates the context's three-emitter buffers (97 bytes per record of
 * capacity). */
int qcs_loc_set_three_emitter_capture(qcs_loc_data *ctx, int on);
const float *qcs_loc_device_three_emitter_params(const qcs_loc_data *ctx);
/* Targets (n x 11: dx, dy of emitters 0..2, log(peak / range) of each,
 * sigma - 1.3, (background - min) / range; emitters ordered by peak x (R -
 * distance from the ROI centre)) and validity (n) of the records whose plain
 * three-emitter fit in the last capturing call kept an emitter; d_scale from
 * qcs_learned_features_device. */
int qcs_loc_three_emitter_targets_device(qcs_loc_data *ctx, const uint16_t *d_rois, const qcs_loc_para *p, int n,
                                         const float *d_scale, float *d_targets, float *d_valid, void *stream);
/* Learned calls without multi-emitter fitting refit plainly every learned fit
 * that is not accepted or whose deviance exceeds dev_th (on, the default).
 * With on = 0 the learned fits' results stand: no refit pass and rejected
 * fits stay rejected (the plain fit might have accepted some of them).
 * Multi-emitter calls always route the poor single fits by a plain refit or,
 * with qcs_learned_set_direct_two_emitter, to the two-emitter fit. */
int qcs_learned_set_single_refits(qcs_learned_net *net, int on);
/* Multi-emitter learned calls: a learned single-emitter fit that is rejected
 * or judged poor by the deviance bound and has SNR > 6 goes straight to the
 * two-emitter fit (the reference's rule for its rejected single fits, applied
 * to the learned fit) instead of being refitted plainly first (on != 0; GS2D
 * networks; default off).  More localizations and lower RMSE on records with
 * several emitters, at the cost of a longer two-emitter queue.  No
 * counterpart in the reference. */
int qcs_learned_set_direct_two_emitter(qcs_learned_net *net, int on);
/* Iteration cap of the learned-start fits (no counterpart in the reference):
 * runs qcs_learned_localize_device on the caller's n device records with
 * every schedule compiled for the network's shape (BFGS iterations x
 * line-search steps) and returns the fastest whose fraction of accepted
 * records is within 0.5 points of the best schedule's (ground truth is not
 * needed: a schedule too short for the data shows as rejected and refitted
 * records).  Overwrites the context's rows; n >= 64. */
int qcs_learned_autotune(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                         const qcs_loc_para *p, int n, int *iters, int *bisections, void *stream);
#define QCS_TWO_FALLBACK_3E 0
#define QCS_TWO_FALLBACK_PLAIN 1
#define QCS_TWO_FALLBACK_NONE 2
int qcs_learned_set_two_emitter(qcs_learned_net *net, qcs_learned_net *two, int iters, int bisections,
                                float dev_th, int fallback);
/* Two-emitter fits that the last learned call on c redid with the reference's
 * two-emitter fit (synchronises the device). */
int qcs_learned_refit_2e_num(qcs_loc_data *c, int *n);
/* Training targets of a QCS_LEARNED_GS2D_2E network from the plain
 * multi-emitter call just made on c over the same n records (GS2D, ROI size 7,
 * 9 or 11): for each record whose two-emitter fit kept both emitters, 8 floats
 * (dx, dy of the first emitter row and of the second, log(peak e- / range) of
 * each, sigma - 1.3, (background e- - min) / range; ranges d_scale from
 * qcs_learned_features_device) and valid = 1; zeros elsewhere. */
int qcs_loc_two_emitter_targets_device(qcs_loc_data *c, const uint16_t *d_rois, const qcs_loc_para *p, int n,
                                       const float *d_scale, float *d_targets, float *d_valid, void *stream);
/* Start points (as qcs_learned_start_device) and emitter-count classes
 * (uint8 per record, at the routing threshold, or 0.5 when routing is off)
 * of n device records. */
int qcs_learned_classes_device(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                               float *d_start, uint8_t *d_classes, void *stream);
/* Start points of n device records (GS2D n x 5: peak e-, x, y, sigma,
 * background e-; AS3D n x 6: peak e-, x, y, sigma_x, sigma_y, background
 * e-; QCS_LEARNED_GS2D_2E n x 8: peak e-, x, y of emitter 0, the same of
 * emitter 1, sigma, background e-); d_work holds qcs_learned_work_bytes(n)
 * bytes (unused by the fused path). */
int qcs_learned_start_device(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                             float *d_start, float *d_work, void *stream);
size_t qcs_learned_work_bytes(int n);
/* Single-emitter fits (GS2D or AS3D, ROISize 7, 9 or 11) from given start
 * points d_start (GS2D n x 5: peak e-, x, y in ROI pixels, sigma, background
 * e-; AS3D n x 6: peak e-, x, y, sigma_x, sigma_y, background e-) with the
 * plain fit's weighted loss and accept rules, `iters` BFGS iterations of
 * `bisections` line-search steps each (<= 0: the reference's 11; schedules:
 * 2..4 iterations of 6 steps or 3 of 11; GS2D 7x7 also 2..5 or 8 of 11 and 2
 * or 3 of 4 or 8) and the loss's analytic gradient; fits that are not
 * accepted or whose Poisson deviance exceeds dev_th (<= 0: 2 R^2 + 2, 100 for 7x7) are refitted
 * by the plain kernel; then CRLB.  Rows in the context (n).  With
 * p->MultiEmitterFitEn the single-emitter fit is the first stage of the
 * reference's cascade (bfgs_top.cu:26-204): it runs over the single-emitter
 * queue, a plain refit decides which rejects go on to the two-emitter fit,
 * and the 2E / 3E stages, appended rows and CRLB follow as in
 * qcs_loc_localize_device. */
int qcs_fit_from_start_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p,
                              int n, const float *d_start, int iters, int bisections, float dev_th, void *stream);
/* The same with emitter-count classes d_classes (uint8 per record, or NULL;
 * multi-emitter fitting only): class 1 joins the two-emitter queue and class
 * 2 the three-emitter queue without the stages before. */
int qcs_fit_from_start_classes_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle,
                                      const qcs_loc_para *p, int n, const float *d_start, const uint8_t *d_classes,
                                      int iters, int bisections, float dev_th, void *stream);
/* Localization from learned start points with the schedule of
 * qcs_fit_from_start_device (the network's shape must be the call's:
 * QCS_ERR_ROISIZE otherwise), and, with multi-emitter fitting on (GS2D) and a
 * count threshold set, the network's emitter-count classes.  Rows in the
 * context like qcs_loc_localize_device.  One network may serve several
 * contexts on different streams at once: the inference buffers a network
 * owns (conv networks, and the MLP with fused inference off) pass from call
 * to call in stream order.  A CUDA graph holding such a call must not run
 * beside another call of the same network. */
int qcs_learned_localize_device(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                                const qcs_loc_para *p, int n, int iters, int bisections, float dev_th,
                                void *stream);
/* qcs_learned_localize_device with the record count in device memory (*d_n,
 * at most max_n; e.g. qcs_extract_device_roi_num after extraction), like
 * qcs_loc_localize_device_n; GS2D with multi-emitter fitting on, d_wle
 * required.  The fused inference reads the count on the device; the
 * layer-by-layer inference computes all max_n records. */
int qcs_learned_localize_device_n(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                                  const qcs_loc_para *p, const int *d_n, int max_n, int iters, int bisections,
                                  float dev_th, void *stream);
/* Inference path of qcs_learned_localize_device: fused = 1 (default) runs the
 * whole network per 128-ROI tile in one tcgen05 kernel; 0 runs it layer by
 * layer through the training GEMMs. */
int qcs_learned_set_inference(qcs_learned_net *net, int fused);
/* QCS_OK, or QCS_ERR_CUDA if a fused-inference launch gave up waiting for its
 * tensor-core work (waits for the device). */
int qcs_learned_fused_status(qcs_learned_net *net);
/* qcs_learned_localize_device on host records, asynchronously like
 * qcs_loc_localize_async (finish with qcs_loc_finish).  One network may serve
 * several contexts at once: its start points go to each context's own
 * buffer, and its weight image is rebuilt only after a parameter change
 * (change parameters only while no call using the network is in flight). */
int qcs_learned_localize_async(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *h_rois, const float *h_wle,
                               const qcs_loc_para *p, int n, int iters, int bisections, float dev_th,
                               void *stream);
/* Number of plain single-emitter refits of the last qcs_learned_localize_device call (waits for it). */
int qcs_learned_refit_num(qcs_loc_data *c, int *n);

/* ---- super-resolution render (ImageRenderData_TypeDef) ------------------ */
typedef struct qcs_render_data qcs_render_data;
/* ImageRenderData_TypeDef::Init (ImgRender/ImageRender_top.cu:223): a float SR
 * image of p->SRImageWidth x p->SRImageHigh, zeroed; for 3D localization types
 * (LocType != GS2D) also the z-weighted colour map; the display maximum and
 * QCS_RENDER_HIST_LEN-bin histogram; room for `capacity` host rows per call
 * (<= 0: QCS_MAX_POINT_NUM). */
int qcs_render_init(const qcs_loc_para *p, int capacity, qcs_render_data **out);
int qcs_render_deinit(qcs_render_data *r);
/* ResetFillImgTop (ImageRender_top.cu:168-183): the images back to zero. */
int qcs_render_reset(qcs_render_data *r, void *stream);
/* ResetFillMaxVal(0) (ImageRender_top.cu:68-79): display maximum, histogram
 * and the row count behind the periodic histogram rescale back to zero. */
int qcs_render_reset_max(qcs_render_data *r, void *stream);
/* FluoRenderTop(h_LocArry, LocPara, RenderingMode, FixedlocPrec, FluoNum,
 * stream) (ImageRender_top.cu:29): adds n host rows (12 floats each) to the
 * image with mode QCS_RENDER_*; fixed_prec (nm) for QCS_RENDER_1PHOTON_FIXED.
 * Rows are selected and widened as in FluoRenderWithPrec_2D / _3D
 * (ImageRender_2d.cu:55-155, ImageRender_3d.cu:60-148); the histogram step is
 * skipped while the running maximum is 0 (the reference divides by it). */
int qcs_render_rows(qcs_render_data *r, const float *h_rows, const qcs_loc_para *p, int mode, float fixed_prec, int n,
                    void *stream);
/* The same for rows already on the device, the count read at d_n (NULL: max_n)
 * when the kernels run: the hand-off from a localization call, e.g.
 * qcs_loc_device_rows(ctx) with qcs_loc_device_valid_num(ctx), no host round
 * trip (no counterpart in the reference, which copies rows from the host). */
int qcs_render_rows_device(qcs_render_data *r, const float *d_rows, const int *d_n, int max_n, const qcs_loc_para *p,
                           int mode, float fixed_prec, void *stream);
/* d_SRIntensityImg, d_SRColorMapImg (NULL for 2D) (ImageRender_top.h). */
float *qcs_render_d_image(qcs_render_data *r);
float *qcs_render_d_colormap(qcs_render_data *r);
/* Copies the image, colour map, maximum and histogram (any may be NULL) to the
 * host and waits. */
int qcs_render_read(qcs_render_data *r, float *h_img, float *h_colormap, int *h_max, int *h_hist, void *stream);

/* ---- localization file (12 float32 per row) ------------------------------ */
/* The worker's LocFile.Write(WriteLocArry, WriteLocNum * OutParaNumGS2D *
 * sizeof(float)) (Plugin for ImageJ/QC-STORM_ CPPDLL/QC-STORM_ CPPDLL/
 * OnlineLocalizationLD.cpp:284): rows appended as 12 native float32 each, no
 * header, the file utility/Output file load and postprocessing/
 * py_LoadBinaryLocData.py reads with np.fromfile(...).reshape(-1, 12). */
typedef struct qcs_locfile qcs_locfile;
/* append = 0 truncates; capacity: most rows per qcs_locfile_write_device call
 * (<= 0: 2 x QCS_MAX_POINT_NUM), for its two pinned staging buffers. */
int qcs_locfile_open(const char *path, int append, int capacity, qcs_locfile **out);
/* Appends n host rows (after any device rows queued before). */
int qcs_locfile_write(qcs_locfile *f, const float *h_rows, int n);
/* Appends rows on the device, their count read at d_n (NULL: max_n) -- e.g.
 * the output of qcs_zero_remove_device -- without waiting: the copy and the
 * append run in order on `stream` (a host function appends after the copy).
 * Reuses a staging buffer only after its previous append; rows[0, max_n) must
 * stay valid until the copy has run.  Appends happen in the order of their
 * stream: give every call on one file the same stream. */
int qcs_locfile_write_device(qcs_locfile *f, const float *d_rows, const int *d_n, int max_n, void *stream);
/* Waits for queued appends and flushes the file. */
int qcs_locfile_flush(qcs_locfile *f);
/* Rows in the file (after qcs_locfile_flush for device rows). */
long long qcs_locfile_rows(const qcs_locfile *f);
/* Waits for queued appends and closes; reports a failed write. */
int qcs_locfile_close(qcs_locfile *f);

/* ---- FP64 Fisher-matrix CRLB side output --------------------------------- */
/*
 * No counterpart in the reference, whose CRLB columns (9, 10) hold a diagonal
 * x / y estimate (LocPrecCalc_GaussianCRLB.h:65-243: Fisher information of
 * x alone from numerical second derivatives on a fixed grid, emitter at its
 * centre); those columns are left as they are.  This bound uses the full
 * Fisher information of the fitted single-emitter model on the ROI's R x R
 * pixel centres: mu = N / (2 pi sx sy) exp(-dx^2/(2 sx^2) - dy^2/(2 sy^2)) + B
 * in photoelectrons, parameters x, y, N, B and sigma (GS2D, DH3D) or sigma_x,
 * sigma_y (AS3D), Poisson noise with read noise as extra variance
 * (I_ij = sum dmu_i dmu_j / (mu + ReadNoise_e^2)), built and inverted
 * (Cholesky) in FP64 on the GPU.  For n device rows (12 floats, as the
 * localization writes them; rows with column 0 <= 0 are skipped) writes
 * n x QCS_FISHER_COLS floats to d_out: the square roots of the inverse's
 * diagonal (x, y in nm; photons and background in photons, i.e. divided by
 * QE; widths in pixels; z in nm through the calibration polynomial's
 * Jacobian, AS3D only) and a status.  d_rois (may be NULL): the first n_rois
 * rows are the single-emitter rows of those records (row i from record i),
 * which places the emitter at its fitted position in its ROI; other rows put
 * it at the ROI centre, as the reference's estimate does.  Asynchronous on
 * `stream`; allocates nothing.
 */
#define QCS_FISHER_COLS 8
#define QCS_FISHER_X 0          /* nm */
#define QCS_FISHER_Y 1          /* nm */
#define QCS_FISHER_Z 2          /* nm, AS3D (0 otherwise) */
#define QCS_FISHER_PHOTONS 3    /* total photons */
#define QCS_FISHER_BACKGROUND 4 /* photons per pixel */
#define QCS_FISHER_SIGMA_X 5    /* pixels */
#define QCS_FISHER_SIGMA_Y 6    /* pixels */
#define QCS_FISHER_STATUS 7     /* QCS_FISHER_OK / _INVALID / _SINGULAR */
#define QCS_FISHER_OK 0
#define QCS_FISHER_INVALID 1    /* rejected row, or photons / widths out of range */
#define QCS_FISHER_SINGULAR 2   /* Fisher matrix not positive definite */
int qcs_crlb_fisher_fp64(const qcs_loc_para *p, const float *d_rows, int n, const uint16_t *d_rois, int n_rois,
                         float *d_out, void *stream);

/* ---- allocation-free localization --------------------------------------- */
/*
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory: code recording the localization into a CUDA graph while its stream
 * is captured (cudaMalloc is not allowed during capture), hosts that own all
 * device memory through their own pool, and camera-rate loops that cannot
 * take the device-wide synchronisation of cudaMalloc/cudaFree mid-stream.
 * Same result as qcs_loc_localize_device (classify, single-emitter fit,
 * 2E/3E cascade, CRLB) on caller-owned device buffers: n records d_rois, WLE
 * rows d_wle (required), rows into d_rows (room for 2 x n rows, 16-byte
 * aligned, else QCS_ERR_ARG), row count
 * into *d_nvalid (device int, may be NULL).  Allocates nothing: its queues
 * and counters live in one fixed library array, so n is limited to
 * QCS_NOALLOC_MAX_ROIS (else QCS_ERR_CAPACITY).  The first call on a device
 * looks up that array's address; make it before any stream capture.  After a
 * device reset the next call looks the address up again in the new context,
 * so that call, too, must come before any capture.  QE <= 0 is refused
 * (QCS_ERR_ARG) before any device work.  All
 * calls on a device share the array: calls that overlap on the GPU race and
 * must not be issued.  Asynchronous on `stream`.
 */
#define QCS_NOALLOC_MAX_ROIS 8192
int qcs_localize_noalloc(const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n, float *d_rows,
                         int *d_nvalid, void *stream);

/* ---- diagnostics --------------------------------------------------------- */
/* Sustained special-function-unit rate of the loss's __expf/__logf pair on
 * the current device: *ops MUFU operations in *ms milliseconds.  Used as the
 * measured peak of the fit kernel's roofline; no counterpart in the reference. */
int qcs_measure_mufu_rate(int iters, float *ms, double *ops);

#ifdef __cplusplus
}
#endif

#endif /* QCSTORM_B200_H */
