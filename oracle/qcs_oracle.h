/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle of the QC-STORM MLEbfgs path.
 *
 * A plain-C restatement of the reference algorithm (file:line citations in
 * qcs_oracle_impl.h), used by the tests as the parity checker and by
 * bench.py as the timed CPU baseline.  It is never called by the product
 * library.  The float build (suffix _f32) follows the reference's operation
 * order so that, compiled with -ffp-contract=off against glibc expf/logf, it
 * reproduces the host build of the reference bit for bit (pinned by
 * tests/test_oracle_pin.py against oracle/_ref/libqcs_ref_host.so).  The
 * double build (suffix _f64) runs the same fixed schedule in FP64 and gives
 * the "error against FP64" of each result.
 */
#ifndef QCS_ORACLE_H
#define QCS_ORACLE_H

#include <stdint.h>
#include "../include/qcstorm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of OpenMP threads used by the batch entry points (0 = all cores). */
void qcso_set_threads(int n);
int qcso_get_threads(void);

/* WLE pre-pass: PSF width, nearest neighbour, molecule type.  wle: n x 6. */
int qcso_wle(const qcs_loc_para *p, const uint16_t *rois, int n, float *wle);

/* Whole BFGS_MLELocalization: classify, single fit, 2E/3E cascade, CRLB.
 * out: out_cap x 12; *n_valid = rows written; ratios: 7 floats or NULL. */
int qcso_localize_f32(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n,
                      float *out, int out_cap, int *n_valid, float *ratios);
int qcso_localize_f64(const qcs_loc_para *p, const uint16_t *rois, const float *wle, int n,
                      float *out, int out_cap, int *n_valid, float *ratios);

/* One single-emitter fit pass over all n ROIs (kind 0 GS2D, 1 AS3D), no
 * cascade and no CRLB: the kernel-level output. out: n x 12. */
int qcso_fit_single_f32(int kind, const qcs_loc_para *p, const uint16_t *rois, const float *wle,
                        int n, float *out);
int qcso_fit_single_f64(int kind, const qcs_loc_para *p, const uint16_t *rois, const float *wle,
                        int n, float *out);

/* CRLB columns 9/10 over n rows, in place. */
int qcso_crlb(const qcs_loc_para *p, float *loc, int n);

/* FP64 Fisher-matrix CRLB side output of n rows (qcs_crlb_fisher_fp64):
 * out n x QCS_FISHER_COLS; rois / n_rois as in the product's entry point. */
int qcso_crlb_fisher_f64(const qcs_loc_para *p, const float *rows, int n, const uint16_t *rois, int n_rois,
                         float *out);

/* ROI extraction over n_frames frames fed in batches of `batch` frames, as
 * consecutive ExtractMolecules calls; rois_out cap x R(R+1), wle_out cap x 6.
 * flags selects the arithmetic of the two steps whose rounding depends on how
 * the reference is built and run:
 *   QCSO_EXTRACT_FMA_CONV        smoothing taps accumulated with fused
 *                                multiply-add, as nvcc compiles the
 *                                reference's convolution kernels (without
 *                                it: separately rounded, the host build);
 *   QCSO_EXTRACT_EXACT_VARIANCE  variance from exact integer sums (the
 *                                product's deterministic definition; without
 *                                it: float sums in pixel order, the order the
 *                                host build's one-block-at-a-time run adds in). */
#define QCSO_EXTRACT_FMA_CONV 1
#define QCSO_EXTRACT_EXACT_VARIANCE 2
int qcso_extract(const qcs_loc_para *p, const uint16_t *frames, int n_frames, int batch,
                 int start_frame, int flags, uint16_t *rois_out, float *wle_out, int cap,
                 int *n_roi, int *first_frame, int *end_frame);

/* RemoveZeroLocalizations: rows n x 12 in, kept rows into out (n x 12), count in *n_out. */
/* Super-resolution render of n rows into img (SRImageWidth x SRImageHigh) and,
 * for 3D types, the z-weighted colormap; max_val and hist (400 ints) are the
 * running display maximum and histogram.  All four are read and updated. */
int qcso_render(const qcs_loc_para *p, const float *rows, int n, int mode, float fixed_prec, float *img,
                float *colormap, int *max_val, int *hist);

int qcso_zero_remove(const float *rows, int n, int sort_frame, int first_frame, int end_frame, float *out,
                     int *n_out);

/* ConsecutiveFit_WeightedAvg over n_groups groups of sizes[g] rows in turn (is_end[g]: the call's
 * IsEndProc); each call's output rows back to back in out, their count in out_n[g], its 10 on-time
 * ratios at ontime[10 g]; gpu_rounding: fused weighted sums and GPU float-to-int truncation. */
int qcso_consec(const qcs_loc_para *p, const float *rows, const int *sizes, const int *is_end, int n_groups,
                int gpu_rounding, float *out, int *out_n, float *ontime);

/* GetStatisticalInf over n_groups groups of sizes[g] rows in turn (after ResetAllDat); after call g:
 * hist[g * 6400 ..] the four 1600-bin histograms, means[g * 10 ..] the means (see qcs_oracle_stat.c). */
int qcso_stat(const qcs_loc_para *p, const float *rows, const int *sizes, int n_groups, int *hist, float *means);
/* UpdateOntimeRatio: the exponential fit of n (>= 4) on-time ratios, the mean on
 * time, and the ratios with entries 4.. summed into entry 3 and 0..3 clamped. */
int qcso_ontime(const float *ratios, int n, float *mean_ontime, float *out);

#ifdef __cplusplus
}
#endif

#endif
