// Host-side entry points of the qcstorm_b200 kernels (all asynchronous on a
// caller-given stream; device pointers only).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "qcs_device.cuh"

namespace qcs {

struct FitLaunch {
    const uint16_t *rois;  // records, R*(R+1) uint16 each
    const float *wle;      // 6 floats per record
    Queue q;               // which records this launch fits
    int max_count;         // upper bound of the queue length (grid size)
    float *loc;            // 12-float rows, indexed by record id
    uint8_t *to2e;         // single-emitter kinds: per-record "send to 2E" flag (may be null)
    MultiOut mo;           // multi-emitter kinds: per-slot result + second-emitter row
    CorePara para;
    cudaStream_t stream;
    // when set: the unweighted Poisson log-likelihood sum(n ln mu - mu) of the
    // fitted model, FP64, per record id (one-thread and multi-emitter group
    // kernels; the likelihood-ratio model selection)
    double *ll = nullptr;
    // learned-start single fits with multi-emitter fitting (to2e set): a fit
    // that is rejected or judged poor and has SNR > 6 goes straight to the
    // two-emitter queue (the reference's rule for rejected single fits) instead
    // of a plain refit; fits with SNR <= 6 are still refitted
    int direct2e = 0;
    // multi-emitter kinds: the one-thread-per-ROI kernel even where the lane-group
    // kernel exists (queues of every record, where throughput, not one ROI's
    // latency, sets the time)
    int thread_per_roi = 0;
    // multi-emitter kinds: the longest queue the lane-group kernel fits (0: the
    // default, about three of its waves; the autotuner measures it)
    int group_limit = 0;
};

// kind: FitKind (qcs_fit_math.cuh); R: ROI size.
cudaError_t launch_fit(int kind, int R, const FitLaunch &a);
// Multi-emitter kinds and sizes with a lane-group kernel, and the default
// queue-length limit up to which it fits a stage (0 where there is none).
bool multi_group_available(int kind, int R);
int multi_group_default_limit(int kind, int R);

// Single-emitter kinds with `lanes` lanes per ROI (8; also 4 and 16 for GS2D
// 7x7): the rows of launch_fit bit for bit, lower latency.  Sizes: GS2D 7, 9,
// 11, 13 and AS3D 7, 9, 11 (group_fit_supported).
bool group_fit_supported(int kind, int R);
cudaError_t launch_fit_group(int kind, int R, int lanes, const FitLaunch &a);

// Single-emitter fits (GS2D / AS3D, ROI sizes 7, 9, 11; the fit kinds of
// launch_fit) of up to kMixedMax launches of different ROI sizes in one
// persistent launch: rows and 2E flags of each launch_fit(kind[i], R[i],
// f[i]) bit for bit.  Records must start on a 4-byte boundary; ll unused.
// d_next: one device int of scratch (set to zero on the stream first).
constexpr int kMixedMax = 6;
bool mixed_fit_supported(int kind, int R);
cudaError_t launch_fit_mixed(const FitLaunch *f, const int *kind, const int *R, int count, int *d_next,
                             cudaStream_t s);

// Single-emitter fit (kind kGS2D or kAS3D; R = 7, 9, 11) of the records of
// a.q (grid from a.max_count) started from start[P * id] (GS2D P = 5: peak
// e-, x, y, sigma, background e-; AS3D P = 6: peak e-, x, y, sigma_x,
// sigma_y, background e-) with `iters` BFGS iterations of `bisections`
// line-search steps (learned_schedule_supported); rows into a.loc,
// refit[id] = 1 for fits to redo with the plain kernel, a.to2e[id] = 0 when
// a.to2e is set.
bool learned_schedule_supported(int kind, int R, int iters, int bisections);
cudaError_t launch_fit_learned(int kind, int R, int iters, int bisections, const FitLaunch &a, const float *start,
                               float dev_th, uint8_t *refit);
// Learned-start GS2D two-emitter fit (R = 7, 9, 11) of the records of a.q
// (grid from a.max_count) from start[8 id ..] (peak e-, x, y of emitter 0 and
// of emitter 1, sigma, background e-) with `iters` iterations of `bisections`
// steps (learned_2e_supported): rows and stage results as launch_fit(k2E);
// poor fits get refit[slot] = 1 (to3e = 0: to redo with the plain kernel) or
// stage result 0 and no rows (to3e = 1: on to the three-emitter fit).
bool learned_2e_supported(int R, int iters, int bisections);
cudaError_t launch_fit_learned_2e(int R, int iters, int bisections, const FitLaunch &a, const float *start,
                                  float dev_th, uint8_t *refit, int to3e);
// Learned-start GS2D three-emitter fit (R = 7, 9, 11) of the records of a.q
// (grid from a.max_count) from start[11 id ..] (peak e-, x, y of emitters 0,
// 1, 2, sigma, background e-) with `iters` iterations of `bisections` steps
// (learned_3e_supported): rows and stage results as launch_fit(k3E); poor fits
// get refit[slot] = 1 (to redo with the plain kernel).
bool learned_3e_supported(int R, int iters, int bisections);
cudaError_t launch_fit_learned_3e(int R, int iters, int bisections, const FitLaunch &a, const float *start,
                                  float dev_th, uint8_t *refit);
// slots[] / ids[]: the queue slots i < min(*n_dev, max_n) with flags[i] != 0
// and q[i]; *count = their number.
cudaError_t launch_flag_slots(const uint8_t *flags, const int *n_dev, int max_n, const int *q, int *slots, int *ids,
                              int *count, cudaStream_t s);
// res[slots[k]] = res_k[k] and, when 2, extra[slots[k]] = extra_k[k] (12 floats), k < min(*count, max_n).
cudaError_t launch_merge_refit(const int *slots, const int *count, int max_n, const int8_t *res_k,
                               const float *extra_k, int8_t *res, float *extra, cudaStream_t s);
// ids[] = the indices i < n with flags[i] != 0 (any order), *count = their number.
cudaError_t launch_flag_queue(const uint8_t *flags, int n, int *ids, int *count, cudaStream_t s);

// CRLB columns 9/10 of rows [0, *n_dev) (or [0, n) when n_dev is null);
// grid sized for max_rows.  LocPrecCalc_GaussianCRLB.h:65-243.
// ids (optional): the rows are loc[ids[i]] for i < count; skip (optional,
// indexed by row): rows with skip[row] != 0 are left unchanged.
cudaError_t launch_crlb(float *loc, const int *n_dev, int n, int max_rows, int loc_type, float ReadNoise_e, float QE,
                        float PixelSize, cudaStream_t s, const int *ids = nullptr, const uint8_t *skip = nullptr);

// WLE pre-pass over n records: PSF width, same-frame nearest neighbour and
// molecule type into wle (6 floats per record).  scratch must hold
// wle_scratch_bytes(n) bytes.
size_t wle_scratch_bytes(int n);

// WLE pre-pass of a localization context: the nearest-neighbour key sort
// runs (inside a CUDA graph's IF node) only when the records are not already
// in (frame, y, x) order.  scratch: wle_scratch_bytes(capacity) bytes, owned
// by the caller.  Calls above capacity, or on a stream being captured, take
// launch_wle.
struct WleSorter;
cudaError_t wle_sorter_create(int capacity, void *scratch, WleSorter **out);
void wle_sorter_destroy(WleSorter *w);
cudaError_t launch_wle_ctx(WleSorter *w, const uint16_t *rois, int n, int R, int loc_type, float *wle,
                           cudaStream_t s);
cudaError_t launch_wle(const uint16_t *rois, int n, int R, int loc_type, float *wle, void *scratch, cudaStream_t s);

// The same pass over records [d_span[0], d_span[0] + d_span[1]) (read on the
// device; d_span[1] <= max_n) that are already in ascending (frame, y, x)
// order, as ROI extraction writes them, with keys[i] = frame << 32 | y << 16 | x
// of record i: no sort, no scratch, no host sync.
cudaError_t launch_wle_presorted(const uint16_t *rois, const unsigned long long *keys, const int *d_span, int max_n,
                                 int R, int loc_type, float *wle, cudaStream_t s);

// FP64 Fisher-matrix CRLB of localization rows (qcs_crlb_fisher_fp64): n
// rows, or min(*n_dev, n) when n_dev is set; rois: the records of the first
// n_rois rows (may be null); out: n x QCS_FISHER_COLS floats.
cudaError_t launch_crlb_fisher(const qcs_loc_para &p, const float *rows, int n, const int *n_dev,
                               const uint16_t *rois, int n_rois, float *out, cudaStream_t s);

}  // namespace qcs
