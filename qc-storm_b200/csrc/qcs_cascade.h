// Device-side cascade of the localization call (see qcs_cascade.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"

namespace qcs {

// Device counters of one localization call.
enum {
    kCntSingle = 0,      // single-emitter queue length
    kCnt2E = 1,          // two-emitter queue length (classified + rejected singles)
    kCnt2EClassify = 2,  // two-emitter queue entries that came from the classifier
    kCnt3E = 3,          // three-emitter queue length
    kCntRejected = 4,    // ROIs rejected by the last multi-emitter stage
    kCntRows = 5,        // rows produced (records + appended second emitters)
    kCntValid = 6,       // rows produced, capped at the row capacity
    kCnt3EClassify = 7,  // three-emitter queue entries that came from the classifier (learned classes)
    kCntRefit = 8,       // learned path: records refitted by the plain single-emitter fit
    kCntRefit2E = 9,     // learned path: two-emitter fits redone by the plain two-emitter fit
    kCntSel1 = 10,       // likelihood-ratio selection: records that keep the one-emitter model
    kCntSel2 = 11,       //   ... the two-emitter model
    kCntSel3 = 12,       //   ... the three-emitter model
    kCntRefit3E = 13,    // learned path: three-emitter fits redone by the plain three-emitter fit
    kCntMixedNext = 14,  // mixed-size call (first context): the persistent launch's next tile
    kCntNum = 16
};

// Scratch of one context, sized for `capacity` records.
struct CascadeState {
    int *q_single;   // capacity
    int *q2;         // capacity
    int *q3;         // capacity
    uint8_t *to2e;   // capacity, indexed by record
    int8_t *res2;    // capacity, indexed by 2E queue slot
    int8_t *res3;    // capacity, indexed by 3E queue slot
    float *extra2;   // capacity x 12
    float *extra3;   // capacity x 12
    int *counters;   // kCntNum
    int *scan;       // cascade_scan_ints(capacity): the multi-block compactions' tile counts
};

// ints of CascadeState::scan for `capacity` records
constexpr int cascade_scan_ints(int capacity) { return 4 + 3 * ((capacity + 1023) / 1024 + 1); }

// Learned start points of the GS2D two-emitter stage: the stage fits its
// queue from start[8 id ..] with iters x bisections (launch_fit_learned_2e),
// the plain two-emitter fit redoes the fits it judges poor (refit, per queue
// slot; slots / ids: scratch of the queue's capacity) and their results go
// back to the slots they came from, so the stages after it see the
// reference's layout; or, with to3e, the poor fits go on to the three-emitter
// fit as the reference's rejected two-emitter fits do.
struct TwoEmitterStart {
    const float *start;
    int iters, bisections;
    float dev_th;
    int to3e;  // 1: poor fits go on to the three-emitter fit; 0: plain refit; 2: no refit (their results stand)
    uint8_t *refit;
    int *slots, *ids;
};

// Learned starts of the GS2D three-emitter stage: start points (11 per
// record), schedule, deviance bound; per 3E-queue slot refit flags, and the
// slots and record ids of the plain refits.
struct ThreeEmitterStart {
    const float *start;
    int iters, bisections;
    float dev_th;  // < 0: no plain refits (the learned fits' results stand)
    uint8_t *refit;
    int *slots, *ids;
};

struct CascadeArgs {
    qcs_loc_para para;
    const uint16_t *rois;  // device, n records
    const float *wle;      // device, n x 6
    int n;                 // record count, or its upper bound when n_dev is set
    const int *n_dev = nullptr;  // device record count (read on the device), or null
    float *loc;            // device, max_rows x 12
    int max_rows;
    cudaStream_t stream;
    const uint8_t *pred = nullptr;  // learned emitter-count class per record, or null (the reference's split)
    int lanes = 1;  // lanes per ROI of the single-emitter fit: 1 (one thread per ROI) or 4 / 8 / 16 (group kernel)
    const TwoEmitterStart *two = nullptr;  // learned two-emitter starts (GS2D), or null (the reference's)
    const ThreeEmitterStart *three = nullptr;  // learned three-emitter starts (GS2D), or null (the reference's)
    float *params3 = nullptr;  // when set: the plain three-emitter fits' parameters, 11 per 3E-queue slot
    // when set: recorded after the two- / three-emitter start points, computed on another stream; the
    // multi-emitter stages wait for it
    cudaEvent_t starts_ready = nullptr;
    int group_limit2 = 0, group_limit3 = 0;  // tuned lane-group queue limits of the 2E / 3E stages (0: default)
};

// The whole localization call: queues, single-emitter fit, 2E / 3E fits,
// CRLB.
cudaError_t run_cascade(const CascadeArgs &a, const CascadeState &st);

// Likelihood-ratio model selection (a selectable mode in place of the
// reference's SNR cascade; GS2D or DH3D with multi-emitter fitting): every
// record is fitted with one, two and three emitters (the reference's fits,
// schedules and accept rules), the unweighted Poisson log-likelihood of each
// fitted model is summed in FP64, and a record keeps the smallest accepted
// model unless a larger accepted one raises 2 ln L by more than `threshold`
// per added emitter.  Its rows (the chosen model's, up to two emitters as the
// reference writes them) then take the cascade's output layout and CRLB.
struct LrScratch {
    float *loc2, *loc3;      // capacity x 12: rows of the two- and three-emitter fits
    double *ll1, *ll2, *ll3;  // capacity: their log-likelihoods
    float threshold;
};
cudaError_t run_cascade_lr(const CascadeArgs &a, const CascadeState &st, const LrScratch &lr);

// Its phases, for callers that replace the single-emitter fit (the learned
// path): the queues; the single-emitter launch run_cascade makes over them;
// everything after the single-emitter fit (which must have set to2e for
// every record of the single queue when multi-emitter fitting is on).
cudaError_t cascade_classify(const CascadeArgs &a, const CascadeState &st);
struct FitLaunch cascade_single_launch(const CascadeArgs &a, const CascadeState &st);
cudaError_t cascade_tail(const CascadeArgs &a, const CascadeState &st);

}  // namespace qcs
