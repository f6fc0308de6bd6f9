// C ABI of libqcstorm_b200 (include/qcstorm_b200.h): localization contexts
// (LDLocData_TypeDef), the WLE pre-pass (WLEParameterEstimation_TypeDef) and
// kernel-level entry points.  All device memory of a context is allocated
// once at init for its record capacity; calls allocate nothing.
#include <cstdio>
#include <cstring>
#include <string>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_cascade.h"
#include "qcs_error.h"
#include "qcs_fit_math.cuh"
#include "qcs_kernels.h"
#include "qcs_learned.h"

namespace {

thread_local std::string g_err;

}  // namespace

int qcs::fail(int code, const char *what, cudaError_t e) {
    g_err = what;
    if (e != cudaSuccess) {
        g_err += ": ";
        g_err += cudaGetErrorString(e);
    }
    return code;
}

namespace {

using qcs::fail;

int check_para(const qcs_loc_para *p, bool multi_ok_sizes = true) {
    if (!p) return fail(QCS_ERR_ARG, "null parameter struct");
    if (p->LocType < QCS_LOCTYPE_GS2D || p->LocType > QCS_LOCTYPE_DH3D) return fail(QCS_ERR_ARG, "LocType out of range");
    const int R = p->ROISize;
    if (R < 5 || R > 17 || (R & 1) == 0) return fail(QCS_ERR_ROISIZE, "ROISize must be odd, 5..17");
    if (multi_ok_sizes && p->MultiEmitterFitEn && R > 13)
        return fail(QCS_ERR_ROISIZE, "multi-emitter fitting supports ROISize 5..13");
    if (!(p->QE > 0.0f)) return fail(QCS_ERR_ARG, "QE must be positive");
    return QCS_OK;
}

}  // namespace

struct qcs_loc_data {
    qcs_loc_para para;
    int R, whole, capacity, max_rows;
    uint16_t *d_rois = nullptr;
    float *d_wle = nullptr;
    float *d_loc = nullptr;
    void *d_wle_scratch = nullptr;
    size_t wle_scratch = 0;
    qcs::WleSorter *wle_sorter = nullptr;  // WLE pre-pass, sort only for out-of-order records
    qcs::CascadeState st{};
    void *d_state = nullptr;
    float *h_loc = nullptr;
    int *h_counters = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // high-priority stream for work overlapped with the main stream
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the two- / three-emitter start points of a learned call run on their own stream, overlapping the
    // single-emitter stage; the multi-emitter stages wait for ev_sready
    cudaStream_t starts = nullptr;
    cudaEvent_t ev_sfork = nullptr, ev_sready = nullptr;
    cudaEvent_t starts_ready = nullptr;  // set for the duration of such a call
    cudaEvent_t ev_done = nullptr;  // end of the last asynchronous host call
    float *d_start = nullptr;       // learned start points, capacity x 6 (one block with the three below)
    int *q_refit = nullptr;         // learned multi-emitter path: records to refit plainly
    uint8_t *d_refit = nullptr;     //   their per-record flags
    uint8_t *d_cls = nullptr;       //   emitter-count class per record
    float *d_start2 = nullptr;      // two-emitter start points, capacity x 8 (one block with the three below)
    uint8_t *d_refit2 = nullptr;    //   per 2E-queue slot refit flags
    int *d_slots2 = nullptr;        //   slots and record ids of the two-emitter refits
    int *d_ids2 = nullptr;
    const qcs::TwoEmitterStart *two = nullptr;  // set for the duration of a learned call with a two-emitter net
    // three-emitter block (allocated on first use): start points (capacity x 11), refit flags, refit slots and
    // ids, and the captured parameters of the plain three-emitter fits (capacity x 11)
    float *d_start3 = nullptr, *d_params3 = nullptr;
    uint8_t *d_refit3 = nullptr;
    int *d_slots3 = nullptr, *d_ids3 = nullptr;
    int capture3 = 0;  // qcs_loc_set_three_emitter_capture
    const qcs::ThreeEmitterStart *three = nullptr;  // set for the duration of a learned call with a 3E net
    // autotuned lanes per ROI of the single-emitter fit by batch size: batches of
    // at most tune_n[k] records use tune_lanes[k] (first match); none: 1
    int tune_count = 0;
    int tune_n[8] = {0};
    int tune_lanes[8] = {0};
    // tuned longest queues the lane-group multi-emitter kernels fit (2E / AS3D-2E, 3E; 0: their default)
    int tune_limit2 = 0, tune_limit3 = 0;
    // model selection of multi-emitter calls: QCS_SELECT_CASCADE (the reference's) or QCS_SELECT_LR
    int sel_mode = QCS_SELECT_CASCADE;
    float sel_th = QCS_SELECT_LR_DEFAULT_TH;
    void *d_lr = nullptr;           // QCS_SELECT_LR scratch: loc2 / loc3 rows, three log-likelihood arrays
    int lr_stats = 0;               // the last call ran the likelihood-ratio selection
    int pending = 0;                // an asynchronous host call awaits qcs_loc_finish
    int pending_n = 0;
    int valid = 0;
    float ratios[7] = {0, 0, 0, 0, 0, 0, 0};
};

extern "C" {

void qcs_loc_para_default(qcs_loc_para *p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->KAdc = 0.45f;
    p->Offset = 100.0f;
    p->QE = 0.72f;
    p->ReadNoise_e = 1.3f;
    p->ROISize = 7;
    p->LocType = QCS_LOCTYPE_GS2D;
    p->MultiEmitterFitEn = 0;
    p->WLEEn = 1;
    p->ConsecFit_DistanceTh_nm = 80.0f;
    p->ConsecFitEn = 0;
    p->PixelSize = 100.0f;
    p->PixelZoom = 5.0f;
    p->SNR_th = 5.0f;
    p->ColorMode_3D = 0;
    p->ImageWidth = 2048;
    p->ImageHigh = 2048;
    p->TotalFrameNum = 1;
    p->MinZDepth = -500.0f;
    p->MaxZDepth = 500.0f;
    p->ZDepthCorrFactor = 1.0f;
    p->p1_XGY = 1.0f;
    p->p1_XLY = 1.0f;
    p->DH_RotateType = 0;
    p->DH_MeanDistance = 10.0f;
    p->DH_DistanceTh = 2.0f;
    p->ImagesPerGroup = 50;
    p->IsHollowTube = 0;
    p->StrucuteSize_2D = 40.0f;
    p->SpatialResolutionCalcEn = 1;
    p->SRImageWidth = ((int)(p->ImageWidth * p->PixelZoom) + 3) / 4 * 4;
    p->SRImageHigh = ((int)(p->ImageHigh * p->PixelZoom) + 3) / 4 * 4;
}

const char *qcs_last_error(void) { return g_err.c_str(); }

int qcs_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n > 0;
}

int qcs_loc_deinit(qcs_loc_data *c) {
    if (!c) return QCS_OK;
    cudaFree(c->d_rois);
    cudaFree(c->d_wle);
    cudaFree(c->d_loc);
    cudaFree(c->d_wle_scratch);
    cudaFree(c->d_state);
    cudaFreeHost(c->h_loc);
    cudaFreeHost(c->h_counters);
    if (c->pending && c->ev_done) cudaEventSynchronize(c->ev_done);
    qcs::wle_sorter_destroy(c->wle_sorter);
    cudaFree(c->d_start);
    cudaFree(c->d_start2);
    cudaFree(c->d_start3);
    cudaFree(c->d_lr);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->starts) cudaStreamDestroy(c->starts);
    if (c->ev_sfork) cudaEventDestroy(c->ev_sfork);
    if (c->ev_sready) cudaEventDestroy(c->ev_sready);
    delete c;
    return QCS_OK;
}

int qcs_loc_init_capacity(const qcs_loc_para *p, int capacity, qcs_loc_data **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    int st = check_para(p, false);
    if (st) return st;
    if (capacity <= 0) capacity = QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_loc_data *c = new qcs_loc_data();
    c->para = *p;
    c->R = p->ROISize;
    c->whole = c->R * (c->R + 1);
    c->capacity = capacity;
    c->max_rows = 2 * capacity;
    const size_t cap = (size_t)capacity;
    auto A = [&](void **ptr, size_t bytes) { return cudaMalloc(ptr, bytes > 0 ? bytes : 1); };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = A((void **)&c->d_rois, cap * c->whole * sizeof(uint16_t));
    if (e == cudaSuccess) e = A((void **)&c->d_wle, cap * QCS_WLE_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = A((void **)&c->d_loc, (size_t)c->max_rows * QCS_OUT_PARA_NUM * sizeof(float));
    c->wle_scratch = qcs::wle_scratch_bytes(capacity);
    if (e == cudaSuccess) e = A(&c->d_wle_scratch, c->wle_scratch);
    // cascade state in one allocation; every part starts on a 256-byte boundary whatever the capacity (the
    // kernels move 12-float rows as float4, which needs 16-byte alignment)
    auto round256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t a_int = round256(cap * sizeof(int)), a_u8 = round256(cap), a_row = round256(cap * 12 * sizeof(float));
    const size_t a_scan = round256((size_t)qcs::cascade_scan_ints(capacity) * sizeof(int));
    const size_t bytes = 3 * a_int + 3 * a_u8 + 2 * a_row + 256 + a_scan;
    if (e == cudaSuccess) e = A(&c->d_state, bytes);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_loc, (size_t)c->max_rows * QCS_OUT_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_counters, qcs::kCntNum * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    int prio_least = 0, prio_greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->starts, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_sfork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_sready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = qcs::wle_sorter_create(capacity, c->d_wle_scratch, &c->wle_sorter);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming);
    const size_t b_start = round256(cap * 6 * sizeof(float)), b_refit = round256(cap * sizeof(int));
    if (e == cudaSuccess) e = A((void **)&c->d_start, b_start + b_refit + 2 * round256(cap));
    const size_t b_start2 = round256(cap * 8 * sizeof(float));
    if (e == cudaSuccess) e = A((void **)&c->d_start2, b_start2 + round256(cap) + 2 * b_refit);
    if (e != cudaSuccess) {
        qcs_loc_deinit(c);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_loc_init", e);
    }
    char *s = static_cast<char *>(c->d_state);
    c->st.q_single = reinterpret_cast<int *>(s); s += a_int;
    c->st.q2 = reinterpret_cast<int *>(s); s += a_int;
    c->st.q3 = reinterpret_cast<int *>(s); s += a_int;
    c->st.to2e = reinterpret_cast<uint8_t *>(s); s += a_u8;
    c->st.res2 = reinterpret_cast<int8_t *>(s); s += a_u8;
    c->st.res3 = reinterpret_cast<int8_t *>(s); s += a_u8;
    c->st.extra2 = reinterpret_cast<float *>(s); s += a_row;
    c->st.extra3 = reinterpret_cast<float *>(s); s += a_row;
    c->st.counters = reinterpret_cast<int *>(s); s += 256;
    c->st.scan = reinterpret_cast<int *>(s);
    char *b = reinterpret_cast<char *>(c->d_start);
    c->q_refit = reinterpret_cast<int *>(b + b_start);
    c->d_refit = reinterpret_cast<uint8_t *>(b + b_start + b_refit);
    c->d_cls = c->d_refit + round256(cap);
    char *b2 = reinterpret_cast<char *>(c->d_start2);
    c->d_refit2 = reinterpret_cast<uint8_t *>(b2 + b_start2);
    c->d_slots2 = reinterpret_cast<int *>(b2 + b_start2 + round256(cap));
    c->d_ids2 = reinterpret_cast<int *>(b2 + b_start2 + round256(cap) + b_refit);
    *out = c;
    return QCS_OK;
}

int qcs_loc_init(const qcs_loc_para *p, qcs_loc_data **out) { return qcs_loc_init_capacity(p, QCS_MAX_POINT_NUM, out); }

int qcs_loc_capacity(const qcs_loc_data *c) { return c ? c->capacity : 0; }

static int check_call(qcs_loc_data *c, const qcs_loc_para *p, int n) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    int st = check_para(p);
    if (st) return st;
    if (p->ROISize != c->R) return fail(QCS_ERR_ROISIZE, "ROISize differs from the one the context was created with");
    if (n < 0) return fail(QCS_ERR_ARG, "negative ROI count");
    if (n > c->capacity) return fail(QCS_ERR_CAPACITY, "ROI count above the context capacity");
    if (c->pending) return fail(QCS_ERR_ARG, "an asynchronous call on this context awaits qcs_loc_finish");
    return QCS_OK;
}

// The call runs the likelihood-ratio selection: the mode is set and the
// parameters ask for GS2D (or DH3D) multi-emitter fitting.
static bool use_lr(const qcs_loc_data *c, const qcs_loc_para *p) {
    return c->sel_mode == QCS_SELECT_LR && c->d_lr && p->MultiEmitterFitEn &&
           (p->LocType == QCS_LOCTYPE_GS2D || p->LocType == QCS_LOCTYPE_DH3D);
}

static qcs::LrScratch lr_scratch(const qcs_loc_data *c) {
    const size_t cap = (size_t)c->capacity;
    qcs::LrScratch lr;
    char *b = static_cast<char *>(c->d_lr);
    lr.loc2 = reinterpret_cast<float *>(b);
    lr.loc3 = lr.loc2 + cap * 12;
    lr.ll1 = reinterpret_cast<double *>(lr.loc3 + cap * 12);  // 2 x cap x 48 bytes: 8-byte aligned
    lr.ll2 = lr.ll1 + cap;
    lr.ll3 = lr.ll2 + cap;
    lr.threshold = c->sel_th;
    return lr;
}

// The call's localization: the reference's cascade, or the likelihood-ratio selection.
static cudaError_t run_localization(qcs_loc_data *c, const qcs::CascadeArgs &a) {
    c->lr_stats = use_lr(c, &a.para) ? 1 : 0;
    if (c->lr_stats) return qcs::run_cascade_lr(a, c->st, lr_scratch(c));
    if (c->capture3 && c->d_params3) {
        qcs::CascadeArgs b = a;
        b.params3 = c->d_params3;
        return qcs::run_cascade(b, c->st);
    }
    return qcs::run_cascade(a, c->st);
}

// The context's three-emitter block, allocated on first use (outside any
// stream capture: an allocation cannot be captured).
static int ensure_three(qcs_loc_data *c) {
    if (c->d_start3) return QCS_OK;
    auto round256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t cap = (size_t)c->capacity;
    const size_t b_par = round256(cap * 11 * sizeof(float)), b_int = round256(cap * sizeof(int));
    char *b = nullptr;
    const cudaError_t e = cudaMalloc((void **)&b, 2 * b_par + round256(cap) + 2 * b_int);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "three-emitter buffers", e);
    c->d_start3 = reinterpret_cast<float *>(b);
    c->d_params3 = reinterpret_cast<float *>(b + b_par);
    c->d_refit3 = reinterpret_cast<uint8_t *>(b + 2 * b_par);
    c->d_slots3 = reinterpret_cast<int *>(b + 2 * b_par + round256(cap));
    c->d_ids3 = reinterpret_cast<int *>(b + 2 * b_par + round256(cap) + b_int);
    return QCS_OK;
}

static int tuned_lanes(const qcs_loc_data *c, int n) {
    for (int k = 0; k < c->tune_count; ++k)
        if (n <= c->tune_n[k]) return c->tune_lanes[k];
    return 1;
}

int qcs_loc_localize_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p,
                            int n, void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    if (!d_rois && n > 0) return fail(QCS_ERR_ARG, "null ROI pointer");
    const float *wle = d_wle;
    if (!wle && n > 0) {
        QCS_CUDA(qcs::launch_wle_ctx(c->wle_sorter, d_rois, n, c->R, p->LocType, c->d_wle, s), "WLE pre-pass");
        wle = c->d_wle;
    }
    qcs::CascadeArgs a;
    a.para = *p;
    a.rois = d_rois;
    a.wle = wle;
    a.n = n;
    a.loc = c->d_loc;
    a.max_rows = c->max_rows;
    a.stream = s;
    a.lanes = tuned_lanes(c, n);
    a.group_limit2 = c->tune_limit2;
    a.group_limit3 = c->tune_limit3;
    QCS_CUDA(run_localization(c, a), "localization cascade");
    return QCS_OK;
}

int qcs_loc_localize_mixed_device(qcs_loc_data *const *ctx, const uint16_t *const *d_rois,
                                  const float *const *d_wle, const qcs_loc_para *p, const int *n, int count,
                                  void *stream) {
    static_assert(QCS_MIXED_MAX == qcs::kMixedMax, "mixed-size entries");
    if (!ctx || !d_rois || !d_wle || !p || !n) return fail(QCS_ERR_ARG, "null argument");
    if (count < 1 || count > QCS_MIXED_MAX) return fail(QCS_ERR_ARG, "entry count outside 1..QCS_MIXED_MAX");
    int kind[QCS_MIXED_MAX], R[QCS_MIXED_MAX];
    for (int i = 0; i < count; ++i) {
        int st = check_call(ctx[i], &p[i], n[i]);
        if (st) return st;
        for (int j = 0; j < i; ++j)
            if (ctx[j] == ctx[i]) return fail(QCS_ERR_ARG, "a context appears twice");
        if (use_lr(ctx[i], &p[i])) return fail(QCS_ERR_ARG, "likelihood-ratio selection runs per call");
        if (p[i].LocType != QCS_LOCTYPE_GS2D && p[i].LocType != QCS_LOCTYPE_AS3D && p[i].LocType != QCS_LOCTYPE_DH3D)
            return fail(QCS_ERR_ROISIZE, "fit kind outside GS2D / AS3D / DH3D");
        kind[i] = p[i].LocType == QCS_LOCTYPE_AS3D ? qcs::kAS3D : qcs::kGS2D;
        R[i] = p[i].ROISize;
        if (!qcs::mixed_fit_supported(kind[i], R[i])) return fail(QCS_ERR_ROISIZE, "ROI size outside 7, 9, 11");
        if (n[i] > 0 && !d_rois[i]) return fail(QCS_ERR_ARG, "null ROI pointer");
        if ((reinterpret_cast<uintptr_t>(d_rois[i]) & 3) != 0)
            return fail(QCS_ERR_ARG, "records must start on a 4-byte boundary");
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx[0]->stream;
    qcs::CascadeArgs a[QCS_MIXED_MAX];
    qcs::FitLaunch f[QCS_MIXED_MAX];
    for (int i = 0; i < count; ++i) {
        qcs_loc_data *c = ctx[i];
        const float *wle = d_wle[i];
        if (!wle && n[i] > 0) {
            QCS_CUDA(qcs::launch_wle_ctx(c->wle_sorter, d_rois[i], n[i], c->R, p[i].LocType, c->d_wle, s),
                     "WLE pre-pass");
            wle = c->d_wle;
        }
        c->lr_stats = 0;
        a[i].para = p[i];
        a[i].rois = d_rois[i];
        a[i].wle = wle;
        a[i].n = n[i];
        a[i].loc = c->d_loc;
        a[i].max_rows = c->max_rows;
        a[i].stream = s;
        a[i].group_limit2 = c->tune_limit2;
        a[i].group_limit3 = c->tune_limit3;
        QCS_CUDA(qcs::cascade_classify(a[i], c->st), "queues");
        f[i] = qcs::cascade_single_launch(a[i], c->st);
    }
    QCS_CUDA(qcs::launch_fit_mixed(f, kind, R, count, ctx[0]->st.counters + qcs::kCntMixedNext, s),
             "mixed-size single-emitter fit");
    for (int i = 0; i < count; ++i) QCS_CUDA(qcs::cascade_tail(a[i], ctx[i]->st), "localization cascade");
    return QCS_OK;
}

int qcs_loc_localize_device_n(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p,
                              const int *d_n, int max_n, void *stream) {
    int st = check_call(c, p, max_n);
    if (st) return st;
    if (!d_rois || !d_wle || !d_n) return fail(QCS_ERR_ARG, "null pointer");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    qcs::CascadeArgs a;
    a.para = *p;
    a.rois = d_rois;
    a.wle = d_wle;
    a.n = max_n;
    a.n_dev = d_n;
    a.loc = c->d_loc;
    a.max_rows = c->max_rows;
    a.stream = s;
    a.group_limit2 = c->tune_limit2;
    a.group_limit3 = c->tune_limit3;
    QCS_CUDA(run_localization(c, a), "localization cascade");
    return QCS_OK;
}

}  // extern "C"

namespace {
// rows for n records after a learned-start call; refits stay counted at
// st.counters[kCntSingle]
__global__ void learned_counters_kernel(qcs::CascadeState st, int n) {
    st.counters[qcs::kCntRefit] = st.counters[qcs::kCntSingle];
    st.counters[qcs::kCnt2E] = 0;
    st.counters[qcs::kCnt2EClassify] = 0;
    st.counters[qcs::kCnt3E] = 0;
    st.counters[qcs::kCntRejected] = 0;
    st.counters[qcs::kCntRows] = n;
    st.counters[qcs::kCntValid] = n;
}

// fit kind of a learned-start call; -1 when the shape has no learned path
int learned_kind(const qcs_loc_para *p) {
    if (p->ROISize != 7 && p->ROISize != 9 && p->ROISize != 11) return -1;
    if (p->LocType == QCS_LOCTYPE_GS2D) return qcs::kGS2D;
    if (p->LocType == QCS_LOCTYPE_AS3D && !p->MultiEmitterFitEn) return qcs::kAS3D;
    return -1;
}
// Deviance bound of the learned fits' judge: a good fit's unweighted Poisson
// deviance is near a chi-square with about R*R degrees of freedom, so the
// bound scales with the pixel count (100 for 7x7 ROIs).
float default_dev_th(int R) { return 2.0f * (float)(R * R) + 2.0f; }
const char *kLearnedShapes = "start-point fits: GS2D or AS3D, ROISize 7, 9 or 11 (multi-emitter fitting: GS2D)";
const char *kLearnedSchedules =
    "schedule: 2..4 iterations of 6 bisections or 3 of 11 (GS2D 7x7 also 2..5 or 8 of 11, 2 or 3 of 4 or 8)";

// Emitter-count class of each of n records from the cascade state of a plain
// multi-emitter call: 0 for records the call did not send to the two-emitter
// fit, then, over the 2E queue, 1 where that fit kept the ROI and 2 where it
// passed it on to the three-emitter fit.
__global__ void labels_zero_kernel(float *__restrict__ cls, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cls[i] = 0.0f;
}
__global__ void labels_2e_kernel(qcs::CascadeState st, int n, float *__restrict__ cls) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= st.counters[qcs::kCnt2E]) return;
    const int id = st.q2[k];
    if (id >= 0 && id < n) cls[id] = st.res2[k] == 0 ? 2.0f : 1.0f;
}

// Two-emitter targets (QCS_LEARNED_GS2D_2E network outputs) of the records
// whose plain two-emitter fit kept both emitters, read from the cascade state
// of a plain multi-emitter call: the first emitter's row at loc[id], the
// second's at extra2[slot].  valid[id] = 1 for those records (zero on entry).
template <int R>
__global__ void two_targets_kernel(qcs::CascadeState st, const uint16_t *__restrict__ rois,
                                   const float *__restrict__ loc, const float *__restrict__ scale, int n, float qe,
                                   float *__restrict__ tgt, float *__restrict__ valid) {
    enum { PIX = R * R, WHOLE = R * (R + 1), HALF = R / 2 };
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= st.counters[qcs::kCnt2E]) return;
    const int id = st.q2[k];
    if (id < 0 || id >= n || st.res2[k] != 2) return;
    const float *r0 = loc + (size_t)id * 12, *r1 = st.extra2 + (size_t)k * 12;
    const uint16_t *h = rois + (size_t)id * WHOLE + PIX;
    const float centre = R / 2.0f, lo = scale[2 * id], rng = scale[2 * id + 1];
    float *t = tgt + (size_t)id * 8;
    t[0] = r0[QCS_POS_XPOS] + (float)HALF - (float)h[0] - centre;
    t[1] = r0[QCS_POS_YPOS] + (float)HALF - (float)h[1] - centre;
    t[2] = r1[QCS_POS_XPOS] + (float)HALF - (float)h[0] - centre;
    t[3] = r1[QCS_POS_YPOS] + (float)HALF - (float)h[1] - centre;
    t[4] = logf(fmaxf(r0[QCS_POS_PPHO] * qe, 1e-3f) / rng);
    t[5] = logf(fmaxf(r1[QCS_POS_PPHO] * qe, 1e-3f) / rng);
    t[6] = r0[QCS_POS_SIGX] - 1.3f;
    t[7] = (r0[QCS_POS_BAKG] * qe - lo) / rng;
    valid[id] = 1.0f;
}

// Three-emitter targets (QCS_LEARNED_GS2D_3E network outputs) of the records
// whose plain three-emitter fit kept an emitter, from the parameters that
// fit captured (qcs_loc_set_three_emitter_capture): dx, dy of the three
// emitters, log(peak / range) of each, sigma - 1.3, (background - min) /
// range, the emitters ordered by peak x (R - distance from the centre), the
// order of the fit's own emitter selection.  valid[id] = 1 for those records.
template <int R>
__global__ void three_targets_kernel(qcs::CascadeState st, const float *__restrict__ params,
                                     const float *__restrict__ scale, int n, float *__restrict__ tgt,
                                     float *__restrict__ valid) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= st.counters[qcs::kCnt3E]) return;
    const int id = st.q3[k];
    if (id < 0 || id >= n || st.res3[k] == 0) return;
    const float *v = params + (size_t)k * 11;
    const float centre = R / 2.0f, lo = scale[2 * id], rng = scale[2 * id + 1];
    float key[3];
    int order[3] = {0, 1, 2};
    for (int e = 0; e < 3; ++e) {  // the fit's selection key (positions outside the ROI count as far away)
        float x = v[3 * e + 1], y = v[3 * e + 2];
        if (fabsf(x - centre) >= R / 2) x = -100.0f;
        if (fabsf(y - centre) >= R / 2) y = -100.0f;
        key[e] = v[3 * e] * (R - sqrtf((x - centre) * (x - centre) + (y - centre) * (y - centre)));
    }
    for (int a = 0; a < 2; ++a)  // three elements: sort by key, descending
        for (int b = 0; b < 2 - a; ++b)
            if (key[order[b]] < key[order[b + 1]]) {
                const int t = order[b];
                order[b] = order[b + 1];
                order[b + 1] = t;
            }
    float *t = tgt + (size_t)id * 11;
    for (int j = 0; j < 3; ++j) {
        const int e = order[j];
        t[2 * j] = v[3 * e + 1] - centre;
        t[2 * j + 1] = v[3 * e + 2] - centre;
        t[6 + j] = logf(fmaxf(v[3 * e] * QCS_ASCALE, 1e-3f) / rng);
    }
    t[9] = sqrtf(0.5f / (fmaxf(v[9], 1e-6f) * QCS_SSCALE)) - 1.3f;
    t[10] = (v[10] * QCS_BSCALE - lo) / rng;
    valid[id] = 1.0f;
}

// The learned multi-emitter call: the cascade's queues (with the predicted
// classes when cls is set), the learned-start single-emitter fit over the
// single queue, a plain refit of the fits it flags (which also flags the
// rejects that go on to the 2E fit), then the reference's 2E / 3E stages and
// the CRLB.
// direct2e (qcs_learned_set_direct_two_emitter, network-driven calls only):
// bright ROIs whose learned single fit is rejected or judged poor go straight
// to the two-emitter stage, without a plain refit first; otherwise every
// flagged fit is refitted plainly, which reproduces the reference's decisions.
cudaError_t learned_multi(qcs_loc_data *c, const uint16_t *d_rois, const float *wle, const qcs_loc_para *p, int n,
                          const int *n_dev, const float *d_start, const uint8_t *cls, int iters, int bisections,
                          float dev_th, cudaStream_t s, bool direct2e = false) {
    qcs::CascadeArgs a;
    a.para = *p;
    a.rois = d_rois;
    a.wle = wle;
    a.n = n;
    a.n_dev = n_dev;
    a.loc = c->d_loc;
    a.max_rows = c->max_rows;
    a.stream = s;
    a.pred = cls;
    a.two = c->two;
    a.three = c->three;
    a.starts_ready = c->starts_ready;
    a.group_limit2 = c->tune_limit2;
    a.group_limit3 = c->tune_limit3;
    cudaError_t e;
    if ((e = qcs::cascade_classify(a, c->st)) != cudaSuccess) return e;
    qcs::FitLaunch f = qcs::cascade_single_launch(a, c->st);
    f.direct2e = direct2e ? 1 : 0;
    if ((e = cudaMemsetAsync(c->d_refit, 0, (size_t)n, s)) != cudaSuccess) return e;
    const int R = p->ROISize;
    if ((e = qcs::launch_fit_learned(qcs::kGS2D, R, iters, bisections, f, d_start, dev_th, c->d_refit)) != cudaSuccess)
        return e;
    if ((e = qcs::launch_flag_queue(c->d_refit, n, c->q_refit, c->st.counters + qcs::kCntRefit, s)) != cudaSuccess)
        return e;
    f.q = qcs::Queue{c->q_refit, c->st.counters + qcs::kCntRefit, 0};
    // multi-emitter records refit by the thousands (every poor single fit of a ROI with several emitters):
    // a throughput-bound queue, one thread per ROI (the rows are the group kernel's bit for bit)
    if ((e = qcs::launch_fit(qcs::kGS2D, R, f)) != cudaSuccess) return e;
    return qcs::cascade_tail(a, c->st);
}

// When the GS2D network has a two-emitter network attached: its start points
// of the call's records into the context and the context's two-emitter stage
// set to use them (cleared by the caller after the call).
// The inference runs over all n records, not only the 2E queue: the queue is
// known only after the single-emitter stage, and the fused kernel's bulk
// copies read contiguous tiles of records.  It costs ~25 us per 100,000
// 11x11 records (about 0.5% of a learned multi-emitter call) and is enqueued
// before the single-emitter fits, which do not wait for it.
int two_emitter_starts(qcs_loc_data *c, const qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois,
                       int n, const int *n_dev, cudaStream_t s, qcs::TwoEmitterStart *two) {
    c->two = nullptr;
    int iters = 0, bisections = 0, to3e = 1;
    float dev_th = 0.0f;
    qcs_learned_net *net2 = qcs::learned::two_emitter(net, &iters, &bisections, &dev_th, &to3e);
    if (!net2 || p->LocType != QCS_LOCTYPE_GS2D || !p->MultiEmitterFitEn || n <= 0) return QCS_OK;
    QCS_CUDA(qcs::learned::start_points(net2, p, d_rois, n, c->d_start2, s, nullptr, n_dev),
             "two-emitter start points");
    *two = qcs::TwoEmitterStart{c->d_start2, iters, bisections, dev_th > 0.0f ? dev_th : default_dev_th(p->ROISize),
                                to3e, c->d_refit2, c->d_slots2, c->d_ids2};
    c->two = two;
    return QCS_OK;
}

// When the GS2D network has a three-emitter network attached: its start
// points of the call's records (all n, as for the two-emitter network) and the
// context's three-emitter stage set to use them (cleared by the caller).
int three_emitter_starts(qcs_loc_data *c, const qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois,
                         int n, const int *n_dev, cudaStream_t s, qcs::ThreeEmitterStart *three) {
    c->three = nullptr;
    int iters = 0, bisections = 0;
    float dev_th = 0.0f;
    qcs_learned_net *net3 = qcs::learned::three_emitter(net, &iters, &bisections, &dev_th);
    if (!net3 || p->LocType != QCS_LOCTYPE_GS2D || !p->MultiEmitterFitEn || n <= 0) return QCS_OK;
    if (!c->d_start3) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        QCS_CUDA(cudaStreamIsCapturing(s, &cs), "capture status");
        if (cs != cudaStreamCaptureStatusNone)
            return fail(QCS_ERR_STATE, "three-emitter start points: make one call outside a stream capture first");
        const int st = ensure_three(c);
        if (st) return st;
    }
    QCS_CUDA(qcs::learned::start_points(net3, p, d_rois, n, c->d_start3, s, nullptr, n_dev),
             "three-emitter start points");
    *three = qcs::ThreeEmitterStart{c->d_start3, iters, bisections,
                                    dev_th != 0.0f ? dev_th : default_dev_th(p->ROISize), c->d_refit3, c->d_slots3,
                                    c->d_ids3};
    c->three = three;
    return QCS_OK;
}

// The two- and three-emitter start points of a learned multi-emitter call
// (those of the networks attached to net), on the context's start-point
// stream forked from s: they overlap the single-emitter stage, and the
// cascade's multi-emitter stages wait for c->starts_ready (cleared by the
// caller after the call).
int multi_starts(qcs_loc_data *c, const qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                 const int *n_dev, cudaStream_t s, qcs::TwoEmitterStart *two, qcs::ThreeEmitterStart *three) {
    c->starts_ready = nullptr;
    c->two = nullptr;
    c->three = nullptr;
    int i2 = 0, b2 = 0, i3 = 0, b3 = 0, t3 = 0;
    float d2 = 0.0f, d3 = 0.0f;
    const bool any = qcs::learned::two_emitter(net, &i2, &b2, &d2, &t3) != nullptr ||
                     qcs::learned::three_emitter(net, &i3, &b3, &d3) != nullptr;
    if (!any || p->LocType != QCS_LOCTYPE_GS2D || !p->MultiEmitterFitEn || n <= 0) return QCS_OK;
    QCS_CUDA(cudaEventRecord(c->ev_sfork, s), "fork");
    QCS_CUDA(cudaStreamWaitEvent(c->starts, c->ev_sfork, 0), "fork");
    int st = two_emitter_starts(c, net, p, d_rois, n, n_dev, c->starts, two);
    if (st == QCS_OK) st = three_emitter_starts(c, net, p, d_rois, n, n_dev, c->starts, three);
    // joined even after an error, so that a capture in progress stays well formed
    QCS_CUDA(cudaEventRecord(c->ev_sready, c->starts), "join");
    if (st != QCS_OK) {
        QCS_CUDA(cudaStreamWaitEvent(s, c->ev_sready, 0), "join");
        c->two = nullptr;
        c->three = nullptr;
        return st;
    }
    c->starts_ready = c->ev_sready;
    return QCS_OK;
}

int fit_from_start(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p, int n,
                   const float *d_start, const uint8_t *d_classes, int iters, int bisections, float dev_th,
                   void *stream, bool direct2e, bool refits = true);
}  // namespace

extern "C" {

int qcs_fit_from_start_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p,
                              int n, const float *d_start, int iters, int bisections, float dev_th, void *stream) {
    return qcs_fit_from_start_classes_device(c, d_rois, d_wle, p, n, d_start, nullptr, iters, bisections, dev_th,
                                             stream);
}

int qcs_fit_from_start_classes_device(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle,
                                      const qcs_loc_para *p, int n, const float *d_start, const uint8_t *d_classes,
                                      int iters, int bisections, float dev_th, void *stream) {
    return fit_from_start(c, d_rois, d_wle, p, n, d_start, d_classes, iters, bisections, dev_th, stream, false);
}

}  // extern "C"

namespace {
// qcs_fit_from_start_classes_device; direct2e as in learned_multi (on for the
// network-driven calls)
int fit_from_start(qcs_loc_data *c, const uint16_t *d_rois, const float *d_wle, const qcs_loc_para *p, int n,
                   const float *d_start, const uint8_t *d_classes, int iters, int bisections, float dev_th,
                   void *stream, bool direct2e, bool refits) {
    int st = check_call(c, p, n);
    if (st) return st;
    const int kind = learned_kind(p);
    if (kind < 0) return fail(QCS_ERR_ARG, kLearnedShapes);
    if (d_classes && !p->MultiEmitterFitEn)
        return fail(QCS_ERR_ARG, "emitter-count classes need multi-emitter fitting");
    if (bisections <= 0) bisections = 11;
    if (!qcs::learned_schedule_supported(kind, p->ROISize, iters, bisections)) return fail(QCS_ERR_ARG, kLearnedSchedules);
    if (n == 0) return QCS_OK;
    if (!d_rois || !d_start) return fail(QCS_ERR_ARG, "null pointer");
    if (!(dev_th > 0.0f)) dev_th = default_dev_th(p->ROISize);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    const float *wle = d_wle;
    if (!wle) {
        QCS_CUDA(qcs::launch_wle_ctx(c->wle_sorter, d_rois, n, c->R, p->LocType, c->d_wle, s), "WLE pre-pass");
        wle = c->d_wle;
    }
    if (p->MultiEmitterFitEn) {
        QCS_CUDA(learned_multi(c, d_rois, wle, p, n, nullptr, d_start, d_classes, iters, bisections, dev_th, s,
                               direct2e),
                 "learned multi-emitter localization");
        return QCS_OK;
    }
    qcs::FitLaunch f;
    f.rois = d_rois;
    f.wle = wle;
    f.q = qcs::Queue{nullptr, nullptr, n};
    f.max_count = n;
    f.loc = c->d_loc;
    f.to2e = nullptr;
    f.mo = qcs::MultiOut{nullptr, nullptr};
    f.para = qcs::core_para(*p);
    f.stream = s;
    QCS_CUDA(qcs::launch_fit_learned(kind, p->ROISize, iters, bisections, f, d_start, dev_th, c->st.to2e),
             "start-point fit");
    if (!refits) {
        // the learned fits' results stand: no refit queue, the CRLB of every row
        QCS_CUDA(cudaMemsetAsync(c->st.counters + qcs::kCntSingle, 0, sizeof(int), s), "refit count");
        learned_counters_kernel<<<1, 1, 0, s>>>(c->st, n);
        QCS_CUDA(cudaGetLastError(), "counters");
        QCS_CUDA(qcs::launch_crlb(c->d_loc, nullptr, n, n, p->LocType, p->ReadNoise_e, p->QE, p->PixelSize, s),
                 "CRLB");
        return QCS_OK;
    }
    // plain refit of the flagged records
    QCS_CUDA(qcs::launch_flag_queue(c->st.to2e, n, c->st.q_single, c->st.counters + qcs::kCntSingle, s),
             "refit queue");
    // The plain refits (a short, latency-bound queue) and their CRLB run on
    // the high-priority side stream while the main stream computes the CRLB
    // of every other row; the two touch disjoint rows.
    QCS_CUDA(cudaEventRecord(c->ev_fork, s), "fork");
    QCS_CUDA(cudaStreamWaitEvent(c->side, c->ev_fork, 0), "fork");
    f.q = qcs::Queue{c->st.q_single, c->st.counters + qcs::kCntSingle, 0};
    f.stream = c->side;
    QCS_CUDA(qcs::launch_fit_group(kind, p->ROISize, 8, f), "plain refit");
    QCS_CUDA(qcs::launch_crlb(c->d_loc, c->st.counters + qcs::kCntSingle, 0, n, p->LocType, p->ReadNoise_e, p->QE,
                              p->PixelSize, c->side, c->st.q_single, nullptr),
             "refit CRLB");
    QCS_CUDA(cudaEventRecord(c->ev_join, c->side), "join");
    learned_counters_kernel<<<1, 1, 0, s>>>(c->st, n);
    QCS_CUDA(cudaGetLastError(), "counters");
    QCS_CUDA(qcs::launch_crlb(c->d_loc, nullptr, n, n, p->LocType, p->ReadNoise_e, p->QE, p->PixelSize, s, nullptr,
                              c->st.to2e),
             "CRLB");
    QCS_CUDA(cudaStreamWaitEvent(s, c->ev_join, 0), "join");
    return QCS_OK;
}
}  // namespace

extern "C" {

int qcs_learned_localize_device(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                                const qcs_loc_para *p, int n, int iters, int bisections, float dev_th, void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (learned_kind(p) < 0) return fail(QCS_ERR_ARG, kLearnedShapes);
    int lt = -1, rs = 0;
    qcs_learned_shape(net, &lt, &rs, nullptr);
    if (lt != p->LocType || rs != p->ROISize)
        return fail(QCS_ERR_ROISIZE, "the network was built for another localization type or ROI size");
    if (n == 0) return QCS_OK;
    if (!d_rois) return fail(QCS_ERR_ARG, "null ROI pointer");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    // emitter-count routing: multi-emitter fitting on and a threshold set
    uint8_t *cls = (p->MultiEmitterFitEn && qcs_learned_count_threshold(net) > 0.0f) ? c->d_cls : nullptr;
    QCS_CUDA(qcs::learned::start_points(net, p, d_rois, n, c->d_start, s, cls), "learned start points");
    qcs::TwoEmitterStart two;
    qcs::ThreeEmitterStart three;
    if (p->MultiEmitterFitEn && (st = multi_starts(c, net, p, d_rois, n, nullptr, s, &two, &three)) != QCS_OK)
        return st;
    st = fit_from_start(c, d_rois, d_wle, p, n, c->d_start, cls, iters, bisections, dev_th, s,
                        qcs::learned::direct_two_emitter(net), qcs::learned::single_refits(net));
    if (c->starts_ready && st != QCS_OK) cudaStreamWaitEvent(s, c->starts_ready, 0);  // joined on every path
    c->two = nullptr;
    c->three = nullptr;
    c->starts_ready = nullptr;
    return st;
}

int qcs_learned_localize_device_n(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                                  const qcs_loc_para *p, const int *d_n, int max_n, int iters, int bisections,
                                  float dev_th, void *stream) {
    int st = check_call(c, p, max_n);
    if (st) return st;
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (learned_kind(p) != qcs::kGS2D || !p->MultiEmitterFitEn)
        return fail(QCS_ERR_ARG, "device-count learned localization: GS2D 7/9/11 with multi-emitter fitting");
    int lt = -1, rs = 0;
    qcs_learned_shape(net, &lt, &rs, nullptr);
    if (lt != p->LocType || rs != p->ROISize)
        return fail(QCS_ERR_ROISIZE, "the network was built for another localization type or ROI size");
    if (!d_rois || !d_wle || !d_n) return fail(QCS_ERR_ARG, "null pointer");
    if (bisections <= 0) bisections = 11;
    if (!qcs::learned_schedule_supported(qcs::kGS2D, p->ROISize, iters, bisections))
        return fail(QCS_ERR_ARG, kLearnedSchedules);
    if (!(dev_th > 0.0f)) dev_th = default_dev_th(p->ROISize);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    uint8_t *cls = qcs_learned_count_threshold(net) > 0.0f ? c->d_cls : nullptr;
    if (max_n == 0) return QCS_OK;
    QCS_CUDA(qcs::learned::start_points(net, p, d_rois, max_n, c->d_start, s, cls, d_n), "learned start points");
    qcs::TwoEmitterStart two;
    qcs::ThreeEmitterStart three;
    if ((st = multi_starts(c, net, p, d_rois, max_n, d_n, s, &two, &three)) != QCS_OK) return st;
    const cudaError_t e =
        learned_multi(c, d_rois, d_wle, p, max_n, d_n, c->d_start, cls, iters, bisections, dev_th, s,
                      qcs::learned::direct_two_emitter(net));
    if (c->starts_ready && e != cudaSuccess) cudaStreamWaitEvent(s, c->starts_ready, 0);  // joined on every path
    c->two = nullptr;
    c->three = nullptr;
    c->starts_ready = nullptr;
    QCS_CUDA(e, "learned multi-emitter localization");
    return QCS_OK;
}

int qcs_learned_refit_num(qcs_loc_data *c, int *n) {
    if (!c || !n) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaDeviceSynchronize(), "localization");
    QCS_CUDA(cudaMemcpy(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost),
             "read counters");
    *n = c->h_counters[qcs::kCntRefit];
    return QCS_OK;
}

int qcs_loc_count_labels_device(qcs_loc_data *c, int n, float *d_labels, void *stream) {
    if (!c || !d_labels) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0 || n > c->capacity) return fail(QCS_ERR_CAPACITY, "record count outside the context capacity");
    if (n == 0) return QCS_OK;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    labels_zero_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_labels, n);
    labels_2e_kernel<<<(n + 255) / 256, 256, 0, s>>>(c->st, n, d_labels);
    QCS_CUDA(cudaGetLastError(), "count labels");
    return QCS_OK;
}

int qcs_learned_refit_2e_num(qcs_loc_data *c, int *n) {
    if (!c || !n) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaDeviceSynchronize(), "localization");
    QCS_CUDA(cudaMemcpy(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost),
             "read counters");
    *n = c->h_counters[qcs::kCntRefit2E];
    return QCS_OK;
}

int qcs_learned_refit_3e_num(qcs_loc_data *c, int *n) {
    if (!c || !n) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaDeviceSynchronize(), "localization");
    QCS_CUDA(cudaMemcpy(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost),
             "read counters");
    *n = c->h_counters[qcs::kCntRefit3E];
    return QCS_OK;
}

int qcs_loc_set_three_emitter_capture(qcs_loc_data *c, int on) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (on) {
        const int st = ensure_three(c);
        if (st) return st;
    }
    c->capture3 = on ? 1 : 0;
    return QCS_OK;
}

const float *qcs_loc_device_three_emitter_params(const qcs_loc_data *c) { return c ? c->d_params3 : nullptr; }

int qcs_loc_three_emitter_targets_device(qcs_loc_data *c, const uint16_t *d_rois, const qcs_loc_para *p, int n,
                                         const float *d_scale, float *d_targets, float *d_valid, void *stream) {
    if (!c || !p || !d_rois || !d_scale || !d_targets || !d_valid) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0 || n > c->capacity) return fail(QCS_ERR_CAPACITY, "record count outside the context capacity");
    if (p->LocType != QCS_LOCTYPE_GS2D || !p->MultiEmitterFitEn || p->ROISize != c->R ||
        !(c->R == 7 || c->R == 9 || c->R == 11))
        return fail(QCS_ERR_ARG, "three-emitter targets: GS2D 7/9/11 with multi-emitter fitting");
    if (!c->capture3 || !c->d_params3)
        return fail(QCS_ERR_STATE, "three-emitter targets: set qcs_loc_set_three_emitter_capture before the plain call");
    if (n == 0) return QCS_OK;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(cudaMemsetAsync(d_targets, 0, (size_t)n * 11 * sizeof(float), s), "clear targets");
    QCS_CUDA(cudaMemsetAsync(d_valid, 0, (size_t)n * sizeof(float), s), "clear valid");
    const int grid = (n + 255) / 256;
    if (c->R == 7)
        three_targets_kernel<7><<<grid, 256, 0, s>>>(c->st, c->d_params3, d_scale, n, d_targets, d_valid);
    else if (c->R == 9)
        three_targets_kernel<9><<<grid, 256, 0, s>>>(c->st, c->d_params3, d_scale, n, d_targets, d_valid);
    else
        three_targets_kernel<11><<<grid, 256, 0, s>>>(c->st, c->d_params3, d_scale, n, d_targets, d_valid);
    QCS_CUDA(cudaGetLastError(), "three-emitter targets");
    return QCS_OK;
}

int qcs_loc_two_emitter_targets_device(qcs_loc_data *c, const uint16_t *d_rois, const qcs_loc_para *p, int n,
                                       const float *d_scale, float *d_targets, float *d_valid, void *stream) {
    if (!c || !p || !d_rois || !d_scale || !d_targets || !d_valid) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0 || n > c->capacity) return fail(QCS_ERR_CAPACITY, "record count outside the context capacity");
    if (p->LocType != QCS_LOCTYPE_GS2D || !p->MultiEmitterFitEn || p->ROISize != c->R ||
        !(c->R == 7 || c->R == 9 || c->R == 11))
        return fail(QCS_ERR_ARG, "two-emitter targets: GS2D 7/9/11 with multi-emitter fitting");
    if (n == 0) return QCS_OK;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(cudaMemsetAsync(d_targets, 0, (size_t)n * 8 * sizeof(float), s), "clear targets");
    QCS_CUDA(cudaMemsetAsync(d_valid, 0, (size_t)n * sizeof(float), s), "clear valid");
    const int grid = (n + 255) / 256;
    const float qe = p->QE;
    if (c->R == 7)
        two_targets_kernel<7><<<grid, 256, 0, s>>>(c->st, d_rois, c->d_loc, d_scale, n, qe, d_targets, d_valid);
    else if (c->R == 9)
        two_targets_kernel<9><<<grid, 256, 0, s>>>(c->st, d_rois, c->d_loc, d_scale, n, qe, d_targets, d_valid);
    else
        two_targets_kernel<11><<<grid, 256, 0, s>>>(c->st, d_rois, c->d_loc, d_scale, n, qe, d_targets, d_valid);
    QCS_CUDA(cudaGetLastError(), "two-emitter targets");
    return QCS_OK;
}

const float *qcs_loc_device_rows(const qcs_loc_data *c) { return c ? c->d_loc : nullptr; }
const int *qcs_loc_device_valid_num(const qcs_loc_data *c) { return c ? c->st.counters + qcs::kCntValid : nullptr; }
uint16_t *qcs_loc_device_roi_buffer(qcs_loc_data *c) { return c ? c->d_rois : nullptr; }
float *qcs_loc_device_wle_buffer(qcs_loc_data *c) { return c ? c->d_wle : nullptr; }

static void compute_ratios(qcs_loc_data *c, const qcs_loc_para *p, int n) {
    const int *k = c->h_counters;
    const float div = (float)(n < 1 ? 1 : n);
    for (int i = 0; i < 7; ++i) c->ratios[i] = 0;
    if (n <= 0) return;
    const int single = k[qcs::kCntSingle];
    c->ratios[0] = (float)single / div;
    c->ratios[3] = (float)single / div;
    if (c->lr_stats) {
        // every record fitted with one, two and three emitters; the final
        // ratios are the models the likelihood-ratio test kept
        c->ratios[1] = c->ratios[2] = c->ratios[0];
        c->ratios[3] = (float)k[qcs::kCntSel1] / div;
        c->ratios[4] = (float)k[qcs::kCntSel2] / div;
        c->ratios[5] = (float)k[qcs::kCntSel3] / div;
        c->ratios[6] = (float)k[qcs::kCntRejected] / div;
        return;
    }
    if (p->MultiEmitterFitEn) {
        const int n2 = k[qcs::kCnt2E], n2c = k[qcs::kCnt2EClassify], n3 = k[qcs::kCnt3E], rej = k[qcs::kCntRejected];
        const int n3c = k[qcs::kCnt3EClassify];  // learned classes only: records sent straight to 3E
        c->ratios[1] = (float)n2 / div;
        c->ratios[2] = (float)n3 / div;
        c->ratios[3] = (float)(single - (n2 - n2c)) / div;
        if (p->LocType == QCS_LOCTYPE_GS2D) {
            c->ratios[4] = (float)(n2 - (n3 - n3c)) / div;
            c->ratios[5] = (float)(n3 - rej) / div;
        } else {
            c->ratios[4] = (float)(n2 - rej) / div;
        }
        c->ratios[6] = (float)rej / div;
    }
}

int qcs_loc_bfgs_mle_localization(qcs_loc_data *c, const uint16_t *h_rois, const float *h_wle,
                                  const qcs_loc_para *p, int n, void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    c->valid = 0;
    for (int i = 0; i < 7; ++i) c->ratios[i] = 0;
    if (n == 0) return QCS_OK;
    if (!h_rois) return fail(QCS_ERR_ARG, "null ROI pointer");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(cudaMemcpyAsync(c->d_rois, h_rois, (size_t)n * c->whole * sizeof(uint16_t), cudaMemcpyHostToDevice, s),
             "copy ROI records");
    if (h_wle)
        QCS_CUDA(cudaMemcpyAsync(c->d_wle, h_wle, (size_t)n * QCS_WLE_PARA_NUM * sizeof(float),
                                 cudaMemcpyHostToDevice, s),
                 "copy WLE records");
    st = qcs_loc_localize_device(c, c->d_rois, h_wle ? c->d_wle : nullptr, p, n, s);
    if (st) return st;
    QCS_CUDA(cudaMemcpyAsync(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost, s),
             "read counters");
    // without multi-emitter fitting every record has its row (zero when rejected): the n rows come back with the
    // counters, one wait; with it the row count is read first
    const bool one_pass = !p->MultiEmitterFitEn && !use_lr(c, p) && n <= c->max_rows;
    if (one_pass)
        QCS_CUDA(cudaMemcpyAsync(c->h_loc, c->d_loc, (size_t)n * QCS_OUT_PARA_NUM * sizeof(float),
                                 cudaMemcpyDeviceToHost, s),
                 "read localizations");
    QCS_CUDA(cudaStreamSynchronize(s), "localization");
    const int rows = c->h_counters[qcs::kCntValid];
    if (!one_pass && rows > 0) {
        QCS_CUDA(cudaMemcpyAsync(c->h_loc, c->d_loc, (size_t)rows * QCS_OUT_PARA_NUM * sizeof(float),
                                 cudaMemcpyDeviceToHost, s),
                 "read localizations");
        QCS_CUDA(cudaStreamSynchronize(s), "read localizations");
    }
    c->valid = rows;
    compute_ratios(c, p, n);
    return QCS_OK;
}

}  // extern "C"

// Host records in, rows and counters out, on stream s, without waiting:
// device_call runs the localization of the records copied to c->d_rois.
template <class F>
static int enqueue_host_call(qcs_loc_data *c, const uint16_t *h_rois, const float *h_wle, const qcs_loc_para *p,
                             int n, cudaStream_t s, F device_call) {
    if (c->pending) return fail(QCS_ERR_ARG, "the previous asynchronous call awaits qcs_loc_finish");
    c->valid = 0;
    for (int i = 0; i < 7; ++i) c->ratios[i] = 0;
    c->pending_n = n;
    if (n > 0) {
        if (!h_rois) return fail(QCS_ERR_ARG, "null ROI pointer");
        QCS_CUDA(cudaMemcpyAsync(c->d_rois, h_rois, (size_t)n * c->whole * sizeof(uint16_t), cudaMemcpyHostToDevice,
                                 s),
                 "copy ROI records");
        if (h_wle)
            QCS_CUDA(cudaMemcpyAsync(c->d_wle, h_wle, (size_t)n * QCS_WLE_PARA_NUM * sizeof(float),
                                     cudaMemcpyHostToDevice, s),
                     "copy WLE records");
        int st = device_call(h_wle ? c->d_wle : nullptr);
        if (st) return st;
        // rows: one per record, then at most two appended emitters per record
        const long long most = p->MultiEmitterFitEn ? 3ll * n : (long long)n;
        const int rows = (int)(most < c->max_rows ? most : c->max_rows);
        QCS_CUDA(cudaMemcpyAsync(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost,
                                 s),
                 "read counters");
        QCS_CUDA(cudaMemcpyAsync(c->h_loc, c->d_loc, (size_t)rows * QCS_OUT_PARA_NUM * sizeof(float),
                                 cudaMemcpyDeviceToHost, s),
                 "read localizations");
    }
    QCS_CUDA(cudaEventRecord(c->ev_done, s), "record completion");
    c->pending = 1;
    return QCS_OK;
}

extern "C" {

int qcs_loc_localize_async(qcs_loc_data *c, const uint16_t *h_rois, const float *h_wle, const qcs_loc_para *p, int n,
                           void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return enqueue_host_call(c, h_rois, h_wle, p, n, s, [&](const float *d_wle) {
        return qcs_loc_localize_device(c, c->d_rois, d_wle, p, n, s);
    });
}

int qcs_learned_localize_async(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *h_rois, const float *h_wle,
                               const qcs_loc_para *p, int n, int iters, int bisections, float dev_th,
                               void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    if (!net) return fail(QCS_ERR_ARG, "null network");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return enqueue_host_call(c, h_rois, h_wle, p, n, s, [&](const float *d_wle) {
        return qcs_learned_localize_device(c, net, c->d_rois, d_wle, p, n, iters, bisections, dev_th, s);
    });
}

int qcs_loc_finish(qcs_loc_data *c, const qcs_loc_para *p) {
    if (!c || !p) return fail(QCS_ERR_ARG, "null argument");
    if (!c->pending) return fail(QCS_ERR_ARG, "no asynchronous call to finish");
    c->pending = 0;
    QCS_CUDA(cudaEventSynchronize(c->ev_done), "localization");
    if (c->pending_n == 0) return QCS_OK;
    c->valid = c->h_counters[qcs::kCntValid];
    compute_ratios(c, p, c->pending_n);
    return QCS_OK;
}

int qcs_loc_read_rows(qcs_loc_data *c, const qcs_loc_para *p, void *stream) {
    if (!c || !p) return fail(QCS_ERR_ARG, "null argument");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(cudaMemcpyAsync(c->h_counters, c->st.counters, qcs::kCntNum * sizeof(int), cudaMemcpyDeviceToHost, s),
             "read counters");
    QCS_CUDA(cudaStreamSynchronize(s), "localization");
    const int rows = c->h_counters[qcs::kCntValid];
    if (rows > 0)
        QCS_CUDA(cudaMemcpyAsync(c->h_loc, c->d_loc, (size_t)rows * QCS_OUT_PARA_NUM * sizeof(float),
                                 cudaMemcpyDeviceToHost, s),
                 "read localizations");
    QCS_CUDA(cudaStreamSynchronize(s), "read localizations");
    c->valid = rows;
    // records of the call: single-emitter queue plus the classifier's 2E and 3E entries
    const int n = c->h_counters[qcs::kCntSingle] +
                  (p->MultiEmitterFitEn ? c->h_counters[qcs::kCnt2EClassify] + c->h_counters[qcs::kCnt3EClassify] : 0);
    compute_ratios(c, p, n);
    return QCS_OK;
}

int qcs_learned_autotune(qcs_loc_data *c, qcs_learned_net *net, const uint16_t *d_rois, const float *d_wle,
                         const qcs_loc_para *p, int n, int *iters, int *bisections, void *stream) {
    if (!iters || !bisections) return fail(QCS_ERR_ARG, "null output");
    int st = check_call(c, p, n);
    if (st) return st;
    if (!net || !d_rois) return fail(QCS_ERR_ARG, "null argument");
    if (n < 64) return fail(QCS_ERR_ARG, "autotuning needs at least 64 records");
    const int kind = learned_kind(p);
    if (kind < 0) return fail(QCS_ERR_ARG, kLearnedShapes);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    // every schedule compiled for the shape; the fastest whose acceptance stays within 0.5 points of the
    // best schedule's (refits and rejected fits are what a too-short schedule costs)
    const int sched[][2] = {{2, 4}, {2, 6}, {2, 8}, {3, 4}, {3, 6}, {3, 8}, {4, 6}, {2, 11}, {3, 11}, {4, 11}, {5, 11},
                            {8, 11}};
    float ms[12] = {0};
    double acc[12] = {0};
    bool ran[12] = {false};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    QCS_CUDA(cudaEventCreate(&e0), "tuning events");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(QCS_ERR_CUDA, "tuning events");
    }
    int rc = QCS_OK;
    for (int i = 0; i < 12 && rc == QCS_OK; ++i) {
        const int it = sched[i][0], nb = sched[i][1];
        if (!qcs::learned_schedule_supported(kind, p->ROISize, it, nb)) continue;
        rc = qcs_learned_localize_device(c, net, d_rois, d_wle, p, n, it, nb, 0.0f, s);  // warm-up
        if (rc == QCS_OK && cudaEventRecord(e0, s) != cudaSuccess) rc = fail(QCS_ERR_CUDA, "tuning");
        for (int r = 0; r < 2 && rc == QCS_OK; ++r)
            rc = qcs_learned_localize_device(c, net, d_rois, d_wle, p, n, it, nb, 0.0f, s);
        if (rc == QCS_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                             cudaEventElapsedTime(&ms[i], e0, e1) != cudaSuccess))
            rc = fail(QCS_ERR_CUDA, "tuning");
        if (rc == QCS_OK) rc = qcs_loc_read_rows(c, p, s);
        if (rc == QCS_OK) {
            long kept = 0;
            for (int r = 0; r < c->valid; ++r) kept += c->h_loc[(size_t)r * QCS_OUT_PARA_NUM] > 0.0f;
            acc[i] = (double)kept / n;
            ran[i] = true;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != QCS_OK) return rc;
    double best_acc = 0;
    for (int i = 0; i < 12; ++i)
        if (ran[i] && acc[i] > best_acc) best_acc = acc[i];
    int pick = -1;
    for (int i = 0; i < 12; ++i)
        if (ran[i] && acc[i] >= best_acc - 0.005 && (pick < 0 || ms[i] < ms[pick])) pick = i;
    if (pick < 0) return fail(QCS_ERR_ARG, kLearnedSchedules);
    *iters = sched[pick][0];
    *bisections = sched[pick][1];
    return QCS_OK;
}

const float *qcs_loc_h_loc_arry(const qcs_loc_data *c) { return c ? c->h_loc : nullptr; }
int qcs_loc_valid_num(const qcs_loc_data *c) { return c ? c->valid : 0; }

int qcs_loc_fit_ratios(const qcs_loc_data *c, float *out7) {
    if (!c || !out7) return fail(QCS_ERR_ARG, "null argument");
    for (int i = 0; i < 7; ++i) out7[i] = c->ratios[i];
    return QCS_OK;
}

int qcs_wle_estimate(qcs_loc_data *c, const uint16_t *h_rois, int n, const qcs_loc_para *p, float *h_wle) {
    int st = check_call(c, p, n);
    if (st) return st;
    if (n == 0) return QCS_OK;
    if (!h_rois || !h_wle) return fail(QCS_ERR_ARG, "null pointer");
    cudaStream_t s = c->stream;
    QCS_CUDA(cudaMemcpyAsync(c->d_rois, h_rois, (size_t)n * c->whole * sizeof(uint16_t), cudaMemcpyHostToDevice, s),
             "copy ROI records");
    QCS_CUDA(qcs::launch_wle_ctx(c->wle_sorter, c->d_rois, n, c->R, p->LocType, c->d_wle, s), "WLE pre-pass");
    QCS_CUDA(cudaMemcpyAsync(h_wle, c->d_wle, (size_t)n * QCS_WLE_PARA_NUM * sizeof(float), cudaMemcpyDeviceToHost, s),
             "read WLE records");
    QCS_CUDA(cudaStreamSynchronize(s), "WLE pre-pass");
    return QCS_OK;
}

int qcs_wle_estimate_device(qcs_loc_data *c, const uint16_t *d_rois, int n, const qcs_loc_para *p, float *d_wle,
                            void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    if (n == 0) return QCS_OK;
    if (!d_rois || !d_wle) return fail(QCS_ERR_ARG, "null pointer");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(qcs::launch_wle_ctx(c->wle_sorter, d_rois, n, c->R, p->LocType, d_wle, s), "WLE pre-pass");
    return QCS_OK;
}

int qcs_fit_single_device(int loc_type, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n,
                          float *d_loc, void *stream) {
    int st = check_para(p, false);
    if (st) return st;
    if (n < 0) return fail(QCS_ERR_ARG, "negative ROI count");
    if (n == 0) return QCS_OK;
    if (!d_rois || !d_wle || !d_loc) return fail(QCS_ERR_ARG, "null pointer");
    qcs::FitLaunch f;
    f.rois = d_rois;
    f.wle = d_wle;
    f.q = qcs::Queue{nullptr, nullptr, n};
    f.max_count = n;
    f.loc = d_loc;
    f.to2e = nullptr;
    f.mo = qcs::MultiOut{nullptr, nullptr};
    qcs_loc_para q = *p;
    q.MultiEmitterFitEn = 0;
    f.para = qcs::core_para(q);
    f.stream = static_cast<cudaStream_t>(stream);
    QCS_CUDA(qcs::launch_fit(loc_type == QCS_LOCTYPE_AS3D ? qcs::kAS3D : qcs::kGS2D, p->ROISize, f), "fit launch");
    return QCS_OK;
}

int qcs_fit_single_group_device(int loc_type, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle,
                                int n, float *d_loc, int lanes, void *stream) {
    int st = check_para(p, false);
    if (st) return st;
    if (n < 0) return fail(QCS_ERR_ARG, "negative ROI count");
    const int kind = loc_type == QCS_LOCTYPE_AS3D ? qcs::kAS3D : qcs::kGS2D;
    if (!qcs::group_fit_supported(kind, p->ROISize))
        return fail(QCS_ERR_ARG, "group fit: GS2D 7/9/11/13 or AS3D 7/9/11 ROIs");
    if (lanes != 8 && !((lanes == 4 || lanes == 16) && kind == qcs::kGS2D && p->ROISize == 7))
        return fail(QCS_ERR_ARG, "lanes per ROI: 8, or 4 / 16 for GS2D 7x7");
    if (n == 0) return QCS_OK;
    if (!d_rois || !d_wle || !d_loc) return fail(QCS_ERR_ARG, "null pointer");
    qcs::FitLaunch f;
    f.rois = d_rois;
    f.wle = d_wle;
    f.q = qcs::Queue{nullptr, nullptr, n};
    f.max_count = n;
    f.loc = d_loc;
    f.to2e = nullptr;
    f.mo = qcs::MultiOut{nullptr, nullptr};
    qcs_loc_para q = *p;
    q.MultiEmitterFitEn = 0;
    f.para = qcs::core_para(q);
    f.stream = static_cast<cudaStream_t>(stream);
    QCS_CUDA(qcs::launch_fit_group(kind, p->ROISize, lanes, f), "group fit launch");
    return QCS_OK;
}

int qcs_loc_autotune(qcs_loc_data *c, const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n,
                     void *stream) {
    int st = check_call(c, p, n);
    if (st) return st;
    if (!d_rois || !d_wle) return fail(QCS_ERR_ARG, "null pointer");
    if (n < 64) return fail(QCS_ERR_ARG, "autotuning needs at least 64 records");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    const int kind = p->LocType == QCS_LOCTYPE_AS3D ? qcs::kAS3D : qcs::kGS2D;
    c->tune_count = 0;
    c->tune_limit2 = c->tune_limit3 = 0;
    // the single-emitter lanes exist for the sizes with a lane-group kernel; the multi-emitter stages for GS2D
    // and AS3D calls with multi-emitter fitting (DH3D has no two-emitter stage)
    const bool single_ok = qcs::group_fit_supported(kind, p->ROISize) && p->LocType != QCS_LOCTYPE_DH3D;
    const bool multi_ok = p->MultiEmitterFitEn && p->LocType != QCS_LOCTYPE_DH3D;
    if (!single_ok && !multi_ok) return QCS_OK;
    // lanes per ROI to try: 1 (one thread per ROI) and 8; 4 and 16 exist for GS2D 7x7 only
    const int cand7[4] = {1, 4, 8, 16}, cand_other[2] = {1, 8};
    const bool gs7 = kind == qcs::kGS2D && p->ROISize == 7;
    const int *cand = gs7 ? cand7 : cand_other;
    const int ncand = gs7 ? 4 : 2;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    QCS_CUDA(cudaEventCreate(&e0), "tuning events");
    cudaError_t e = cudaEventCreate(&e1);
    qcs_loc_para q = *p;
    q.MultiEmitterFitEn = 0;
    qcs::FitLaunch f;
    f.rois = d_rois;
    f.wle = d_wle;
    f.loc = c->d_loc;
    f.to2e = nullptr;
    f.mo = qcs::MultiOut{nullptr, nullptr};
    f.para = qcs::core_para(q);
    f.stream = s;
    int sizes[8], k = 0;
    if (single_ok) {
        for (int m = 256; m < n && k < 7; m *= 4) sizes[k++] = m;
        sizes[k++] = n;
    }
    for (int i = 0; i < k && e == cudaSuccess; ++i) {
        const int m = sizes[i];
        f.q = qcs::Queue{nullptr, nullptr, m};
        f.max_count = m;
        float best = 1e30f;
        int best_lanes = 1;
        for (int j = 0; j < ncand && e == cudaSuccess; ++j) {
            const int lanes = cand[j];
            auto run = [&]() {
                return lanes == 1 ? qcs::launch_fit(kind, p->ROISize, f) : qcs::launch_fit_group(kind, p->ROISize, lanes, f);
            };
            e = run();  // warm-up
            if (e == cudaSuccess) e = cudaEventRecord(e0, s);
            for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = run();
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms < best) {
                best = ms;
                best_lanes = lanes;
            }
        }
        c->tune_n[i] = m;  // batches above the largest tuned size keep one thread per ROI
        c->tune_lanes[i] = best_lanes;
    }
    // Multi-emitter stages: the longest queue for which the lane-group kernel beats one thread per ROI,
    // timed on queues of the caller's first m records (the rows are the same either way).
    if (e == cudaSuccess && multi_ok) {
        const int kinds[2] = {p->LocType == QCS_LOCTYPE_AS3D ? qcs::kAS3D2E : qcs::k2E,
                              p->LocType == QCS_LOCTYPE_GS2D ? qcs::k3E : -1};
        int *limits[2] = {&c->tune_limit2, &c->tune_limit3};
        qcs::FitLaunch g;
        g.rois = d_rois;
        g.wle = d_wle;
        g.loc = c->d_loc;
        g.to2e = nullptr;
        g.mo = qcs::MultiOut{c->st.res2, c->st.extra2};
        g.para = qcs::core_para(*p);
        g.stream = s;
        for (int st2 = 0; st2 < 2 && e == cudaSuccess; ++st2) {
            const int kind2 = kinds[st2];
            *limits[st2] = 0;
            if (kind2 < 0 || !qcs::multi_group_available(kind2, p->ROISize)) continue;
            int limit = 0;
            bool group_wins_all = true;
            for (int m = 64; e == cudaSuccess; m *= 2) {
                const int mm = m < n ? m : n;
                g.q = qcs::Queue{nullptr, nullptr, mm};
                g.max_count = mm;
                float t[2] = {0, 0};
                for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
                    g.thread_per_roi = mode;           // 0: lane groups for any length, 1: one thread per ROI
                    g.group_limit = mode ? 0 : (1 << 30);
                    e = qcs::launch_fit(kind2, p->ROISize, g);  // warm-up
                    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
                    for (int r = 0; r < 2 && e == cudaSuccess; ++r) e = qcs::launch_fit(kind2, p->ROISize, g);
                    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&t[mode], e0, e1);
                }
                if (t[0] < t[1])
                    limit = mm;
                else
                    group_wins_all = false;
                if (!group_wins_all || mm == n) break;
            }
            // lane groups still ahead at the largest queue tried: keep the larger of it and the default
            if (group_wins_all) {
                const int d = qcs::multi_group_default_limit(kind2, p->ROISize);
                limit = limit > d ? limit : d;
            }
            *limits[st2] = limit > 0 ? limit : -1;  // -1: always one thread per ROI
        }
    }
    if (e1) cudaEventDestroy(e1);
    cudaEventDestroy(e0);
    if (e != cudaSuccess) {
        c->tune_count = 0;
        c->tune_limit2 = c->tune_limit3 = 0;
        return fail(QCS_ERR_CUDA, "autotuning", e);
    }
    c->tune_count = k;
    return QCS_OK;
}

// the current GPU's name with blanks as underscores (the cache's tag)
static std::string gpu_tag() {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    std::string name(prop.name);
    for (char &ch : name)
        if (ch == ' ' || ch == '\t' || ch == '\n') ch = '_';
    return name;
}

int qcs_loc_save_tuning(const qcs_loc_data *c, const char *path) {
    if (!c || !path) return fail(QCS_ERR_ARG, "null argument");
    FILE *f = fopen(path, "w");
    if (!f) return fail(QCS_ERR_ARG, "cannot open the tuning file for writing");
    fprintf(f, "qcstorm_b200_tuning 1\ngpu %s\nroi_size %d\nloc_type %d\nmulti %d\nlanes %d", gpu_tag().c_str(),
            c->para.ROISize, c->para.LocType, c->para.MultiEmitterFitEn, c->tune_count);
    for (int i = 0; i < c->tune_count; ++i) fprintf(f, " %d %d", c->tune_n[i], c->tune_lanes[i]);
    fprintf(f, "\nlimits %d %d\n", c->tune_limit2, c->tune_limit3);
    const bool ok = fclose(f) == 0;
    return ok ? QCS_OK : fail(QCS_ERR_ARG, "writing the tuning file failed");
}

int qcs_loc_load_tuning(qcs_loc_data *c, const char *path) {
    if (!c || !path) return fail(QCS_ERR_ARG, "null argument");
    FILE *f = fopen(path, "r");
    if (!f) return fail(QCS_ERR_ARG, "cannot open the tuning file");
    char gpu[256] = {0};
    int version = 0, R = 0, lt = 0, multi = 0, count = 0, sizes[8], lanes[8], l2 = 0, l3 = 0;
    bool ok = fscanf(f, " qcstorm_b200_tuning %d gpu %255s roi_size %d loc_type %d multi %d lanes %d", &version, gpu,
                     &R, &lt, &multi, &count) == 6 &&
              version == 1 && count >= 0 && count <= 8;
    for (int i = 0; ok && i < count; ++i) ok = fscanf(f, " %d %d", &sizes[i], &lanes[i]) == 2;
    ok = ok && fscanf(f, " limits %d %d", &l2, &l3) == 2;
    fclose(f);
    if (!ok) return fail(QCS_ERR_ARG, "not a tuning file");
    if (gpu_tag() != gpu || R != c->para.ROISize || lt != c->para.LocType || multi != c->para.MultiEmitterFitEn)
        return fail(QCS_ERR_STATE, "the tuning file was written for another GPU model or ROI shape");
    int st = qcs_loc_set_tuning(c, sizes, lanes, count);
    if (st) return st;
    return qcs_loc_set_tuning_multi(c, l2, l3);
}

int qcs_loc_tuning_multi(const qcs_loc_data *c, int *limit_2e, int *limit_3e) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (limit_2e) *limit_2e = c->tune_limit2;
    if (limit_3e) *limit_3e = c->tune_limit3;
    return QCS_OK;
}

int qcs_loc_set_tuning_multi(qcs_loc_data *c, int limit_2e, int limit_3e) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (limit_2e < -1 || limit_3e < -1) return fail(QCS_ERR_ARG, "limits: -1 (one thread per ROI), 0 (default) or > 0");
    c->tune_limit2 = limit_2e;
    c->tune_limit3 = limit_3e;
    return QCS_OK;
}

int qcs_loc_tuning(const qcs_loc_data *c, int *sizes, int *lanes, int max_entries) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    for (int i = 0; i < c->tune_count && i < max_entries; ++i) {
        if (sizes) sizes[i] = c->tune_n[i];
        if (lanes) lanes[i] = c->tune_lanes[i];
    }
    return c->tune_count;
}

int qcs_loc_set_tuning(qcs_loc_data *c, const int *sizes, const int *lanes, int count) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (count < 0 || count > 8 || (count > 0 && (!sizes || !lanes))) return fail(QCS_ERR_ARG, "0..8 entries");
    for (int i = 0; i < count; ++i)
        if (lanes[i] != 1 && lanes[i] != 4 && lanes[i] != 8 && lanes[i] != 16)
            return fail(QCS_ERR_ARG, "lanes per ROI: 1, 4, 8 or 16");
    for (int i = 0; i < count; ++i) {
        c->tune_n[i] = sizes[i];
        c->tune_lanes[i] = lanes[i];
    }
    c->tune_count = count;
    return QCS_OK;
}

int qcs_loc_set_model_selection(qcs_loc_data *c, int mode, float threshold) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (mode != QCS_SELECT_CASCADE && mode != QCS_SELECT_LR)
        return fail(QCS_ERR_ARG, "mode: QCS_SELECT_CASCADE or QCS_SELECT_LR");
    if (threshold < 0.0f || threshold != threshold) return fail(QCS_ERR_ARG, "threshold must be >= 0");
    if (c->pending) return fail(QCS_ERR_STATE, "an asynchronous call on this context awaits qcs_loc_finish");
    if (mode == QCS_SELECT_LR && !c->d_lr) {
        const size_t cap = (size_t)c->capacity;
        const size_t bytes = 2 * cap * 12 * sizeof(float) + 3 * cap * sizeof(double);
        QCS_CUDA(cudaMalloc(&c->d_lr, bytes > 0 ? bytes : 16), "likelihood-ratio scratch");
    }
    c->sel_mode = mode;
    c->sel_th = threshold > 0.0f ? threshold : QCS_SELECT_LR_DEFAULT_TH;
    return QCS_OK;
}

int qcs_loc_model_selection(const qcs_loc_data *c, int *mode, float *threshold) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (mode) *mode = c->sel_mode;
    if (threshold) *threshold = c->sel_th;
    return QCS_OK;
}

int qcs_crlb_device(const qcs_loc_para *p, float *d_loc, int n, void *stream) {
    if (!p) return fail(QCS_ERR_ARG, "null parameter struct");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n == 0) return QCS_OK;
    if (!d_loc) return fail(QCS_ERR_ARG, "null pointer");
    QCS_CUDA(qcs::launch_crlb(d_loc, nullptr, n, n, p->LocType, p->ReadNoise_e, p->QE, p->PixelSize,
                              static_cast<cudaStream_t>(stream)),
             "CRLB launch");
    return QCS_OK;
}

}  // extern "C"
