// Allocation-free localization: the whole cascade of qcs_loc_localize_device
// (classify, single-emitter fit, 2E/3E fits, CRLB) for callers that cannot
// allocate device memory.
//
// Who needs it: a caller that records the localization into a CUDA graph
// while its stream is being captured (cudaMalloc is not allowed during
// capture), a host that owns all device memory through its own pool and
// forbids raw cudaMalloc in plug-ins, and a camera-rate acquisition loop that
// cannot afford the implicit device synchronisation of cudaMalloc/cudaFree in
// the middle of a frame stream.  Such a caller allocates its input records,
// WLE rows and output rows once, up front, and calls this entry point, which
// allocates nothing: its queues, per-slot results and counters live in one
// file-scope device array of fixed size.
//
// Limits and rules:
//   * at most QCS_NOALLOC_MAX_ROIS records per call (larger n: QCS_ERR_CAPACITY);
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is kept per device together with
//     the CUDA context it was looked up in; after a device reset (a new
//     primary context) the next call looks it up again, so that call must
//     also come before any capture;
//   * every call on a device shares the one array, which keeps the previous
//     call's contents: calls that overlap on the GPU (different streams, no
//     ordering between them) race on it and must not be issued;
//   * nothing in the array needs to start at zero: each call's first kernel
//     writes the counters, and every queue entry and per-slot result is
//     written before it is read in the same call.
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <cuda.h>  // CUcontext / CUresult types only; the entry point is fetched through the runtime
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_cascade.h"

namespace {

constexpr size_t kMax = QCS_NOALLOC_MAX_ROIS;
constexpr size_t kAlign = 256;
constexpr size_t al(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
// q_single, q2, q3 | to2e, res2, res3 | extra2, extra3 | counters | compaction tile counts
constexpr size_t kOffQ = 0;
constexpr size_t kOffFlags = kOffQ + 3 * al(kMax * sizeof(int));
constexpr size_t kOffExtra = kOffFlags + 3 * al(kMax);
constexpr size_t kOffCounters = kOffExtra + 2 * al(kMax * 12 * sizeof(float));
constexpr size_t kOffScan = kOffCounters + al(qcs::kCntNum * sizeof(int));
constexpr size_t kScratchBytes = kOffScan + al(qcs::cascade_scan_ints((int)kMax) * sizeof(int));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};  // context each address was looked up in

// The calling thread's current CUDA context (the library links only the
// runtime, so the driver's cuCtxGetCurrent is fetched through it once).
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
bool current_context(CUcontext *ctx) {
    static CtxGetCurrentFn fn = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
        looked_up = true;
    }
    *ctx = nullptr;
    return fn && fn(ctx) == CUDA_SUCCESS && *ctx;
}

// Status codes carry the error (QCS_ERR_*); the message is kept for debuggers.
thread_local char g_msg[160];

int noalloc_fail(int code, const char *msg) {
    snprintf(g_msg, sizeof(g_msg), "%s", msg);
    return code;
}

}  // namespace

extern "C" int qcs_localize_noalloc(const qcs_loc_para *p, const uint16_t *d_rois, const float *d_wle, int n,
                                    float *d_rows, int *d_nvalid, void *stream) {
    g_msg[0] = 0;
    if (!p || !d_rois || !d_wle || !d_rows || n < 0) return noalloc_fail(QCS_ERR_ARG, "null pointer or negative n");
    if (n > QCS_NOALLOC_MAX_ROIS) return noalloc_fail(QCS_ERR_CAPACITY, "n above QCS_NOALLOC_MAX_ROIS");
    if (reinterpret_cast<uintptr_t>(d_rows) & 15)
        return noalloc_fail(QCS_ERR_ARG, "d_rows must be 16-byte aligned (rows are written 16 bytes at a time)");
    const int R = p->ROISize;
    if (R < 5 || R > 17 || (R & 1) == 0 || (p->MultiEmitterFitEn && R > 13))
        return noalloc_fail(QCS_ERR_ROISIZE, "unsupported ROISize");
    if (p->LocType < QCS_LOCTYPE_GS2D || p->LocType > QCS_LOCTYPE_DH3D) return noalloc_fail(QCS_ERR_ARG, "LocType");
    if (!(p->QE > 0.0f)) return noalloc_fail(QCS_ERR_ARG, "QE must be positive");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(QCS_ERR_CUDA, "no current CUDA device");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        CUcontext ctx = nullptr;
        const bool have_ctx = current_context(&ctx);
        if (!g_scratch_addr[dev] || (have_ctx && ctx != g_scratch_ctx[dev])) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) return noalloc_fail(QCS_ERR_CUDA, "cudaGetSymbolAddress of the scratch array");
            g_scratch_addr[dev] = ptr;
            if (!have_ctx) current_context(&ctx);  // cudaGetSymbolAddress made the primary context current
            g_scratch_ctx[dev] = ctx;
        }
        base = static_cast<unsigned char *>(g_scratch_addr[dev]);
    }
    if (n == 0) {
        if (d_nvalid) {
            cudaError_t e = cudaMemsetAsync(d_nvalid, 0, sizeof(int), static_cast<cudaStream_t>(stream));
            if (e != cudaSuccess) return noalloc_fail(QCS_ERR_CUDA, "clear the row count");
        }
        return QCS_OK;
    }
    qcs::CascadeState st;
    st.q_single = reinterpret_cast<int *>(base + kOffQ);
    st.q2 = reinterpret_cast<int *>(base + kOffQ + al(kMax * sizeof(int)));
    st.q3 = reinterpret_cast<int *>(base + kOffQ + 2 * al(kMax * sizeof(int)));
    st.to2e = reinterpret_cast<uint8_t *>(base + kOffFlags);
    st.res2 = reinterpret_cast<int8_t *>(base + kOffFlags + al(kMax));
    st.res3 = reinterpret_cast<int8_t *>(base + kOffFlags + 2 * al(kMax));
    st.extra2 = reinterpret_cast<float *>(base + kOffExtra);
    st.extra3 = reinterpret_cast<float *>(base + kOffExtra + al(kMax * 12 * sizeof(float)));
    st.counters = reinterpret_cast<int *>(base + kOffCounters);
    st.scan = reinterpret_cast<int *>(base + kOffScan);
    qcs::CascadeArgs a;
    a.para = *p;
    a.rois = d_rois;
    a.wle = d_wle;
    a.n = n;
    a.loc = d_rows;
    a.max_rows = 2 * n;
    a.stream = static_cast<cudaStream_t>(stream);
    cudaError_t e = qcs::run_cascade(a, st);
    if (e != cudaSuccess) return noalloc_fail(QCS_ERR_CUDA, cudaGetErrorString(e));
    if (d_nvalid) {
        e = cudaMemcpyAsync(d_nvalid, st.counters + qcs::kCntValid, sizeof(int), cudaMemcpyDeviceToDevice, a.stream);
        if (e != cudaSuccess) return noalloc_fail(QCS_ERR_CUDA, "copy the row count");
    }
    return QCS_OK;
}
