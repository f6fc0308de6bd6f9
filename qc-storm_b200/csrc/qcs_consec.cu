// Consecutive-frame merging (ConsecutiveFit_TypeDef::ConsecutiveFit_WeightedAvg,
// ConsecutiveFit/ConsecutiveFit_top.cu:22-98, kernels ConsecutiveFit.cu:18-220):
// a molecule that stays on over consecutive frames gives one localization per
// frame; chains of localizations in consecutive frames closer than
// ConsecFit_DistanceTh_nm are merged into their first row (sums of photons and
// background, positions and widths averaged with weights 10 / CRLB_x), the
// other rows of a chain zeroed, and the chain lengths counted (on-time
// histogram).  Each call merges the previous call's group with the new one,
// outputs the previous group (now final) and keeps the new group for the next
// call, as the reference does.
//
// The reference links each row by scanning, one thread per row, every row from
// the start of its 32-row block to the end of the next frame, O(rows x rows of
// two frames).  Here the rows are sorted once by (frame, integer y) and each
// row binary-searches the next frame's rows within its distance threshold in
// y, O(rows log rows); the chosen link is the same (the closest row of the next
// frame in integer distance, the first in row order on ties, among rows at or
// after the start of the row's 32-row block) for rows in frame order, the order
// RemoveZeroLocalizations with frame sorting leaves them in.  The merge and
// removal kernels are the reference's per-row arithmetic (weighted sums as
// nvcc fuses them), so the rows equal its CUDA build's bit for bit; the CRLB
// pass recomputes, as the reference's unbounded 32-thread launch does, the
// previous group's rows and the new group's rows up to the next multiple of 32.
#include <cstdint>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"
#include "qcs_kernels.h"

using qcs::fail;

namespace {

constexpr int kTPB = 256;
constexpr int kBlockRows = 32;  // the reference's ThreadsPerBlock: the link scan starts at its block's first row

__device__ __forceinline__ uint64_t link_key(int frame, int y) {
    return ((uint64_t)(uint32_t)frame << 32) | (uint64_t)((uint32_t)y ^ 0x80000000u);
}

// (frame, integer y) sort keys of the rows; float-to-int as the reference's
// implicit conversions (truncation; NaN -> 0; saturation)
__global__ void keys_kernel(const float *__restrict__ rows, int T, uint64_t *__restrict__ keys,
                            int *__restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    const float *r = rows + (size_t)i * 12;
    keys[i] = link_key((int)r[QCS_POS_FRME], (int)r[QCS_POS_YPOS]);
    vals[i] = i;
}

// first index in [0, n) whose key is >= k
__device__ __forceinline__ int lower_bound(const uint64_t *__restrict__ a, int n, uint64_t k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// gpuFindConsecutiveMolecules: bwd[i] = the closest row of the next frame
// within the threshold (-2: none), fwd[that row] = 1.
__global__ void link_kernel(const float *__restrict__ rows, int T, const uint64_t *__restrict__ skeys,
                            const int *__restrict__ svals, float th_px, int *__restrict__ fwd, int *__restrict__ bwd) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= T) return;
    const float *r1 = rows + (size_t)gid * 12;
    const int X1 = (int)r1[QCS_POS_XPOS], Y1 = (int)r1[QCS_POS_YPOS], F1 = (int)r1[QCS_POS_FRME];
    float th2 = th_px;
    th2 = th2 * th2;
    int best = -1;
    if (F1 < 0x7fffffff && th2 > 0.0f) {
        const int gid0 = gid - gid % kBlockRows;
        // every dy with dy * dy < th2, and one more
        const long long r = (long long)ceilf(sqrtf(th2));
        long long ylo = (long long)Y1 - r, yhi = (long long)Y1 + r;
        if (ylo < -2147483648LL) ylo = -2147483648LL;
        if (yhi > 2147483647LL) yhi = 2147483647LL;
        const uint64_t klo = link_key(F1 + 1, (int)ylo), khi = link_key(F1 + 1, (int)yhi);
        int bd = 0;
        for (int j = lower_bound(skeys, T, klo); j < T && skeys[j] <= khi; ++j) {
            const int c = svals[j];
            if (c < gid0) continue;
            const float *r2 = rows + (size_t)c * 12;
            const unsigned dx = (unsigned)X1 - (unsigned)(int)r2[QCS_POS_XPOS];
            const unsigned dy = (unsigned)Y1 - (unsigned)(int)r2[QCS_POS_YPOS];
            const int d2 = (int)(dx * dx + dy * dy);
            if (!((float)d2 < th2)) continue;
            if (best < 0 || d2 < bd || (d2 == bd && c < best)) {
                best = c;
                bd = d2;
            }
        }
    }
    if (best >= 0) {
        bwd[gid] = best;
        fwd[best] = 1;
    } else {
        bwd[gid] = -2;
    }
}

// gpuConsecutiveFit: every row without a forward link takes its chain's sums
// and precision-weighted averages; chains starting in the new group are counted.
__global__ void merge_kernel(float *__restrict__ rows, int T, int last_n, const int *__restrict__ fwd,
                             const int *__restrict__ bwd, float QE, int *__restrict__ stat) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= T || fwd[gid] != 0) return;
    float wx = 0, wy = 0, wz = 0, wsx = 0, wsy = 0, sp = 0, st = 0, sb = 0, sprec = 0;
    int id = gid, num = 0;
    for (;;) {
        const float *r = rows + (size_t)id * 12;
        const float prec = __fdiv_rn(10.0f, r[QCS_POS_CRBX]);
        sp = __fadd_rn(sp, r[QCS_POS_PPHO]);
        st = __fadd_rn(st, r[QCS_POS_TPHO]);
        sb = __fadd_rn(sb, r[QCS_POS_BAKG]);
        wx = __fmaf_rn(r[QCS_POS_XPOS], prec, wx);
        wy = __fmaf_rn(r[QCS_POS_YPOS], prec, wy);
        wz = __fmaf_rn(r[QCS_POS_ZPOS], prec, wz);
        wsx = __fmaf_rn(r[QCS_POS_SIGX], prec, wsx);
        wsy = __fmaf_rn(r[QCS_POS_SIGY], prec, wsy);
        sprec = __fadd_rn(sprec, prec);
        id = bwd[id];
        num++;
        if (!(id > 0)) break;
    }
    float *h = rows + (size_t)gid * 12;
    h[QCS_POS_PPHO] = sp;
    h[QCS_POS_XPOS] = __fdiv_rn(wx, sprec);
    h[QCS_POS_YPOS] = __fdiv_rn(wy, sprec);
    h[QCS_POS_ZPOS] = __fdiv_rn(wz, sprec);
    h[QCS_POS_SIGX] = __fdiv_rn(wsx, sprec);
    h[QCS_POS_SIGY] = __fdiv_rn(wsy, sprec);
    h[QCS_POS_TPHO] = st;
    h[QCS_POS_BAKG] = sb;
    h[QCS_POS_PSNR] = __fdiv_rn(__fmul_rn(__fsqrt_rn(QE), sp), __fsqrt_rn(__fadd_rn(sp, sb)));
    if (gid >= last_n) {
        const int on = min(max(num - 1, 0), QCS_ONTIME_BINS - 1);
        atomicAdd(stat + QCS_ONTIME_BINS, 1);
        atomicAdd(stat + on, 1);
    }
}

// gpuRemoveConsecutiveFluo: the later rows of each chain are zeroed.
__global__ void remove_kernel(float *__restrict__ rows, int T, const int *__restrict__ fwd,
                              const int *__restrict__ bwd) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= T || fwd[gid] != 0) return;
    for (int next = bwd[gid]; next > 0; next = bwd[next]) {
        float4 *d = reinterpret_cast<float4 *>(rows + (size_t)next * 12);
        d[0] = d[1] = d[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

inline int blocks(int n) { return (n + kTPB - 1) / kTPB; }

}  // namespace

struct qcs_consec {
    int capacity = 0;        // rows per group
    int last_n = 0;          // FluoNum_LastGroup
    int out_n = 0;           // OutFluoNum of the last call
    float *d_last = nullptr;  // capacity x 12: the previous group's rows
    float *d_work = nullptr;  // 2 capacity x 12: previous then new group
    int *d_fwd = nullptr, *d_bwd = nullptr;
    uint64_t *d_keys = nullptr, *d_skeys = nullptr;
    int *d_vals = nullptr, *d_svals = nullptr;
    void *d_sort = nullptr;
    size_t sort_bytes = 0;
    int *d_stat = nullptr;    // on-time histogram, then the chain count
    float *h_out = nullptr;   // pinned, 2 capacity x 12
    int *h_stat = nullptr;    // pinned
    float ontime[QCS_ONTIME_BINS] = {0};
    cudaStream_t stream = nullptr;
};

namespace {

int consec_run(qcs_consec *c, const float *rows, bool device_rows, int n, int is_end, const qcs_loc_para *p,
               cudaStream_t s) {
    const int T = c->last_n + n;
    const size_t rb = 12 * sizeof(float);
    if (c->last_n)
        QCS_CUDA(cudaMemcpyAsync(c->d_work, c->d_last, (size_t)c->last_n * rb, cudaMemcpyDeviceToDevice, s),
                 "previous group");
    if (n)
        QCS_CUDA(cudaMemcpyAsync(c->d_work + (size_t)c->last_n * 12, rows, (size_t)n * rb,
                                 device_rows ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
                 "new group");
    QCS_CUDA(cudaMemsetAsync(c->d_fwd, 0, (size_t)(T > 0 ? T : 1) * sizeof(int), s), "links");
    QCS_CUDA(cudaMemsetAsync(c->d_stat, 0, (QCS_ONTIME_BINS + 1) * sizeof(int), s), "on-time histogram");
    if (T > 0) {
        keys_kernel<<<blocks(T), kTPB, 0, s>>>(c->d_work, T, c->d_keys, c->d_vals);
        size_t tb = c->sort_bytes;
        QCS_CUDA(cub::DeviceRadixSort::SortPairs(c->d_sort, tb, c->d_keys, c->d_skeys, c->d_vals, c->d_svals, T, 0, 64,
                                                 s),
                 "sort rows by frame and y");
        const float th_px = p->ConsecFit_DistanceTh_nm / p->PixelSize;
        link_kernel<<<blocks(T), kTPB, 0, s>>>(c->d_work, T, c->d_skeys, c->d_svals, th_px, c->d_fwd, c->d_bwd);
        merge_kernel<<<blocks(T), kTPB, 0, s>>>(c->d_work, T, c->last_n, c->d_fwd, c->d_bwd, p->QE, c->d_stat);
        remove_kernel<<<blocks(T), kTPB, 0, s>>>(c->d_work, T, c->d_fwd, c->d_bwd);
        QCS_CUDA(cudaGetLastError(), "consecutive-frame kernels");
    }
    // CRLB of the previous group's rows, and of the new group's up to the next multiple of 32
    int nc = (c->last_n + 31) / 32 * 32;
    if (nc > T) nc = T;
    if (nc > 0)
        QCS_CUDA(qcs::launch_crlb(c->d_work, nullptr, nc, nc, p->LocType, p->ReadNoise_e, p->QE, p->PixelSize, s),
                 "CRLB");
    int out_n;
    if (!is_end) {
        out_n = c->last_n;
        if (n)
            QCS_CUDA(cudaMemcpyAsync(c->d_last, c->d_work + (size_t)c->last_n * 12, (size_t)n * rb,
                                     cudaMemcpyDeviceToDevice, s),
                     "keep the new group");
        c->last_n = n;
    } else {
        out_n = T;
        c->last_n = 0;
    }
    c->out_n = out_n;
    QCS_CUDA(cudaMemcpyAsync(c->h_stat, c->d_stat, (QCS_ONTIME_BINS + 1) * sizeof(int), cudaMemcpyDeviceToHost, s),
             "read on-time histogram");
    if (!device_rows && out_n)
        QCS_CUDA(cudaMemcpyAsync(c->h_out, c->d_work, (size_t)out_n * rb, cudaMemcpyDeviceToHost, s), "read rows");
    QCS_CUDA(cudaStreamSynchronize(s), "consecutive-frame merging");
    int valid = c->h_stat[QCS_ONTIME_BINS];
    if (valid <= 0) valid = 1;
    for (int k = 0; k < QCS_ONTIME_BINS; ++k) c->ontime[k] = c->h_stat[k] * 1.0f / valid;
    return QCS_OK;
}

}  // namespace

extern "C" {

int qcs_consec_deinit(qcs_consec *c) {
    if (!c) return QCS_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_last);
    cudaFree(c->d_work);
    cudaFree(c->d_fwd);
    cudaFree(c->d_keys);
    cudaFree(c->d_sort);
    cudaFree(c->d_stat);
    cudaFreeHost(c->h_out);
    cudaFreeHost(c->h_stat);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return QCS_OK;
}

int qcs_consec_init(int capacity, qcs_consec **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    if (capacity <= 0) capacity = 2 * QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_consec *c = new qcs_consec();
    c->capacity = capacity;
    const size_t cap = (size_t)capacity, T = 2 * cap;
    cudaError_t e = cudaMalloc((void **)&c->d_last, cap * 12 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_work, T * 12 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_fwd, 2 * T * sizeof(int));
    // keys, sorted keys, values, sorted values, each from a 256-byte boundary
    const size_t bk = (T * sizeof(uint64_t) + 255) / 256 * 256, bv = (T * sizeof(int) + 255) / 256 * 256;
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_keys, 2 * bk + 2 * bv);
    if (e == cudaSuccess) {
        c->d_bwd = c->d_fwd + T;
        char *b = reinterpret_cast<char *>(c->d_keys);
        c->d_skeys = reinterpret_cast<uint64_t *>(b + bk);
        c->d_vals = reinterpret_cast<int *>(b + 2 * bk);
        c->d_svals = reinterpret_cast<int *>(b + 2 * bk + bv);
        e = cub::DeviceRadixSort::SortPairs(nullptr, c->sort_bytes, c->d_keys, c->d_skeys, c->d_vals, c->d_svals,
                                            (int)T, 0, 64);
    }
    if (e == cudaSuccess) e = cudaMalloc(&c->d_sort, c->sort_bytes > 0 ? c->sort_bytes : 1);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_stat, (QCS_ONTIME_BINS + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_out, T * 12 * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_stat, (QCS_ONTIME_BINS + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        qcs_consec_deinit(c);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_consec_init", e);
    }
    *out = c;
    return QCS_OK;
}

int qcs_consec_fit(qcs_consec *c, const float *h_rows, int n, int is_end, const qcs_loc_para *p, void *stream) {
    if (!c || !p) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n > c->capacity) return fail(QCS_ERR_CAPACITY, "group larger than the merger's capacity");
    if (n > 0 && !h_rows) return fail(QCS_ERR_ARG, "null rows");
    if (!(p->PixelSize > 0.0f)) return fail(QCS_ERR_ARG, "PixelSize must be positive");
    return consec_run(c, h_rows, false, n, is_end, p, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

int qcs_consec_fit_device(qcs_consec *c, const float *d_rows, int n, int is_end, const qcs_loc_para *p,
                          void *stream) {
    if (!c || !p) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n > c->capacity) return fail(QCS_ERR_CAPACITY, "group larger than the merger's capacity");
    if (n > 0 && !d_rows) return fail(QCS_ERR_ARG, "null rows");
    if (!(p->PixelSize > 0.0f)) return fail(QCS_ERR_ARG, "PixelSize must be positive");
    return consec_run(c, d_rows, true, n, is_end, p, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

int qcs_consec_out_num(const qcs_consec *c) { return c ? c->out_n : 0; }
const float *qcs_consec_h_out_loc_arry(const qcs_consec *c) { return c ? c->h_out : nullptr; }
const float *qcs_consec_d_out_loc_arry(const qcs_consec *c) { return c ? c->d_work : nullptr; }

int qcs_consec_read_rows(qcs_consec *c, float *h_out) {
    if (!c || !h_out) return fail(QCS_ERR_ARG, "null argument");
    if (c->out_n > 0)
        QCS_CUDA(cudaMemcpy(h_out, c->d_work, (size_t)c->out_n * 12 * sizeof(float), cudaMemcpyDeviceToHost),
                 "read rows");
    return QCS_OK;
}

int qcs_consec_ontime_ratio(const qcs_consec *c, float *out) {
    if (!c || !out) return fail(QCS_ERR_ARG, "null argument");
    for (int k = 0; k < QCS_ONTIME_BINS; ++k) out[k] = c->ontime[k];
    return QCS_OK;
}

}  // extern "C"
