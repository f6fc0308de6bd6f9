// Removal of rejected (all-zero) localization rows, optionally ordered by
// frame: ZeroLocalizationsRemovel_TypeDef::RemoveZeroLocalizations
// (bfgsMLE_Loc_top/ZeroLocalizationsRemove.cu:21-186).
//
// The reference either copies the rows with peak photons > 1 in row order
// (indices found on the host, :64-102) or, to order by frame, launches one
// kernel per frame that appends that frame's valid rows through an atomic
// counter (:42-61, 161-186) — a launch per frame and arrival order within a
// frame.  Here one pass marks each row with its frame key (or "drop"), a
// stable radix sort orders the row indices by key, and a gather writes the
// kept rows: one sort for any number of frames, row order within a frame
// (deterministic), the row count left on the device.
#include <cstdint>
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"

namespace qcs {
namespace {

constexpr int kTPB = 256;

// Key of a kept row: its frame offset from first_frame (0 without sorting);
// dropped rows get `drop` and sort after every kept row.
__global__ void zero_keys_kernel(const float *__restrict__ rows, int n, const int *__restrict__ n_dev, int sort_frame,
                                 int first_frame, int end_frame, unsigned drop, unsigned *__restrict__ keys,
                                 int *__restrict__ vals, int *__restrict__ kept) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int rows_n = n_dev ? min(max(*n_dev, 0), n) : n;
    if (i >= n) return;
    unsigned key = drop;
    if (i < rows_n) {
        const float *r = rows + (size_t)i * QCS_OUT_PARA_NUM;
        if (sort_frame) {
            // truncating float -> int conversions of the reference (:171-172)
            const int peak = __float2int_rz(r[QCS_POS_PPHO]);
            const int frame = __float2int_rz(r[QCS_POS_FRME]);
            if ((float)peak > 1.0f && frame >= first_frame && frame <= end_frame)
                key = (unsigned)(frame - first_frame);
        } else if (r[QCS_POS_PPHO] > 1.0f) {
            key = 0;
        }
    }
    keys[i] = key;
    vals[i] = i;
    if (key != drop) atomicAdd(kept, 1);
}

__global__ void zero_gather_kernel(const float *__restrict__ rows, const int *__restrict__ order,
                                   const int *__restrict__ kept, float *__restrict__ out, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || k >= *kept) return;
    const float4 *s = reinterpret_cast<const float4 *>(rows + (size_t)order[k] * QCS_OUT_PARA_NUM);
    float4 *d = reinterpret_cast<float4 *>(out + (size_t)k * QCS_OUT_PARA_NUM);
    d[0] = s[0];
    d[1] = s[1];
    d[2] = s[2];
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t sort_bytes(int n) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned *)nullptr, (unsigned *)nullptr, (const int *)nullptr,
                                    (int *)nullptr, n);
    return bytes;
}

}  // namespace
}  // namespace qcs

using qcs::fail;

struct qcs_zero_data {
    int capacity;
    float *d_in = nullptr, *d_out = nullptr;
    void *d_scratch = nullptr;
    size_t sort_temp = 0;
    unsigned *keys_in = nullptr, *keys_out = nullptr;
    int *vals_in = nullptr, *vals_out = nullptr, *kept = nullptr;
    float *h_loc = nullptr;
    int *h_kept = nullptr;
    int valid = 0;
    cudaStream_t stream = nullptr;
};

extern "C" {

int qcs_zero_deinit(qcs_zero_data *c) {
    if (!c) return QCS_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_in);
    cudaFree(c->d_out);
    cudaFree(c->d_scratch);
    cudaFreeHost(c->h_loc);
    cudaFreeHost(c->h_kept);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return QCS_OK;
}

int qcs_zero_init(int capacity, qcs_zero_data **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    if (capacity <= 0) capacity = 2 * QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_zero_data *c = new qcs_zero_data();
    c->capacity = capacity;
    const size_t cap = (size_t)capacity;
    c->sort_temp = qcs::sort_bytes(capacity);
    const size_t scratch = 2 * qcs::align256(cap * 4) + 2 * qcs::align256(cap * 4) + qcs::align256(4) +
                           qcs::align256(c->sort_temp);
    cudaError_t e = cudaMalloc((void **)&c->d_in, cap * QCS_OUT_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_out, cap * QCS_OUT_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_scratch, scratch);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_loc, cap * QCS_OUT_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_kept, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        qcs_zero_deinit(c);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_zero_init", e);
    }
    char *s = static_cast<char *>(c->d_scratch);
    c->keys_in = reinterpret_cast<unsigned *>(s);
    s += qcs::align256(cap * 4);
    c->keys_out = reinterpret_cast<unsigned *>(s);
    s += qcs::align256(cap * 4);
    c->vals_in = reinterpret_cast<int *>(s);
    s += qcs::align256(cap * 4);
    c->vals_out = reinterpret_cast<int *>(s);
    s += qcs::align256(cap * 4);
    c->kept = reinterpret_cast<int *>(s);
    *out = c;
    return QCS_OK;
}

int qcs_zero_remove_device(qcs_zero_data *c, const float *d_rows, int n, const int *d_n, int sort_frame_en,
                           int first_frame, int end_frame, float *d_out, int *d_nvalid, void *stream) {
    if (!c || !d_rows || !d_out) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n > c->capacity) return fail(QCS_ERR_CAPACITY, "row count above the context capacity");
    if (sort_frame_en && end_frame < first_frame) return fail(QCS_ERR_ARG, "end frame before first frame");
    if ((reinterpret_cast<uintptr_t>(d_rows) | reinterpret_cast<uintptr_t>(d_out)) & 15)
        return fail(QCS_ERR_ARG, "row arrays must be 16-byte aligned");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(cudaMemsetAsync(c->kept, 0, sizeof(int), s), "clear count");
    if (n > 0) {
        // keys 0 .. span-1 for kept rows, `span` for dropped ones
        const long long span = sort_frame_en ? (long long)end_frame - first_frame + 1 : 1;
        if (span > 0x7FFFFFFFll) return fail(QCS_ERR_ARG, "frame range too large");
        int bits = 1;
        while (bits < 32 && (1ll << bits) <= span) ++bits;
        const int grid = (n + qcs::kTPB - 1) / qcs::kTPB;
        qcs::zero_keys_kernel<<<grid, qcs::kTPB, 0, s>>>(d_rows, n, d_n, sort_frame_en, first_frame, end_frame,
                                                         (unsigned)span, c->keys_in, c->vals_in, c->kept);
        void *temp = reinterpret_cast<char *>(c->kept) + qcs::align256(4);
        size_t temp_bytes = c->sort_temp;
        QCS_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, c->keys_in, c->keys_out, c->vals_in, c->vals_out, n,
                                                 0, bits, s),
                 "frame sort");
        qcs::zero_gather_kernel<<<grid, qcs::kTPB, 0, s>>>(d_rows, c->vals_out, c->kept, d_out, n);
        QCS_CUDA(cudaGetLastError(), "zero-row removal kernels");
    }
    if (d_nvalid) QCS_CUDA(cudaMemcpyAsync(d_nvalid, c->kept, sizeof(int), cudaMemcpyDeviceToDevice, s), "copy count");
    return QCS_OK;
}

int qcs_zero_remove(qcs_zero_data *c, const float *h_rows, int n, int sort_frame_en, int first_frame, int end_frame,
                    void *stream) {
    if (!c || (!h_rows && n > 0)) return fail(QCS_ERR_ARG, "null argument");
    if (n > c->capacity) return fail(QCS_ERR_CAPACITY, "row count above the context capacity");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    c->valid = 0;
    if (n > 0)
        QCS_CUDA(cudaMemcpyAsync(c->d_in, h_rows, (size_t)n * QCS_OUT_PARA_NUM * sizeof(float), cudaMemcpyHostToDevice,
                                 s),
                 "copy rows");
    int st = qcs_zero_remove_device(c, c->d_in, n, nullptr, sort_frame_en, first_frame, end_frame, c->d_out, nullptr,
                                    s);
    if (st) return st;
    QCS_CUDA(cudaMemcpyAsync(c->h_kept, c->kept, sizeof(int), cudaMemcpyDeviceToHost, s), "read count");
    QCS_CUDA(cudaStreamSynchronize(s), "zero-row removal");
    const int k = *c->h_kept;
    if (k > 0)
        QCS_CUDA(cudaMemcpyAsync(c->h_loc, c->d_out, (size_t)k * QCS_OUT_PARA_NUM * sizeof(float),
                                 cudaMemcpyDeviceToHost, s),
                 "read rows");
    QCS_CUDA(cudaStreamSynchronize(s), "read rows");
    c->valid = k;
    return QCS_OK;
}

const float *qcs_zero_h_loc_arry(const qcs_zero_data *c) { return c ? c->h_loc : nullptr; }
int qcs_zero_valid_num(const qcs_zero_data *c) { return c ? c->valid : 0; }

}  // extern "C"
