// WLE pre-pass (weighted-MLE parameters) over a batch of ROI records:
//   psf_width_kernel   row/column means -> natural cubic spline x10 -> peak ->
//                      two-sided widths sigma L/R/U/D
//                      (WLEParaEstimation_core.h:44-156, SplineInterpolation.h:40-202,
//                      WLEParaEstimation_core.cu:21-28, 91-136)
//   nearest neighbour  same-frame minimum centre distance
//                      (WLEParaEstimation_core.cu:140-183)
//   classify_kernel    molecule type MLEFit / WLEFit / MultiFit
//                      (WLEParaEstimation_core.cu:197-264)
// The floating-point code keeps the reference's expression shapes (bit-equal
// results).  The nearest-neighbour search replaces the reference's O(N^2)
// all-pairs loop with a (frame, y, x) radix sort and a y-bounded scan of the
// sorted neighbours; the integer squared distance it minimises is the same.
// Records produced by ROI extraction are already in (frame, y, x) order;
// launch_wle_presorted takes their range from device memory and scans their
// compact key array without the sort, so the pass needs no host
// synchronisation.
#include <cstdint>
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "qcs_kernels.h"

namespace qcs {
namespace {

constexpr int kInterp = 10;                    // InterpolationRatio
#define QCS_INTERP_GAP (1.0f / kInterp)        // InterpolationGap
#define QCS_PEAK_FIND_RATIO 0.8f               // PeakFindRangeRatio
#define QCS_MAX_WIDTH_DIFF 0.40f               // MaxTolerablePSFWidthDiff

template <int N>
__device__ __forceinline__ void spline_system(float *A, float *b, const float *x_i, const float *y_i) {
    for (int r = 0; r < N; r++)
        for (int c = 0; c < N; c++) A[r * N + c] = 0;
    A[0] = 1;
    A[(N - 1) * N + N - 1] = 1;
    for (int i = 1; i < N - 1; i++) {
        const float h0 = x_i[i] - x_i[i - 1];
        const float h1 = x_i[i + 1] - x_i[i];
        A[i * N + i - 1] = h0;
        A[i * N + i] = 2 * (h0 + h1);
        A[i * N + i + 1] = h1;
    }
    b[0] = 0;
    b[N - 1] = 0;
    for (int i = 1; i < N - 1; i++) {
        const float h0 = x_i[i] - x_i[i - 1];
        const float h1 = x_i[i + 1] - x_i[i];
        const float a0 = y_i[i - 1];
        const float a1 = y_i[i];
        const float a2 = y_i[i + 1];
        b[i] = 3 / h1 * (a2 - a1) - 3 / h0 * (a1 - a0);
    }
}

template <int N>
__device__ __forceinline__ void spline_solve(const float *A, const float *b, float *x) {
    float y[N], Beta[N];
    for (int i = 0; i < N - 1; i++) {
        const float ci = A[i * N + i + 1];
        const float bi = A[i * N + i];
        if (i == 0) {
            Beta[i] = ci / bi;
        } else {
            const float ai = A[i * N + i - 1];
            Beta[i] = ci / (bi - ai * Beta[i - 1]);
        }
    }
    for (int i = 0; i < N; i++) {
        const float bi = A[i * N + i];
        if (i == 0) {
            y[i] = b[i] / bi;
        } else {
            const float ai = A[i * N + i - 1];
            y[i] = (b[i] - ai * y[i - 1]) / (bi - ai * Beta[i - 1]);
        }
    }
    for (int i = N - 1; i >= 0; i--) {
        if (i == N - 1)
            x[i] = y[i];
        else
            x[i] = y[i] - Beta[i] * x[i + 1];
    }
}

template <int N, int M>
__device__ __forceinline__ void spline_interpolate(const float *x_i, const float *y_i, const float *x_o, float *y_o) {
    float An[N], Bn[N], Cn[N], Dn[N];
    for (int i = 0; i < N; i++) An[i] = y_i[i];
    float A[N * N], b[N];
    spline_system<N>(A, b, x_i, y_i);
    spline_solve<N>(A, b, Cn);
    for (int i = 0; i < N - 1; i++) {
        const float hi = x_i[i + 1] - x_i[i];
        Bn[i] = 1 / hi * (An[i + 1] - An[i]) - hi / 3 * (2 * Cn[i] + Cn[i + 1]);
        Dn[i] = (Cn[i + 1] - Cn[i]) / (3 * hi);
    }
    for (int i = 0; i < M; i++) {
        const float xn = x_o[i];
        int ParaSet = xn - 0.0f;  // sample positions start at pixel 0, unit spacing
        if (ParaSet < 0) ParaSet = 0;
        if (ParaSet >= N - 1) ParaSet = N - 2;
        const float xi = x_i[ParaSet];
        y_o[i] = An[ParaSet] + Bn[ParaSet] * (xn - xi) + Cn[ParaSet] * (xn - xi) * (xn - xi) +
                 Dn[ParaSet] * (xn - xi) * (xn - xi) * (xn - xi);
    }
}

__device__ __forceinline__ int find_max_pos(const float *iData, int DataLen, int LSel, int RSel) {
    LSel = max(LSel, 0);
    RSel = min(RSel, DataLen - 1);
    int MaxIdx = DataLen / 2;
    for (int cnt = LSel; cnt <= RSel; cnt++)
        if (iData[cnt] > iData[MaxIdx]) MaxIdx = cnt;
    return MaxIdx;
}

__device__ __forceinline__ void two_sided_width(float *SigmaL, float *SigmaR, const float *MeanData_Intp, int DataLen,
                                                int MaxPos) {
    const float MaxValue = MeanData_Intp[MaxPos];
    const int LLen = MaxPos;
    const int RLen = DataLen - MaxPos - 1;
    const int CmpLen = min(LLen, RLen);
    float SDat_L = 0;
    for (int i = MaxPos - CmpLen; i <= MaxPos; i++) SDat_L = SDat_L + MeanData_Intp[i];
    float SDat_R = 0;
    for (int i = MaxPos; i <= MaxPos + CmpLen; i++) SDat_R = SDat_R + MeanData_Intp[i];
    *SigmaL = SDat_L * QCS_INTERP_GAP / MaxValue / 1.2533f;
    *SigmaR = SDat_R * QCS_INTERP_GAP / MaxValue / 1.2533f;
}

// Records [begin, begin + n): from the arguments, or from span[0], span[1]
// in device memory when span is set (grid-stride loops cover any n).
struct Span {
    int begin, n;
    const int *span;
    __device__ __forceinline__ void get(int &b, int &m) const {
        if (span) {
            b = span[0];
            m = span[1];
        } else {
            b = begin;
            m = n;
        }
    }
};

template <int R>
__device__ __forceinline__ void psf_width_one(const uint16_t *__restrict__ rois, float *__restrict__ wle, int gid) {
    enum { Len = R, ILen = (R - 1) * kInterp + 1, WHOLE = R * (R + 1) };
    const uint16_t *pROI = rois + (size_t)gid * WHOLE;
    float MeanX[Len], MeanY[Len], x0[Len], xn[ILen], yn_MeanX[ILen], yn_MeanY[ILen];
    for (int cnt = 0; cnt < Len; cnt++) {
        MeanX[cnt] = 0;
        MeanY[cnt] = 0;
    }
    for (int r = 0; r < Len; r++) {
        for (int c = 0; c < Len; c++) {
            MeanX[c] = MeanX[c] + pROI[r * R + c];
            MeanY[r] = MeanY[r] + pROI[r * R + c];
        }
    }
    float MinX = MeanX[0];
    float MinY = MeanY[0];
    for (int cnt = 0; cnt < Len; cnt++) {
        MinX = fminf(MinX, MeanX[cnt]);
        MinY = fminf(MinY, MeanY[cnt]);
    }
    for (int cnt = 0; cnt < Len; cnt++) {
        MeanX[cnt] = (MeanX[cnt] - MinX) / Len;
        MeanY[cnt] = (MeanY[cnt] - MinY) / Len;
    }
    for (int cnt = 0; cnt < Len; cnt++) x0[cnt] = cnt;
    for (int cnt = 0; cnt < ILen; cnt++) xn[cnt] = cnt * QCS_INTERP_GAP;
    spline_interpolate<Len, ILen>(x0, MeanX, xn, yn_MeanX);
    spline_interpolate<Len, ILen>(x0, MeanY, xn, yn_MeanY);
    const int FindRegionlen = kInterp * QCS_PEAK_FIND_RATIO;
    const int InterpCenter = ILen / 2;
    const int MaxPos_X = find_max_pos(yn_MeanX, ILen, InterpCenter - FindRegionlen, InterpCenter + FindRegionlen);
    const int MaxPos_Y = find_max_pos(yn_MeanY, ILen, InterpCenter - FindRegionlen, InterpCenter + FindRegionlen);
    float SigmaL, SigmaR, SigmaU, SigmaD;
    two_sided_width(&SigmaL, &SigmaR, yn_MeanX, ILen, MaxPos_X);
    two_sided_width(&SigmaU, &SigmaD, yn_MeanY, ILen, MaxPos_Y);
    float *o = wle + (size_t)gid * QCS_WLE_PARA_NUM;
    o[1] = SigmaL;
    o[2] = SigmaR;
    o[3] = SigmaU;
    o[4] = SigmaD;
}

template <int R>
__global__ void psf_width_kernel(const uint16_t *__restrict__ rois, float *__restrict__ wle, Span sp) {
    int b, n;
    sp.get(b, n);
    for (int k = threadIdx.x + blockDim.x * blockIdx.x; k < n; k += gridDim.x * blockDim.x)
        psf_width_one<R>(rois, wle, b + k);
}

// Sort key: frame (32 bits) | y (16) | x (16) of the ROI centre.
__global__ void nn_keys_kernel(const uint16_t *__restrict__ rois, int n, int whole, int pix,
                               unsigned long long *keys, int *vals) {
    const int i = threadIdx.x + blockDim.x * blockIdx.x;
    if (i >= n) return;
    const uint16_t *h = rois + (size_t)i * whole + pix;
    const unsigned long long frame = (unsigned long long)h[2] + 65536ull * h[3];
    keys[i] = (frame << 32) | ((unsigned long long)h[1] << 16) | h[0];
    vals[i] = i;
}

// Distance to the nearest other ROI centre of the same frame: scans the
// (frame, y, x)-sorted keys k[0..n) outwards from a, in each direction until
// the frame changes or the row distance alone exceeds the best so far.  Keys
// are fetched 8 at a time so that their loads overlap; they are examined in
// the same order as a one-by-one scan, which stops at the same key.
__device__ __forceinline__ float nn_sorted(const unsigned long long *__restrict__ k, int a, int n) {
    const unsigned long long ka = k[a];
    const unsigned long long frame = ka >> 32;
    const int ya = (int)((ka >> 16) & 0xFFFF), xa = (int)(ka & 0xFFFF);
    float best = 100000000.0f;
    bool go = true;
    for (int b = a + 1; go && b < n; b += 8) {
        unsigned long long kb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) kb[j] = (b + j < n) ? __ldg(k + b + j) : ~0ull;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (!go) break;
            if ((kb[j] >> 32) != frame) {
                go = false;
                break;
            }
            const int dy = (int)((kb[j] >> 16) & 0xFFFF) - ya, dx = (int)(kb[j] & 0xFFFF) - xa;
            if ((float)(dy * dy) > best) {
                go = false;
                break;
            }
            best = fminf(best, (float)(dx * dx + dy * dy));
        }
    }
    go = true;
    for (int b = a - 1; go && b >= 0; b -= 8) {
        unsigned long long kb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) kb[j] = (b - j >= 0) ? __ldg(k + b - j) : ~0ull;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (!go) break;
            if ((kb[j] >> 32) != frame) {
                go = false;
                break;
            }
            const int dy = (int)((kb[j] >> 16) & 0xFFFF) - ya, dx = (int)(kb[j] & 0xFFFF) - xa;
            if ((float)(dy * dy) > best) {
                go = false;
                break;
            }
            best = fminf(best, (float)(dx * dx + dy * dy));
        }
    }
    return sqrtf(best);
}

// Minimum distance for each record, over the radix-sorted keys.
__global__ void nn_scan_kernel(const unsigned long long *__restrict__ keys, const int *__restrict__ vals, int n,
                               float *__restrict__ wle) {
    const int a = threadIdx.x + blockDim.x * blockIdx.x;
    if (a >= n) return;
    wle[(size_t)vals[a] * QCS_WLE_PARA_NUM + 0] = nn_sorted(keys, a, n);
}

__device__ __forceinline__ void classify_one(const uint16_t *__restrict__ rois, float *__restrict__ wle, int gid, int R,
                                             int whole, int LocType) {
    float MaxMeanSigmaTh;
    if (LocType == QCS_LOCTYPE_GS2D)
        MaxMeanSigmaTh = R / 2.1f / 2.35f;
    else
        MaxMeanSigmaTh = R / 1.9f / 2.35f;
    const int ROIType_Detection = rois[(size_t)gid * whole + R * R + 4];
    float *w = wle + (size_t)gid * QCS_WLE_PARA_NUM;
    const float NearestNeighborDistance = w[0];
    const float SigmaL = w[1], SigmaR = w[2], SigmaU = w[3], SigmaD = w[4];
    const float diff1 = fabsf(SigmaL - SigmaR) / fminf(SigmaL, SigmaR);
    const float diff2 = fabsf(SigmaU - SigmaD) / fminf(SigmaU, SigmaD);
    const int IsContamination = (diff1 >= QCS_MAX_WIDTH_DIFF) || (diff2 >= QCS_MAX_WIDTH_DIFF);
    const float MeanSigma = (SigmaL + SigmaR + SigmaU + SigmaD) / 4;
    int MoleculeType = QCS_MOLECULE_MLEFIT;
    if ((ROIType_Detection == QCS_ROITYPE_SINGLE) && (IsContamination == 0) && (NearestNeighborDistance >= R) &&
        (MeanSigma <= MaxMeanSigmaTh))
        MoleculeType = QCS_MOLECULE_MLEFIT;
    else if ((ROIType_Detection == QCS_ROITYPE_MULTI) || (MeanSigma > MaxMeanSigmaTh) ||
             (NearestNeighborDistance < (R / 2.0f + 1.0f)))
        MoleculeType = QCS_MOLECULE_MULTIFIT;
    else
        MoleculeType = QCS_MOLECULE_WLEFIT;
    w[5] = MoleculeType;
}

__global__ void classify_kernel(const uint16_t *__restrict__ rois, float *__restrict__ wle, Span sp, int R, int whole,
                                int LocType) {
    int b, n;
    sp.get(b, n);
    for (int k = threadIdx.x + blockDim.x * blockIdx.x; k < n; k += gridDim.x * blockDim.x)
        classify_one(rois, wle, b + k, R, whole, LocType);
}

// Records already in ascending (frame, y, x) order with their keys in a
// compact array: PSF widths, nearest neighbour and molecule type of each
// record in one pass (one thread per record).
template <int R>
__global__ void wle_sorted_kernel(const uint16_t *__restrict__ rois, const unsigned long long *__restrict__ keys,
                                  Span sp, float *__restrict__ wle, int LocType) {
    int b0, n;
    sp.get(b0, n);
    for (int a = threadIdx.x + blockDim.x * blockIdx.x; a < n; a += gridDim.x * blockDim.x) {
        psf_width_one<R>(rois, wle, b0 + a);
        wle[(size_t)(b0 + a) * QCS_WLE_PARA_NUM + 0] = nn_sorted(keys + b0, a, n);
        classify_one(rois, wle, b0 + a, R, R * (R + 1), LocType);
    }
}

template <int R>
void psf_width_launch(const uint16_t *rois, float *wle, Span sp, int grid, int tpb, cudaStream_t s) {
    psf_width_kernel<R><<<grid, tpb, 0, s>>>(rois, wle, sp);
}

cudaError_t launch_psf_width(int R, const uint16_t *rois, float *wle, Span sp, int grid, int tpb, cudaStream_t s) {
    switch (R) {
    case 5: psf_width_launch<5>(rois, wle, sp, grid, tpb, s); break;
    case 7: psf_width_launch<7>(rois, wle, sp, grid, tpb, s); break;
    case 9: psf_width_launch<9>(rois, wle, sp, grid, tpb, s); break;
    case 11: psf_width_launch<11>(rois, wle, sp, grid, tpb, s); break;
    case 13: psf_width_launch<13>(rois, wle, sp, grid, tpb, s); break;
    case 15: psf_width_launch<15>(rois, wle, sp, grid, tpb, s); break;
    case 17: psf_width_launch<17>(rois, wle, sp, grid, tpb, s); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

size_t sort_temp_bytes(int n) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (const int *)nullptr, (int *)nullptr, n);
    return bytes;
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

size_t wle_scratch_bytes(int n) {
    const size_t nn = (size_t)(n > 0 ? n : 1);
    return 2 * align256(nn * 8) + 2 * align256(nn * 4) + align256(sort_temp_bytes((int)nn)) + align256(sizeof(int));
}

cudaError_t launch_wle(const uint16_t *rois, int n, int R, int loc_type, float *wle, void *scratch, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int tpb = 64;
    const int grid = (n + tpb - 1) / tpb;
    const Span sp{0, n, nullptr};
    cudaError_t e = launch_psf_width(R, rois, wle, sp, grid, tpb, s);
    if (e != cudaSuccess) return e;
    const size_t nn = (size_t)n;
    char *p = static_cast<char *>(scratch);
    unsigned long long *k_in = reinterpret_cast<unsigned long long *>(p);
    p += align256(nn * 8);
    unsigned long long *k_out = reinterpret_cast<unsigned long long *>(p);
    p += align256(nn * 8);
    int *v_in = reinterpret_cast<int *>(p);
    p += align256(nn * 4);
    int *v_out = reinterpret_cast<int *>(p);
    p += align256(nn * 4);
    size_t temp = sort_temp_bytes(n);
    const int whole = R * (R + 1);
    nn_keys_kernel<<<grid, tpb, 0, s>>>(rois, n, whole, R * R, k_in, v_in);
    e = cub::DeviceRadixSort::SortPairs(p, temp, k_in, k_out, v_in, v_out, n, 0, 64, s);
    if (e != cudaSuccess) return e;
    nn_scan_kernel<<<grid, tpb, 0, s>>>(k_out, v_out, n, wle);
    classify_kernel<<<grid, tpb, 0, s>>>(rois, wle, sp, R, whole, loc_type);
    return cudaGetLastError();
}

namespace {

// Keys of records [0, n) and padding (all ones, after every real key) up to
// cap; *unsorted = 1 when some record's key is below its predecessor's.
__global__ void nn_keys_flag_kernel(const uint16_t *__restrict__ rois, int n, int cap, int whole, int pix,
                                    unsigned long long *__restrict__ keys, int *__restrict__ vals,
                                    int *__restrict__ unsorted) {
    const int i = threadIdx.x + blockDim.x * blockIdx.x;
    bool bad = false;
    if (i < cap) {
        unsigned long long k = ~0ull;
        if (i < n) {
            const uint16_t *h = rois + (size_t)i * whole + pix;
            k = (((unsigned long long)h[2] + 65536ull * h[3]) << 32) | ((unsigned long long)h[1] << 16) | h[0];
            if (i > 0) {
                const uint16_t *g = h - whole;
                const unsigned long long kp =
                    (((unsigned long long)g[2] + 65536ull * g[3]) << 32) | ((unsigned long long)g[1] << 16) | g[0];
                bad = kp > k;
            }
        }
        keys[i] = k;
        vals[i] = i;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(unsorted, 1);
}

// Sets the sort's IF condition from the flag of nn_keys_flag_kernel.
__global__ void wle_sort_cond_kernel(cudaGraphConditionalHandle h, const int *__restrict__ unsorted) {
    cudaGraphSetConditional(h, *unsorted ? 1u : 0u);
}

// nn_scan_kernel over the sorted keys when the records were out of order,
// else over the records' own keys (already sorted, identity order).
__global__ void nn_scan_select_kernel(const unsigned long long *__restrict__ k_in, const unsigned long long *__restrict__ k_out,
                                      const int *__restrict__ v_out, const int *__restrict__ unsorted, int n,
                                      float *__restrict__ wle) {
    const int a = threadIdx.x + blockDim.x * blockIdx.x;
    if (a >= n) return;
    if (*unsorted)
        wle[(size_t)v_out[a] * QCS_WLE_PARA_NUM + 0] = nn_sorted(k_out, a, n);
    else
        wle[(size_t)a * QCS_WLE_PARA_NUM + 0] = nn_sorted(k_in, a, n);
}

}  // namespace

// The WLE pre-pass of a localization context.  Records produced by ROI
// extraction (and most callers' batches) are already in (frame, y, x)
// order; then the radix sort of the nearest-neighbour keys is the identity
// and only costs time.  Here the keys kernel flags out-of-order records and
// a CUDA graph holds the sort inside an IF node whose condition a one-thread
// kernel sets from that flag, so the sort runs only when needed and the host
// never waits.  The sort covers `capacity` keys (padding sorts last).
struct WleSorter {
    int capacity = 0;
    void *scratch = nullptr;  // wle_scratch_bytes(capacity), owned by the caller
    unsigned long long *k_in = nullptr, *k_out = nullptr;
    int *v_in = nullptr, *v_out = nullptr, *flag = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

void wle_sorter_destroy(WleSorter *w) {
    if (!w) return;
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    if (w->cap) cudaStreamDestroy(w->cap);
    delete w;
}

cudaError_t wle_sorter_create(int capacity, void *scratch, WleSorter **out) {
    *out = nullptr;
    WleSorter *w = new WleSorter();
    w->capacity = capacity;
    w->scratch = scratch;
    const size_t nn = (size_t)capacity;
    char *p = static_cast<char *>(scratch);
    w->k_in = reinterpret_cast<unsigned long long *>(p);
    p += align256(nn * 8);
    w->k_out = reinterpret_cast<unsigned long long *>(p);
    p += align256(nn * 8);
    w->v_in = reinterpret_cast<int *>(p);
    p += align256(nn * 4);
    w->v_out = reinterpret_cast<int *>(p);
    p += align256(nn * 4);
    void *temp = p;
    size_t temp_bytes = sort_temp_bytes(capacity);
    p += align256(temp_bytes);
    w->flag = reinterpret_cast<int *>(p);

    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t kn = nullptr, cn = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&w->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaGraphCreate(&w->graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, w->graph, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        cudaKernelNodeParams kp = {};
        const int *flag = w->flag;
        void *args[] = {&h, &flag};
        kp.func = reinterpret_cast<void *>(wle_sort_cond_kernel);
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(1);
        kp.sharedMemBytes = 0;
        kp.kernelParams = args;
        e = cudaGraphAddKernelNode(&kn, w->graph, nullptr, 0, &kp);
    }
    cudaGraph_t body = nullptr;
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&cn, w->graph, &kn, 1, &cp);
        if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
    }
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(w->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        cudaError_t es = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, w->k_in, w->k_out, w->v_in, w->v_out,
                                                         capacity, 0, 64, w->cap);
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(w->cap, &captured);
        if (e == cudaSuccess) e = es;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&w->exec, w->graph, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        wle_sorter_destroy(w);
        return e;
    }
    *out = w;
    return cudaSuccess;
}

cudaError_t launch_wle_ctx(WleSorter *w, const uint16_t *rois, int n, int R, int loc_type, float *wle,
                           cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return e;
    if (n > w->capacity || cs != cudaStreamCaptureStatusNone)
        return launch_wle(rois, n, R, loc_type, wle, w->scratch, s);
    const int tpb = 64;
    const int grid = (n + tpb - 1) / tpb;
    const Span sp{0, n, nullptr};
    e = launch_psf_width(R, rois, wle, sp, grid, tpb, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(w->flag, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    const int whole = R * (R + 1);
    nn_keys_flag_kernel<<<(w->capacity + tpb - 1) / tpb, tpb, 0, s>>>(rois, n, w->capacity, whole, R * R, w->k_in,
                                                                      w->v_in, w->flag);
    e = cudaGraphLaunch(w->exec, s);
    if (e != cudaSuccess) return e;
    nn_scan_select_kernel<<<grid, tpb, 0, s>>>(w->k_in, w->k_out, w->v_out, w->flag, n, wle);
    classify_kernel<<<grid, tpb, 0, s>>>(rois, wle, sp, R, whole, loc_type);
    return cudaGetLastError();
}

cudaError_t launch_wle_presorted(const uint16_t *rois, const unsigned long long *keys, const int *d_span, int max_n,
                                 int R, int loc_type, float *wle, cudaStream_t s) {
    if (max_n <= 0) return cudaSuccess;
    const int tpb = 64;
    int grid = (max_n + tpb - 1) / tpb;
    if (grid > 148 * 8) grid = 148 * 8;
    const Span sp{0, 0, d_span};
    switch (R) {
    case 5: wle_sorted_kernel<5><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 7: wle_sorted_kernel<7><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 9: wle_sorted_kernel<9><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 11: wle_sorted_kernel<11><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 13: wle_sorted_kernel<13><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 15: wle_sorted_kernel<15><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    case 17: wle_sorted_kernel<17><<<grid, tpb, 0, s>>>(rois, keys, sp, wle, loc_type); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace qcs
