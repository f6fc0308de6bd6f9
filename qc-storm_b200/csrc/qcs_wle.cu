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

template <int R>
__global__ void psf_width_kernel(const uint16_t *__restrict__ rois, float *__restrict__ wle, int n) {
    enum { Len = R, ILen = (R - 1) * kInterp + 1, WHOLE = R * (R + 1) };
    const int gid = threadIdx.x + blockDim.x * blockIdx.x;
    if (gid >= n) return;
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

// Minimum squared distance to another ROI of the same frame, scanning the
// sorted order both ways until the row distance alone exceeds the best.
__global__ void nn_scan_kernel(const unsigned long long *__restrict__ keys, const int *__restrict__ vals, int n,
                               float *__restrict__ wle) {
    const int a = threadIdx.x + blockDim.x * blockIdx.x;
    if (a >= n) return;
    const unsigned long long ka = keys[a];
    const unsigned long long frame = ka >> 32;
    const int ya = (int)((ka >> 16) & 0xFFFF), xa = (int)(ka & 0xFFFF);
    float best = 100000000.0f;
    for (int b = a + 1; b < n; b++) {
        const unsigned long long kb = keys[b];
        if ((kb >> 32) != frame) break;
        const int dy = (int)((kb >> 16) & 0xFFFF) - ya, dx = (int)(kb & 0xFFFF) - xa;
        if ((float)(dy * dy) > best) break;
        best = fminf(best, (float)(dx * dx + dy * dy));
    }
    for (int b = a - 1; b >= 0; b--) {
        const unsigned long long kb = keys[b];
        if ((kb >> 32) != frame) break;
        const int dy = (int)((kb >> 16) & 0xFFFF) - ya, dx = (int)(kb & 0xFFFF) - xa;
        if ((float)(dy * dy) > best) break;
        best = fminf(best, (float)(dx * dx + dy * dy));
    }
    wle[(size_t)vals[a] * QCS_WLE_PARA_NUM + 0] = sqrtf(best);
}

__global__ void classify_kernel(const uint16_t *__restrict__ rois, float *__restrict__ wle, int n, int R, int whole,
                                int LocType) {
    const int gid = threadIdx.x + blockDim.x * blockIdx.x;
    if (gid >= n) return;
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
    return 2 * align256(nn * 8) + 2 * align256(nn * 4) + align256(sort_temp_bytes((int)nn));
}

cudaError_t launch_wle(const uint16_t *rois, int n, int R, int loc_type, float *wle, void *scratch, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int tpb = 64;
    const int grid = (n + tpb - 1) / tpb;
    switch (R) {
    case 5: psf_width_kernel<5><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 7: psf_width_kernel<7><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 9: psf_width_kernel<9><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 11: psf_width_kernel<11><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 13: psf_width_kernel<13><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 15: psf_width_kernel<15><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    case 17: psf_width_kernel<17><<<grid, tpb, 0, s>>>(rois, wle, n); break;
    default: return cudaErrorInvalidValue;
    }
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
    cudaError_t e = cub::DeviceRadixSort::SortPairs(p, temp, k_in, k_out, v_in, v_out, n, 0, 64, s);
    if (e != cudaSuccess) return e;
    nn_scan_kernel<<<grid, tpb, 0, s>>>(k_out, v_out, n, wle);
    classify_kernel<<<grid, tpb, 0, s>>>(rois, wle, n, R, whole, loc_type);
    return cudaGetLastError();
}

}  // namespace qcs
