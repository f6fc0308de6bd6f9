// Diagnostic kernel: sustained rate of the special-function unit (MUFU) for
// the two transcendental intrinsics of the fit loss, __expf and __logf, used
// as the measured peak of the fit kernel's roofline.  Each thread runs eight
// independent log -> scale -> exp chains (two MUFU operations per link).
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"

namespace {

__global__ void mufu_rate_kernel(float *out, int iters, float scale) {
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = 1.5f + 0.01f * (threadIdx.x & 7) + 0.1f * k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = __expf(__logf(v[k]) * scale);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += v[k];
    if (s == 12345.0f) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int qcs_measure_mufu_rate(int iters, float *ms, double *ops) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return QCS_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256;
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * threads) != cudaSuccess) return QCS_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    mufu_rate_kernel<<<blocks, threads>>>(d, iters / 10 + 1, 0.9999f);  // warm-up
    cudaEventRecord(e0);
    mufu_rate_kernel<<<blocks, threads>>>(d, iters, 0.9999f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) return QCS_ERR_CUDA;
    *ms = t;
    *ops = 2.0 * 8.0 * (double)iters * blocks * threads;
    return QCS_OK;
}
