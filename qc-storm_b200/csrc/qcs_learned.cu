// Learned start points for the single-emitter fits (GS2D and AS3D, 7x7, 9x9
// and 11x11 ROIs): a small network predicts each ROI's optimum from its
// pixels, so that the BFGS fit can start near it and run fewer iterations.
// No counterpart in the reference (it starts from the centre / edge-mean
// pre-estimates, bfgsMLE_GS2D_core.h:522-575, bfgsMLE_AS3D_core.h:548-607).
//
// Network (per ROI): 64 (7x7) or 128 (9x9, 11x11) features -> 128 (ReLU) ->
// 128 (ReLU) -> 8 outputs: GS2D dx, dy, sigma - 1.3, log(peak / range),
// (background - min) / range, and three logits of the ROI's emitter-count
// class (0: one emitter; 1: the two-emitter fit's stage; 2: the three-emitter
// fit's stage), with which the multi-emitter cascade sends a ROI straight to
// the stage it would reach; AS3D dx, dy, sigma_x - 1.3, log(peak / range),
// (background - min) / range, sigma_y - 1.3.
// Features: the R*R photoelectron pixels max((adu - offset) * gain, 1) scaled
// to [0, 1] by the ROI's min and range, log(range) / 8, log(min) / 8, zeros.
// Training and inference GEMMs run on the tensor cores (tcgen05) in BF16 with
// FP32 accumulation; master weights and Adam moments are FP32.
// Labels are the converged plain MLEbfgs fits of the same ROIs.
#include <cstdint>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"
#include "qcs_kernels.h"
#include "qcs_learned.h"
#include "qcs_tc.cuh"

namespace qcs {
namespace learned {

constexpr int kGemmThreads = 128;  // 4 warps: one tcgen05 GEMM tile of 128 rows

// One feature of record r (R x R pixels then header words): feature k of
// in_width(R), given the record's photoelectron min lo, 1 / range inv and the
// two scale features.  The fused inference kernel builds the same values.
template <int R>
__device__ __forceinline__ float feature(const uint16_t *r, int k, float offset, float kadc, float lo, float inv,
                                         float f_rng, float f_lo) {
    enum { PIX = R * R };
    if (k < PIX) return (fmaxf(((float)r[k] - offset) * kadc, 1.0f) - lo) * inv;
    if (k == PIX) return f_rng;
    if (k == PIX + 1) return f_lo;
    return 0.0f;
}

// photoelectron min and range of a record's R x R pixels
template <int R>
__device__ __forceinline__ void record_range(const uint16_t *r, float offset, float kadc, float &lo, float &rng) {
    float hi = -1e30f;
    lo = 1e30f;
#pragma unroll
    for (int k = 0; k < R * R; ++k) {
        const float e = fmaxf(((float)r[k] - offset) * kadc, 1.0f);
        lo = fminf(lo, e);
        hi = fmaxf(hi, e);
    }
    rng = fmaxf(hi - lo, 1.0f);
}

// ---------------------------------------------------------------- features
template <int R>
__global__ void features_kernel(const uint16_t *__restrict__ rois, int n, float offset, float kadc,
                                float *__restrict__ feat, float *__restrict__ scale) {
    enum { KIN = in_width(R), WHOLE = R * (R + 1) };
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint16_t *r = rois + (size_t)i * WHOLE;
    float lo, rng;
    record_range<R>(r, offset, kadc, lo, rng);
    const float inv = 1.0f / rng;
    const float f_rng = logf(rng) * 0.125f, f_lo = logf(lo) * 0.125f;
    float *f = feat + (size_t)i * KIN;
    for (int k = 0; k < KIN; ++k) f[k] = feature<R>(r, k, offset, kadc, lo, inv, f_rng, f_lo);
    scale[2 * i] = lo;
    scale[2 * i + 1] = rng;
}

// Targets (used_outputs(LT) per record) from the plain fit rows (12 floats
// per record, record order); valid[i] = 1 for accepted fits.
template <int R, int LT>
__global__ void targets_kernel(const uint16_t *__restrict__ rois, const float *__restrict__ rows,
                               const float *__restrict__ scale, int n, float qe, float *__restrict__ tgt,
                               float *__restrict__ valid) {
    enum { PIX = R * R, WHOLE = R * (R + 1), HALF = R / 2, NU = used_outputs(LT) };
    const float centre = R / 2.0f;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *row = rows + (size_t)i * 12;
    const uint16_t *h = rois + (size_t)i * WHOLE + PIX;
    const float lo = scale[2 * i], rng = scale[2 * i + 1];
    const bool ok = row[QCS_POS_PPHO] > 0.0f && row[QCS_POS_SIGX] > 0.0f;
    float *t = tgt + (size_t)i * NU;
    if (ok) {
        // ROI coordinates of the fitted centre (inverse of the row's x = fit - R/2 + header x)
        t[0] = row[QCS_POS_XPOS] + (float)HALF - (float)h[0] - centre;
        t[1] = row[QCS_POS_YPOS] + (float)HALF - (float)h[1] - centre;
        t[2] = row[QCS_POS_SIGX] - kSigma0;
        t[3] = logf(fmaxf(row[QCS_POS_PPHO] * qe, 1e-3f) / rng);
        t[4] = (row[QCS_POS_BAKG] * qe - lo) / rng;
        if (NU > 5) t[5] = row[QCS_POS_SIGY] - kSigma0;
    } else {
#pragma unroll
        for (int j = 0; j < NU; ++j) t[j] = 0.0f;
    }
    valid[i] = ok ? 1.0f : 0.0f;
}

// ------------------------------------------------------------------- GEMM
// C(m, n) = beta * C(m, n) + sum_k A(m, k) B(k, n), M x N x K, with
// A(m, k) = A[m * sam + k * sak], B(k, n) = B[k * sbk + n * sbn] (FP32 in
// memory, rounded to BF16 for the tensor cores), C row-major with ldc.
// One CTA of 128 threads per 128 x bn tile (bn <= 256, a multiple of 16) and
// K range: the threads stage 64-deep K chunks of both operands into shared
// memory in the UMMA layout (double-buffered), one thread issues four
// tcgen05.mma (M = 128, K = 16) per chunk into an FP32 accumulator in tensor
// memory, and each warp reads its 32 rows back with tcgen05.ld.  With split-K
// (gridDim.z > 1) CTA z sums K range [z kper, (z + 1) kper) into
// part[z][M][N] and gemm_reduce_kernel adds the splits in order, so results
// do not depend on scheduling.
constexpr int kGemmM = 128, kGemmK = 64;

__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_tc_kernel(int M, int N, int K, int bn, const float *__restrict__ A, long long sam, long long sak,
                   const float *__restrict__ B, long long sbk, long long sbn, float *__restrict__ Cm, int ldc,
                   float beta, int kper, float *__restrict__ part, int *__restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t sbase = (raw + 127u) & ~127u;
    uint8_t *base = smem_raw + (sbase - raw);
    const uint32_t a_bytes = kGemmM * kGemmK * 2, b_bytes = (uint32_t)bn * kGemmK * 2;
    const uint32_t sA = sbase, sB = sbase + 2 * a_bytes, sBar = sB + 2 * b_bytes, sTmem = sBar + 16;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kGemmM, n0 = blockIdx.x * bn;
    const int kb = blockIdx.z * kper, ke = min(K, kb + kper);
    const int nchunks = ke > kb ? (ke - kb + kGemmK - 1) / kGemmK : 0;
    uint32_t cols = 32;
    while ((int)cols < bn) cols <<= 1;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sBar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sBar + 8) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sTmem), "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(base + (sTmem - sbase));
    const uint32_t idesc = tc::instr_desc(kGemmM, bn);
    bool ok = true;
    int issued = 0;  // chunks whose MMAs were issued
    for (int c = 0; c < nchunks; ++c) {
        const int buf = c & 1, k0 = kb + c * kGemmK;
        if (c >= 2) {  // the MMAs of chunk c - 2 have read this buffer
            ok = __syncthreads_and(tc::mbar_wait(sBar + 8 * buf, ((c - 2) >> 1) & 1));
            if (!ok) break;
        }
        uint8_t *a_img = base + buf * a_bytes, *b_img = base + 2 * a_bytes + buf * b_bytes;
        // A: row tid, K groups 0..7 of the chunk
        const int gm = m0 + tid;
#pragma unroll
        for (int kg = 0; kg < kGemmK / 8; ++kg) {
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int gk = k0 + kg * 8 + e;
                v[e] = (gm < M && gk < ke) ? __ldg(A + (long long)gm * sam + (long long)gk * sak) : 0.0f;
            }
            *reinterpret_cast<uint4 *>(a_img + (size_t)(kg * kGemmM + tid) * 16) = tc::pack8(v);
        }
        // B: bn rows (n) x 8 K groups
#pragma unroll 4
        for (int u = tid; u < bn * (kGemmK / 8); u += kGemmThreads) {
            const int kg = u / bn, nn = u - kg * bn, gn = n0 + nn;
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int gk = k0 + kg * 8 + e;
                v[e] = (gn < N && gk < ke) ? __ldg(B + (long long)gk * sbk + (long long)gn * sbn) : 0.0f;
            }
            *reinterpret_cast<uint4 *>(b_img + (size_t)(kg * bn + nn) * 16) = tc::pack8(v);
        }
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (tid == 0) {
            const uint32_t a0 = sA + buf * a_bytes, b0 = sB + buf * b_bytes;
#pragma unroll
            for (int ks = 0; ks < kGemmK / 16; ++ks)
                tc::mma_bf16(tmem, tc::smem_desc(a0 + ks * 2 * kGemmM * 16, kGemmM * 16, 128),
                             tc::smem_desc(b0 + ks * 2 * bn * 16, bn * 16, 128), idesc, (c > 0 || ks > 0) ? 1u : 0u);
            tc::mma_commit(sBar + 8 * buf);
        }
        issued = c + 1;
    }
    // the last commit covers every MMA issued before it; after a wait gave up
    // this (bounded) wait still lets the issued MMAs end before the memory is released
    if (issued > 0) {
        const bool done = __syncthreads_and(tc::mbar_wait(sBar + 8 * ((issued - 1) & 1), ((issued - 1) >> 1) & 1));
        ok = ok && done;
    }
    tc::fence_after();
    if (ok) {
        // 64 columns at a time through shared memory (the operand buffers are
        // free once the last MMA has ended): each thread stores its row, then
        // each warp writes whole rows, lanes along the columns (coalesced)
        float *stage = reinterpret_cast<float *>(base);  // [128][65]
        float *out = part ? part + (size_t)blockIdx.z * M * N : Cm;
        const long long ld = part ? N : ldc;
        const float b = part ? 0.0f : beta;
        for (int c0 = 0; c0 < bn; c0 += 64) {
#pragma unroll
            for (int q = 0; q < 64; q += 16) {
                float v[16];
                if (issued > 0) {
                    tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0 + q, v);
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = 0.0f;
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) stage[tid * 65 + q + j] = v[j];
            }
            __syncthreads();
            for (int r = warp * 32; r < warp * 32 + 32; ++r) {
                const int row = m0 + r;
                if (row >= M) break;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = c0 + h * 32 + lane, col = n0 + c;
                    if (c < bn && col < N) {
                        float *dst = out + (size_t)row * ld + col;
                        const float v = stage[r * 65 + h * 32 + lane];
                        *dst = (b == 0.0f) ? v : b * (*dst) + v;
                    }
                }
            }
            __syncthreads();
        }
    } else if (tid == 0 && err) {
        atomicExch(err, 1);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// C = beta C + sum over the splits z = 0, 1, ... of part[z] (in that order).
__global__ void gemm_reduce_kernel(const float *__restrict__ part, int splits, int M, int N, float *__restrict__ Cm,
                                   int ldc, float beta) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * N) return;
    const int r = (int)(i / N), c = (int)(i - (long long)r * N);
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * M * N + i];
    float *dst = Cm + (size_t)r * ldc + c;
    *dst = (beta == 0.0f) ? s : beta * (*dst) + s;
}

size_t gemm_smem_bytes(int bn) { return 2 * (size_t)(kGemmM + bn) * kGemmK * 2 + 32 + 128; }

// Split count for an M x N x K GEMM: enough CTAs to cover the SMs, at least
// four K chunks per split, and partials within `ws_floats`.
int gemm_splits(int M, int N, int K, int bn, size_t ws_floats) {
    const int tiles = ((M + kGemmM - 1) / kGemmM) * ((N + bn - 1) / bn);
    int s = 148 / tiles;
    const int by_k = K / (4 * kGemmK);
    if (s > by_k) s = by_k;
    if (s > 64) s = 64;
    while (s > 1 && (size_t)s * M * N > ws_floats) --s;
    return s < 1 ? 1 : s;
}

cudaError_t gemm(int M, int N, int K, const float *A, long long sam, long long sak, const float *B, long long sbk,
                 long long sbn, float *C, int ldc, float beta, cudaStream_t s, float *ws, size_t ws_floats, int *err) {
    if (M <= 0 || N <= 0) return cudaSuccess;
    int bn = ((N + 15) / 16) * 16;
    if (bn > 256) bn = 256;
    const int splits = ws ? gemm_splits(M, N, K, bn, ws_floats) : 1;
    int kper = (K + splits - 1) / splits;
    kper = ((kper + kGemmK - 1) / kGemmK) * kGemmK;
    const int z = kper > 0 ? (K + kper - 1) / kper : 1;
    const size_t smem = gemm_smem_bytes(bn);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gemm_smem_bytes(256));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grid((N + bn - 1) / bn, (M + kGemmM - 1) / kGemmM, z > 1 ? z : 1);
    float *part = z > 1 ? ws : nullptr;
    gemm_tc_kernel<<<grid, kGemmThreads, smem, s>>>(M, N, K, bn, A, sam, sak, B, sbk, sbn, C, ldc, beta,
                                                    z > 1 ? kper : (K > 0 ? K : 0), part, err);
    if (z > 1)
        gemm_reduce_kernel<<<(int)(((long long)M * N + 255) / 256), 256, 0, s>>>(part, z, M, N, C, ldc, beta);
    return cudaGetLastError();
}

// ------------------------------------------------------ elementwise layers
// Z (rows x cols) += bias; A = relu(Z) (A may alias Z when the caller does not need Z).
__global__ void bias_relu_kernel(float *__restrict__ Z, const float *__restrict__ bias, int rows, int cols,
                                 float *__restrict__ A, int relu) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)rows * cols) return;
    const float z = Z[i] + bias[i % cols];
    Z[i] = z;
    A[i] = relu ? fmaxf(z, 0.0f) : z;
}

// dZ = dA * (Z > 0)
__global__ void relu_back_kernel(float *__restrict__ dA, const float *__restrict__ Z, long long total) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    if (!(Z[i] > 0.0f)) dA[i] = 0.0f;
}

// Column sums of d (rows x cols), two passes with a fixed order: block
// (x, z) sums split z's rows of 32 columns into part[z][cols]; then
// colsum_final adds the splits in order.
__global__ void colsum_part_kernel(const float *__restrict__ d, long long rows, int cols, float *__restrict__ part) {
    __shared__ float acc[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    const long long per = (rows + gridDim.y - 1) / gridDim.y;
    const long long r0 = (long long)blockIdx.y * per, r1 = r0 + per < rows ? r0 + per : rows;
    float s = 0.0f;
    if (c < cols)
        for (long long r = r0 + threadIdx.y; r < r1; r += 8) s += d[r * cols + c];
    acc[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) t += acc[k][threadIdx.x];
        part[(size_t)blockIdx.y * cols + c] = t;
    }
}

__global__ void colsum_final_kernel(const float *__restrict__ part, int splits, int cols, float *__restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * cols + c];
    g[c] = s;
}

cudaError_t column_sums(const float *d, long long rows, int cols, float *g, float *part, cudaStream_t s) {
    int splits = (int)((rows + 255) / 256);
    if (splits > kColsumSplits) splits = kColsumSplits;
    if (splits < 1) splits = 1;
    colsum_part_kernel<<<dim3((cols + 31) / 32, splits), dim3(32, 8), 0, s>>>(d, rows, cols, part);
    colsum_final_kernel<<<(cols + 127) / 128, 128, 0, s>>>(part, splits, cols, g);
    return cudaGetLastError();
}

// Masked weighted MSE on the first nused outputs plus, where cls is set and
// cls[i] >= 0 (GS2D networks), kCountWeight x the softmax cross-entropy of
// the count logits against class cls[i]: loss and dY.
__global__ void mse_kernel(const float *__restrict__ Y, const float *__restrict__ T, const float *__restrict__ valid,
                           const float *__restrict__ cls, int rows, int nout, int nused, int wrow, float inv_count,
                           float *__restrict__ dY,
                           float *__restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const float v = valid[i];
    const float *y = Y + (size_t)i * nout;
    float l = 0.0f;
    for (int j = 0; j < nout; ++j) {
        float d = 0.0f;
        if (j < nused) {
            const float e = y[j] - T[(size_t)i * nused + j];
            d = 2.0f * kTargetWeight[wrow][j] * e * v * inv_count;
            l += kTargetWeight[wrow][j] * e * e * v;
        }
        dY[(size_t)i * nout + j] = d;
    }
    const int label = cls ? (int)cls[i] : -1;
    if (label >= 0 && label < kClasses) {
        const float l0 = y[kCount0], l1 = y[kCount0 + 1], l2 = y[kCount0 + 2];
        const float m = fmaxf(l0, fmaxf(l1, l2));
        const float e[kClasses] = {expf(l0 - m), expf(l1 - m), expf(l2 - m)};
        const float sum = e[0] + e[1] + e[2];
        l += kCountWeight * (logf(sum) - (y[kCount0 + label] - m));
#pragma unroll
        for (int j = 0; j < kClasses; ++j)
            dY[(size_t)i * nout + kCount0 + j] = kCountWeight * (e[j] / sum - (j == label ? 1.0f : 0.0f)) * inv_count;
    }
    atomicAdd(loss, l * inv_count);
}

__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int n, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

__global__ void gather_rows_kernel(const float *__restrict__ src, const int *__restrict__ idx, int rows, int cols,
                                   float *__restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)rows * cols) return;
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    dst[i] = src[(size_t)idx[r] * cols + c];
}

// Predictions -> fit start and, with cls set (GS2D), the emitter-count class
// at threshold th.
template <int R, int LT>
__global__ void start_kernel(const float *__restrict__ Y, const float *__restrict__ scale, int n,
                             float *__restrict__ start, uint8_t *__restrict__ cls, float th) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *y = Y + (size_t)i * out_width(LT);
    if (cls) cls[i] = (uint8_t)count_class(y[kCount0], y[kCount0 + 1], y[kCount0 + 2], th);
    start_from_outputs<R, LT>(y, scale[2 * i], scale[2 * i + 1], start + (size_t)i * start_width(LT));
}

// ------------------------------------------- fused tcgen05 inference ---
// One persistent CTA of 128 threads per 128-ROI tile: features -> layer 1 ->
// ReLU -> layer 2 -> ReLU -> layer 3 -> start point, with every activation
// kept on chip.  The three GEMMs are tcgen05.mma (M = 128, kind::f16, BF16
// operands in shared memory, FP32 accumulators in tensor memory), issued by
// one thread and completed through an mbarrier; each warp reads its 32
// accumulator rows back with tcgen05.ld.
namespace tc {

constexpr int kM = 128;        // ROIs per tile (the MMA's M)
constexpr int kN3 = 16;        // layer-3 N padded to the M = 128 minimum
constexpr int kAlign = 128;
constexpr int kTmemCols = 256;                     // layer 1 / 3 at column 0, layer 2 at column 128

// Shared memory of one CTA for R x R records and KIN features: the weight
// images, the layer-2 operand (the layer-1 operand lives in its first part:
// layer 1's MMA has finished reading it before the layer-1 epilogue writes
// layer 2's operand), one tile of records, barriers.
template <int R>
struct Layout {
    enum : int {
        KIN = in_width(R),
        WHOLE = R * (R + 1),
        W1 = kHidden * KIN, W2 = kHidden * kHidden, W3 = kN3 * kHidden,  // bf16 elements
        REC_BYTES = kM * WHOLE * 2,                                         // one tile of records
        OFF_W1 = 0,
        OFF_W2 = OFF_W1 + W1 * 2,
        OFF_W3 = OFF_W2 + W2 * 2,
        OFF_A2 = OFF_W3 + W3 * 2,
        OFF_A1 = OFF_A2,
        OFF_REC = OFF_A2 + kM * kHidden * 2,
        OFF_BAR = OFF_REC + REC_BYTES,  // MMA barrier, record barrier, TMEM address
        SMEM = OFF_BAR + 32 + kAlign,   // + alignment slack
        WEIGHT_VEC = (W1 + W2 + W3) * 2 / 16,
    };
    static_assert(OFF_A1 + kM * KIN * 2 <= OFF_REC, "layer-1 operand inside the layer-2 buffer");
    static_assert(REC_BYTES % 16 == 0 && OFF_REC % 16 == 0, "a full tile is a whole number of 16-byte blocks");
};

// Relu(D + bias) of this thread's accumulator row (ncols columns from tmem
// column col0) into the next layer's A operand (row tid).
__device__ __forceinline__ void epilogue_hidden(uint32_t taddr_row, const float *__restrict__ bias, uint8_t *a_next,
                                                int tid) {
#pragma unroll 1
    for (int c0 = 0; c0 < kHidden; c0 += 16) {
        float v[16];
        tmem_ld16(taddr_row + c0, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + __ldg(bias + c0 + j), 0.0f);
        *reinterpret_cast<uint4 *>(a_next + (size_t)((c0 >> 3) * kM + tid) * 16) = pack8(v);
        *reinterpret_cast<uint4 *>(a_next + (size_t)(((c0 >> 3) + 1) * kM + tid) * 16) = pack8(v + 8);
    }
}

__device__ __forceinline__ int tile_rows(int tile, int n) { return min(kM, n - tile * kM); }

// bytes of a tile's records moved by the bulk copy (a multiple of 16; the
// rest, under 16 bytes of a ragged last tile, is copied by plain loads)
template <int R>
__device__ __forceinline__ uint32_t bulk_bytes(int rows) {
    return (uint32_t)(rows * R * (R + 1) * 2) & ~15u;
}

// BULK: records reach shared memory by one bulk copy per tile, issued one
// tile ahead (d_rois 16-byte aligned); otherwise each thread reads its own
// record from global memory.  LT: the start point's kind (GS2D / AS3D).
template <bool BULK, int R, int LT>
__global__ void __launch_bounds__(128, 1) mlp_tc_kernel(const uint16_t *__restrict__ rois, int n, float offset,
                                                        float kadc, const uint4 *__restrict__ wimg,
                                                        const float *__restrict__ b1, const float *__restrict__ b2,
                                                        const float *__restrict__ b3, float *__restrict__ start,
                                                        uint8_t *__restrict__ cls, float count_th,
                                                        const int *__restrict__ n_dev, int *__restrict__ err) {
    typedef Layout<R> L;
    enum { KIN = L::KIN, WHOLE = L::WHOLE, NST = start_width(LT) };
    extern __shared__ uint8_t smem_raw[];
    if (n_dev) n = min(max(*n_dev, 0), n);  // record count on the device, at most n
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t sbase = (raw + (kAlign - 1)) & ~(uint32_t)(kAlign - 1);
    uint8_t *base = smem_raw + (sbase - raw);
    const uint32_t sW1 = sbase + L::OFF_W1, sW2 = sbase + L::OFF_W2, sW3 = sbase + L::OFF_W3;
    const uint32_t sA1 = sbase + L::OFF_A1, sA2 = sbase + L::OFF_A2, sRec = sbase + L::OFF_REC;
    const uint32_t sBar = sbase + L::OFF_BAR, sRecBar = sBar + 8, sTmem = sBar + 16;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ntiles = (n + kM - 1) / kM;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sBar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sRecBar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (BULK && (int)blockIdx.x < ntiles)
            bulk_load(sRec, rois + (size_t)blockIdx.x * kM * WHOLE, bulk_bytes<R>(tile_rows(blockIdx.x, n)), sRecBar);
    }
    uint4 *wdst = reinterpret_cast<uint4 *>(base + L::OFF_W1);
    for (int i = tid; i < L::WEIGHT_VEC; i += blockDim.x) wdst[i] = wimg[i];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sTmem), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(base + L::OFF_BAR + 16);
    const uint32_t row_lane = (uint32_t)(warp * 32) << 16;
    uint32_t phase = 0, rec_phase = 0;
    bool ok = true, copy_pending = BULK && (int)blockIdx.x < ntiles;
    uint16_t *srec = reinterpret_cast<uint16_t *>(base + L::OFF_REC);
    int tile = blockIdx.x;
    for (; tile < ntiles; tile += gridDim.x) {
        const int i = tile * kM + tid;
        const int rows = tile_rows(tile, n);
        if (BULK) {
            ok = __syncthreads_and(mbar_wait(sRecBar, rec_phase));
            if (!ok) break;  // rec_phase still names the copy in flight
            rec_phase ^= 1u;
            copy_pending = false;
            const int copied = (int)bulk_bytes<R>(rows) / 2, total = rows * WHOLE;
            if (copied < total) {  // the ragged last tile's last few words (same for every thread)
                if (tid < total - copied) srec[copied + tid] = rois[(size_t)tile * kM * WHOLE + copied + tid];
                __syncthreads();
            }
        }
        // features of this thread's ROI into A1 (row tid)
        float lo = 1.0f, rng = 1.0f;
        if constexpr (R == 7) {
            // 7x7: the 56-word record in registers (seven 16-byte loads from
            // shared memory), features in one pass
            float f[KIN];
#pragma unroll
            for (int k = 0; k < KIN; ++k) f[k] = 0.0f;
            if (tid < rows) {
                uint16_t px[WHOLE];
                if (BULK) {
                    const uint4 *r4 = reinterpret_cast<const uint4 *>(srec + (size_t)tid * WHOLE);
#pragma unroll
                    for (int q = 0; q < WHOLE / 8; ++q) {
                        const uint4 u = r4[q];
                        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                        for (int h = 0; h < 4; ++h) {
                            px[q * 8 + 2 * h] = (uint16_t)(w[h] & 0xFFFFu);
                            px[q * 8 + 2 * h + 1] = (uint16_t)(w[h] >> 16);
                        }
                    }
                } else {
                    const uint16_t *r = rois + (size_t)i * WHOLE;
#pragma unroll
                    for (int k = 0; k < R * R; ++k) px[k] = r[k];
                }
                record_range<R>(px, offset, kadc, lo, rng);
                const float inv = 1.0f / rng;
                const float f_rng = logf(rng) * 0.125f, f_lo = logf(lo) * 0.125f;
#pragma unroll
                for (int k = 0; k < R * R + 2; ++k) f[k] = feature<R>(px, k, offset, kadc, lo, inv, f_rng, f_lo);
            }
#pragma unroll
            for (int kg = 0; kg < KIN / 8; ++kg)
                *reinterpret_cast<uint4 *>(base + L::OFF_A1 + (size_t)(kg * kM + tid) * 16) = pack8(f + 8 * kg);
        } else {
            const uint16_t *r = BULK ? srec + (size_t)tid * WHOLE : rois + (size_t)i * WHOLE;
            float inv = 0.0f, f_rng = 0.0f, f_lo = 0.0f;
            const bool live = tid < rows;
            if (live) {
                record_range<R>(r, offset, kadc, lo, rng);
                inv = 1.0f / rng;
                f_rng = logf(rng) * 0.125f;
                f_lo = logf(lo) * 0.125f;
            }
#pragma unroll 1
            for (int kg = 0; kg < KIN / 8; ++kg) {
                float f[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) f[j] = live ? feature<R>(r, kg * 8 + j, offset, kadc, lo, inv, f_rng, f_lo) : 0.0f;
                *reinterpret_cast<uint4 *>(base + L::OFF_A1 + (size_t)(kg * kM + tid) * 16) = pack8(f);
            }
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        // the records are consumed: fetch the next tile of this CTA while the MMAs run
        if (BULK && tid == 0) {
            const int next = tile + gridDim.x;
            if (next < ntiles) {
                bulk_load(sRec, rois + (size_t)next * kM * WHOLE, bulk_bytes<R>(tile_rows(next, n)), sRecBar);
                copy_pending = true;
            }
        }
        // layer 1: D[128 x 128] at column 0
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < KIN / 16; ++ks)
                mma_bf16(tmem, smem_desc(sA1 + ks * 2 * kM * 16, kM * 16, 128),
                         smem_desc(sW1 + ks * 2 * kHidden * 16, kHidden * 16, 128), instr_desc(kM, kHidden),
                         ks > 0);
            mma_commit(sBar);
        }
        ok = __syncthreads_and(mbar_wait(sBar, phase));
        phase ^= 1u;
        if (!ok) break;
        fence_after();
        epilogue_hidden(tmem + row_lane, b1, base + L::OFF_A2, tid);  // layer 1 has read A1 (aliased here)
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        // layer 2: D[128 x 128] at column 128
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_bf16(tmem + kHidden, smem_desc(sA2 + ks * 2 * kM * 16, kM * 16, 128),
                         smem_desc(sW2 + ks * 2 * kHidden * 16, kHidden * 16, 128), instr_desc(kM, kHidden),
                         ks > 0);
            mma_commit(sBar);
        }
        ok = __syncthreads_and(mbar_wait(sBar, phase));
        phase ^= 1u;
        if (!ok) break;
        fence_after();
        epilogue_hidden(tmem + row_lane + kHidden, b2, base + L::OFF_A2, tid);  // layer 2 has read A2
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        // layer 3: D[128 x 16] at column 0
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_bf16(tmem, smem_desc(sA2 + ks * 2 * kM * 16, kM * 16, 128),
                         smem_desc(sW3 + ks * 2 * kN3 * 16, kN3 * 16, 128), instr_desc(kM, kN3), ks > 0);
            mma_commit(sBar);
        }
        ok = __syncthreads_and(mbar_wait(sBar, phase));
        phase ^= 1u;
        if (!ok) break;
        fence_after();
        float y[16];
        tmem_ld16(tmem + row_lane, y);
        if (tid < rows) {
#pragma unroll
            for (int j = 0; j < out_width(LT); ++j) y[j] += __ldg(b3 + j);
            start_from_outputs<R, LT>(y, lo, rng, start + (size_t)i * NST);
            if (LT == QCS_LOCTYPE_GS2D && cls)
                cls[i] = (uint8_t)count_class(y[kCount0], y[kCount0 + 1], y[kCount0 + 2], count_th);
        }
        fence_before();
        __syncthreads();  // accumulator columns are free for the next tile
        fence_after();
    }
    // error path: a copy issued for the next tile may still be landing in this
    // CTA's shared memory; wait for it (bounded) before the CTA ends
    if (BULK && __syncthreads_or(copy_pending)) mbar_wait(sRecBar, rec_phase);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    if (!ok) {
        // A wait gave up: this CTA's tiles from the failed one on get NaN start
        // points (and the single-emitter class), so their fits are rejected and
        // the deviance judge hands them to the plain refit instead of fitting
        // from a previous call's start points.  The sticky error flag records it.
        for (int t = tile; t < ntiles; t += gridDim.x) {
            if (tid < tile_rows(t, n)) {
                const int r = t * kM + tid;
#pragma unroll
                for (int j = 0; j < NST; ++j) start[(size_t)r * NST + j] = __int_as_float(0x7fc00000);
                if (LT == QCS_LOCTYPE_GS2D && cls) cls[r] = 0;
            }
        }
        if (tid == 0) atomicExch(err, 1);
    }
}

// FP32 master weights -> BF16 operand images (W1 | W2 | W3, N x K K-major).
template <int KIN, int NOUT>
__global__ void weight_image_kernel(const float *__restrict__ par, __nv_bfloat16 *__restrict__ img) {
    constexpr int W1 = kHidden * KIN, W2 = kHidden * kHidden, W3 = kN3 * kHidden;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float *pW1 = par, *pW2 = pW1 + KIN * kHidden + kHidden, *pW3 = pW2 + kHidden * kHidden + kHidden;
    if (i < W1) {
        const int k = i / kHidden, nn = i % kHidden;
        img[img_index(nn, k, kHidden)] = __float2bfloat16_rn(pW1[i]);
    } else if (i < W1 + W2) {
        const int j = i - W1, k = j / kHidden, nn = j % kHidden;
        img[W1 + img_index(nn, k, kHidden)] = __float2bfloat16_rn(pW2[j]);
    } else if (i < W1 + W2 + W3) {
        const int j = i - W1 - W2, k = j / kN3, nn = j % kN3;
        img[W1 + W2 + img_index(nn, k, kN3)] = __float2bfloat16_rn(nn < NOUT ? pW3[k * NOUT + nn] : 0.0f);
    }
}

}  // namespace tc
}  // namespace learned
}  // namespace qcs

using qcs::fail;
namespace L = qcs::learned;

struct qcs_learned_net {
    int loc_type = QCS_LOCTYPE_GS2D;  // the shape the network is built for
    int R = 7;
    // GS2D networks: the two-emitter network whose start points the 2E stage uses, and its schedule
    qcs_learned_net *two = nullptr;
    int owners = 0;  // GS2D networks this (two-emitter) network is attached to
    int direct_2e = 0;  // multi-emitter calls: poor bright single fits straight to the 2E stage
    int single_refits = 1;  // single-emitter calls: plain refits of the rejected or poor learned fits
    int two_iters = 3, two_bisections = 6, two_to3e = 1;
    float two_dev_th = 0.0f;
    // GS2D networks: the three-emitter network whose start points the 3E stage uses, and its schedule
    qcs_learned_net *three = nullptr;
    int three_iters = 4, three_bisections = 6;
    float three_dev_th = 0.0f;
    int kin = 64;                     // input width: in_width(R)
    int nout = 8;                     // outputs per record: out_width(loc_type)
    int params = 0;                   // param_count(kin)
    // parameters (FP32 master copies), their gradients and Adam moments, in one block
    float *d_par = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
    // activations of one batch
    float *d_x = nullptr, *d_z1 = nullptr, *d_a1 = nullptr, *d_z2 = nullptr, *d_a2 = nullptr, *d_y = nullptr;
    float *d_t = nullptr, *d_valid = nullptr, *d_dy = nullptr, *d_d2 = nullptr, *d_d1 = nullptr, *d_loss = nullptr;
    int *d_idx = nullptr;
    float *d_start = nullptr;  // start points and feature work of the last localization call
    size_t start_cap = 0;
    __nv_bfloat16 *d_wimg = nullptr;  // BF16 operand images of the weights (fused inference)
    int *d_err = nullptr;             // set by a tensor-core kernel when an MMA wait gives up
    float *d_ws = nullptr;            // split-K partial sums of the training GEMMs
    size_t ws_floats = 0;
    int arch = QCS_LEARNED_ARCH_MLP;
    qcs::learned::conv::State *conv = nullptr;  // QCS_LEARNED_ARCH_CONV: activations and inference buffers
    unsigned version = 1;             // bumped whenever the parameters change
    unsigned wimg_version = 0;        // parameter version d_wimg was built from
    cudaEvent_t wimg_ready = nullptr; // recorded after d_wimg was built
    cudaEvent_t start_free = nullptr;  // recorded after the last unfused start-point call used d_start
    bool use_tc = true;
    float count_th = 0.0f;            // emitter-count routing threshold; 0 = no routing
    int batch = 0;
    long long step = 0;
};

namespace {

struct Views {
    float *W1, *b1, *W2, *b2, *W3, *b3;
};
Views views(float *p, int kin, int nout = L::kOut) {
    Views v;
    v.W1 = p;
    v.b1 = v.W1 + kin * L::kHidden;
    v.W2 = v.b1 + L::kHidden;
    v.b2 = v.W2 + L::kHidden * L::kHidden;
    v.W3 = v.b2 + L::kHidden;
    v.b3 = v.W3 + L::kHidden * nout;
    return v;
}

inline int blocks(long long n, int t = 256) { return (int)((n + t - 1) / t); }

constexpr size_t kWsFloats = (size_t)1 << 21;  // split-K workspace per network (8 MB)

// threshold of the class outputs: the routing threshold, or 0.5 when routing is off
inline float class_threshold(const qcs_learned_net *net) { return net->count_th > 0.0f ? net->count_th : 0.5f; }

// Forward over `rows` feature rows into net->d_y (and the hidden activations).
cudaError_t forward(qcs_learned_net *net, const float *x, int rows, float *z1, float *a1, float *z2, float *a2,
                    float *y, cudaStream_t s) {
    if (net->conv)
        return L::conv::forward(net->conv, net->d_par, x, rows, net->kin, y, s, net->d_ws, net->ws_floats, net->d_err);
    const Views w = views(net->d_par, net->kin, net->nout);
    cudaError_t e;
    if ((e = L::gemm(rows, L::kHidden, net->kin, x, net->kin, 1, w.W1, L::kHidden, 1, z1, L::kHidden, 0.0f, s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    L::bias_relu_kernel<<<blocks((long long)rows * L::kHidden), 256, 0, s>>>(z1, w.b1, rows, L::kHidden, a1, 1);
    if ((e = L::gemm(rows, L::kHidden, L::kHidden, a1, L::kHidden, 1, w.W2, L::kHidden, 1, z2, L::kHidden, 0.0f, s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    L::bias_relu_kernel<<<blocks((long long)rows * L::kHidden), 256, 0, s>>>(z2, w.b2, rows, L::kHidden, a2, 1);
    const int no = net->nout;
    if ((e = L::gemm(rows, no, L::kHidden, a2, L::kHidden, 1, w.W3, no, 1, y, no, 0.0f, s, net->d_ws, net->ws_floats,
                     net->d_err)))
        return e;
    L::bias_relu_kernel<<<blocks((long long)rows * no), 256, 0, s>>>(y, w.b3, rows, no, y, 0);
    return cudaGetLastError();
}

// Backward of the masked MSE for one batch already forwarded; fills d_grad.
cudaError_t backward(qcs_learned_net *net, int rows, cudaStream_t s) {
    if (net->conv)
        return L::conv::backward(net->conv, net->d_par, net->d_grad, net->d_x, rows, net->kin, net->d_dy, s, net->d_ws,
                                 net->ws_floats, net->d_err);
    const Views w = views(net->d_par, net->kin, net->nout);
    const Views g = views(net->d_grad, net->kin, net->nout);
    cudaError_t e;
    // layer 3: dW3 = a2^T dy, db3 = colsum(dy), d2 = dy W3^T
    const int no = net->nout;
    if ((e = L::gemm(L::kHidden, no, rows, net->d_a2, 1, L::kHidden, net->d_dy, no, 1, g.W3, no, 0.0f,
                     s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    if ((e = L::column_sums(net->d_dy, rows, no, g.b3, net->d_ws, s))) return e;
    if ((e = L::gemm(rows, L::kHidden, no, net->d_dy, no, 1, w.W3, 1, no, net->d_d2, L::kHidden, 0.0f,
                     s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    L::relu_back_kernel<<<blocks((long long)rows * L::kHidden), 256, 0, s>>>(net->d_d2, net->d_z2,
                                                                           (long long)rows * L::kHidden);
    // layer 2
    if ((e = L::gemm(L::kHidden, L::kHidden, rows, net->d_a1, 1, L::kHidden, net->d_d2, L::kHidden, 1, g.W2,
                     L::kHidden, 0.0f, s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    if ((e = L::column_sums(net->d_d2, rows, L::kHidden, g.b2, net->d_ws, s))) return e;
    if ((e = L::gemm(rows, L::kHidden, L::kHidden, net->d_d2, L::kHidden, 1, w.W2, 1, L::kHidden, net->d_d1,
                     L::kHidden, 0.0f, s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    L::relu_back_kernel<<<blocks((long long)rows * L::kHidden), 256, 0, s>>>(net->d_d1, net->d_z1,
                                                                           (long long)rows * L::kHidden);
    // layer 1
    if ((e = L::gemm(net->kin, L::kHidden, rows, net->d_x, 1, net->kin, net->d_d1, L::kHidden, 1, g.W1, L::kHidden,
                     0.0f, s, net->d_ws, net->ws_floats, net->d_err)))
        return e;
    if ((e = L::column_sums(net->d_d1, rows, L::kHidden, g.b1, net->d_ws, s))) return e;
    return cudaGetLastError();
}

// xorshift-based permutation of [0, n) on the host, copied to the device
void shuffle(int *h, int n, unsigned long long &state) {
    for (int i = 0; i < n; ++i) h[i] = i;
    for (int i = n - 1; i > 0; --i) {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        const int j = (int)(state % (unsigned long long)(i + 1));
        const int t = h[i];
        h[i] = h[j];
        h[j] = t;
    }
}

// Compile-time shape for the dispatch below.
template <int R_, int LT_>
struct Shape {
    static constexpr int R = R_, LT = LT_;
};

// f(Shape<R, LT>{}) for the network shape (loc_type, R).
template <class F>
cudaError_t by_shape(int loc_type, int R, F &&f) {
    if (loc_type == QCS_LOCTYPE_AS3D) {
        switch (R) {
        case 7: return f(Shape<7, QCS_LOCTYPE_AS3D>{});
        case 9: return f(Shape<9, QCS_LOCTYPE_AS3D>{});
        case 11: return f(Shape<11, QCS_LOCTYPE_AS3D>{});
        }
    } else if (loc_type == QCS_LOCTYPE_GS2D) {
        switch (R) {
        case 7: return f(Shape<7, QCS_LOCTYPE_GS2D>{});
        case 9: return f(Shape<9, QCS_LOCTYPE_GS2D>{});
        case 11: return f(Shape<11, QCS_LOCTYPE_GS2D>{});
        }
    } else if (loc_type == L::kTwo) {
        switch (R) {
        case 7: return f(Shape<7, L::kTwo>{});
        case 9: return f(Shape<9, L::kTwo>{});
        case 11: return f(Shape<11, L::kTwo>{});
        }
    } else if (loc_type == L::kThree) {
        switch (R) {
        case 7: return f(Shape<7, L::kThree>{});
        case 9: return f(Shape<9, L::kThree>{});
        case 11: return f(Shape<11, L::kThree>{});
        }
    }
    return cudaErrorInvalidValue;
}

// Start points of n ROIs through the fused tcgen05 kernel: BF16 operand
// images of the current weights, then one persistent launch (7x7: two CTAs
// of 101 KB shared memory and 256 tensor-memory columns per SM; 9x9, 11x11:
// one CTA of 123 or 133 KB).
cudaError_t fused_start_points(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                               const int *n_dev, float *start, uint8_t *cls, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (net->conv)
        return L::conv::start_points(net->conv, net->d_par, net->version, net->loc_type, p, d_rois, n, n_dev, start, cls,
                                     class_threshold(net), s, net->d_err);
    const int tiles = (n + L::tc::kM - 1) / L::tc::kM;
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const bool bulk = (reinterpret_cast<uintptr_t>(d_rois) & 15) == 0;
    const Views w = views(net->d_par, net->kin, net->nout);
    const float th = class_threshold(net);
    return by_shape(net->loc_type, net->R, [&](auto sh) -> cudaError_t {
        constexpr int R = decltype(sh)::R, LT = decltype(sh)::LT;
        typedef L::tc::Layout<R> Lay;
        auto kern = bulk ? L::tc::mlp_tc_kernel<true, R, LT> : L::tc::mlp_tc_kernel<false, R, LT>;
        cudaError_t e2 = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::SMEM);
        if (e2 != cudaSuccess) return e2;
        const int per_sm = Lay::SMEM <= 113 * 1024 ? 2 : 1;
        const int grid = tiles < per_sm * sms ? tiles : per_sm * sms;
        // the weight image is rebuilt only after a parameter change; calls on
        // other streams wait for the build that made the current one.  Under
        // stream capture a stale image is rebuilt inside the graph (and again
        // by the next call outside it), and a current one must have been
        // built already: an event recorded outside a capture cannot be waited
        // on inside it.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e2 = cudaStreamIsCapturing(s, &cs);
        if (e2 != cudaSuccess) return e2;
        const bool capturing = cs != cudaStreamCaptureStatusNone;
        if (net->wimg_version != net->version) {
            L::tc::weight_image_kernel<Lay::KIN, L::out_width(LT)><<<blocks(Lay::W1 + Lay::W2 + Lay::W3), 256, 0, s>>>(net->d_par,
                                                                                                  net->d_wimg);
            if (!capturing) {
                e2 = cudaEventRecord(net->wimg_ready, s);
                if (e2 != cudaSuccess) return e2;
                net->wimg_version = net->version;
            }
        } else if (!capturing) {
            e2 = cudaStreamWaitEvent(s, net->wimg_ready, 0);
            if (e2 != cudaSuccess) return e2;
        } else if (cudaEventQuery(net->wimg_ready) != cudaSuccess) {
            return cudaErrorNotReady;  // the build is still in flight: synchronize before capturing
        }
        kern<<<grid, 128, Lay::SMEM, s>>>(d_rois, n, p->Offset, p->KAdc, reinterpret_cast<const uint4 *>(net->d_wimg),
                                          w.b1, w.b2, w.b3, start, cls, th, n_dev, net->d_err);
        return cudaGetLastError();
    });
}

// net's shape against the call's parameters
int check_shape(const qcs_learned_net *net, const qcs_loc_para *p) {
    const int want = (net->loc_type == L::kTwo || net->loc_type == L::kThree) ? QCS_LOCTYPE_GS2D : net->loc_type;
    if (p->ROISize != net->R || p->LocType != want)
        return fail(QCS_ERR_ROISIZE, "the network was built for another localization type or ROI size");
    return QCS_OK;
}

}  // namespace

namespace qcs {
namespace learned {
bool direct_two_emitter(const qcs_learned_net *net) { return net && net->direct_2e; }
bool single_refits(const qcs_learned_net *net) { return !net || net->single_refits; }

qcs_learned_net *three_emitter(const qcs_learned_net *net, int *iters, int *bisections, float *dev_th) {
    if (!net || !net->three) return nullptr;
    *iters = net->three_iters;
    *bisections = net->three_bisections;
    *dev_th = net->three_dev_th;
    return net->three;
}

qcs_learned_net *two_emitter(const qcs_learned_net *net, int *iters, int *bisections, float *dev_th, int *to3e) {
    if (!net || !net->two) return nullptr;
    *to3e = net->two_to3e;
    *iters = net->two_iters;
    *bisections = net->two_bisections;
    *dev_th = net->two_dev_th;
    return net->two;
}
}  // namespace learned
}  // namespace qcs

extern "C" {

int qcs_learned_param_count(void) { return L::param_count(L::in_width(7)); }

int qcs_learned_destroy(qcs_learned_net *net) {
    if (!net) return QCS_OK;
    // a two-emitter network still attached to a GS2D network is in use by it:
    // refuse instead of leaving the owner with a dangling pointer
    if (net->owners > 0)
        return fail(QCS_ERR_STATE, "the network is attached to a GS2D network: detach it first "
                                   "(qcs_learned_set_two_emitter(owner, NULL, ...)) or destroy the owner");
    if (net->two) net->two->owners--;
    net->two = nullptr;
    if (net->three) net->three->owners--;
    net->three = nullptr;
    cudaDeviceSynchronize();  // no call of this network still in flight
    cudaFree(net->d_par);
    cudaFree(net->d_x);
    cudaFree(net->d_idx);
    cudaFree(net->d_start);
    cudaFree(net->d_wimg);
    cudaFree(net->d_err);
    cudaFree(net->d_ws);
    L::conv::destroy(net->conv);
    if (net->wimg_ready) cudaEventDestroy(net->wimg_ready);
    if (net->start_free) cudaEventDestroy(net->start_free);
    delete net;
    return QCS_OK;
}

int qcs_learned_create_for(int loc_type, int roi_size, int batch, unsigned long long seed, qcs_learned_net **out) {
    return qcs_learned_create_arch(QCS_LEARNED_ARCH_MLP, loc_type, roi_size, batch, seed, out);
}

int qcs_learned_arch(const qcs_learned_net *net) { return net ? net->arch : -1; }

int qcs_learned_create_arch(int arch, int loc_type, int roi_size, int batch, unsigned long long seed,
                            qcs_learned_net **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    if (arch != QCS_LEARNED_ARCH_MLP && arch != QCS_LEARNED_ARCH_CONV)
        return fail(QCS_ERR_ARG, "architecture: QCS_LEARNED_ARCH_MLP or QCS_LEARNED_ARCH_CONV");
    if (arch == QCS_LEARNED_ARCH_CONV && loc_type == L::kThree)
        return fail(QCS_ERR_ARG, "three-emitter start points: MLP networks only");
    if (!L::shape_supported(loc_type, roi_size))
        return fail(QCS_ERR_ROISIZE, "learned start points: GS2D or AS3D, ROISize 7, 9 or 11");
    if (batch <= 0) batch = 4096;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_learned_net *net = new qcs_learned_net();
    net->loc_type = loc_type;
    net->R = roi_size;
    net->kin = L::in_width(roi_size);
    net->arch = arch;
    net->nout = L::out_width(loc_type);
    net->params = arch == QCS_LEARNED_ARCH_CONV ? L::conv::param_count(roi_size) : L::param_count(net->kin, net->nout);
    net->ws_floats = arch == QCS_LEARNED_ARCH_CONV ? 4 * kWsFloats : kWsFloats;
    net->batch = batch;
    const int kin = net->kin;
    const size_t P = net->params;
    const size_t B = (size_t)batch;
    const size_t acts = B * (kin + 4 * L::kHidden + L::kOutMax + L::kUsedMax + 1 + L::kOutMax + 2 * L::kHidden) + 4;
    const size_t wimg_bytes = (size_t)(L::kHidden * kin + L::kHidden * L::kHidden + L::tc::kN3 * L::kHidden) * 2;
    cudaError_t e = cudaMalloc((void **)&net->d_par, 4 * P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&net->d_x, acts * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&net->d_idx, B * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&net->d_wimg, wimg_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&net->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&net->d_ws, net->ws_floats * sizeof(float));
    if (e == cudaSuccess && arch == QCS_LEARNED_ARCH_CONV) e = L::conv::create(roi_size, batch, &net->conv);
    if (e == cudaSuccess) e = cudaMemset(net->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&net->wimg_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&net->start_free, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        qcs_learned_destroy(net);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_learned_create", e);
    }
    net->d_grad = net->d_par + P;
    net->d_m = net->d_grad + P;
    net->d_v = net->d_m + P;
    float *a = net->d_x + B * kin;
    net->d_z1 = a;
    a += B * L::kHidden;
    net->d_a1 = a;
    a += B * L::kHidden;
    net->d_z2 = a;
    a += B * L::kHidden;
    net->d_a2 = a;
    a += B * L::kHidden;
    net->d_y = a;
    a += B * L::kOutMax;
    net->d_t = a;
    a += B * L::kUsedMax;
    net->d_valid = a;
    a += B;
    net->d_dy = a;
    a += B * L::kOutMax;
    net->d_d2 = a;
    a += B * L::kHidden;
    net->d_d1 = a;
    a += B * L::kHidden;
    net->d_loss = a;
    // He-style initialisation from a host xorshift generator (uniform, variance 2 / fan_in)
    float *h = new float[P];
    unsigned long long st = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto uni = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (float)((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0f - 1.0f;
    };
    if (net->conv) {
        L::conv::init_params(h, roi_size, seed);
    } else {
        const Views hv = views(h, kin, net->nout);
        for (int i = 0; i < kin * L::kHidden; ++i) hv.W1[i] = uni() * sqrtf(6.0f / kin);
        for (int i = 0; i < L::kHidden; ++i) hv.b1[i] = 0.0f;
        for (int i = 0; i < L::kHidden * L::kHidden; ++i) hv.W2[i] = uni() * sqrtf(6.0f / L::kHidden);
        for (int i = 0; i < L::kHidden; ++i) hv.b2[i] = 0.0f;
        for (int i = 0; i < L::kHidden * net->nout; ++i) hv.W3[i] = uni() * sqrtf(3.0f / L::kHidden);
        for (int i = 0; i < net->nout; ++i) hv.b3[i] = 0.0f;
    }
    e = cudaMemcpy(net->d_par, h, P * sizeof(float), cudaMemcpyHostToDevice);
    delete[] h;
    if (e == cudaSuccess) e = cudaMemset(net->d_m, 0, 2 * P * sizeof(float));
    if (e != cudaSuccess) {
        qcs_learned_destroy(net);
        return fail(QCS_ERR_CUDA, "initialise parameters", e);
    }
    *out = net;
    return QCS_OK;
}

int qcs_learned_create(int batch, unsigned long long seed, qcs_learned_net **out) {
    return qcs_learned_create_for(QCS_LOCTYPE_GS2D, 7, batch, seed, out);
}

int qcs_learned_shape(const qcs_learned_net *net, int *loc_type, int *roi_size, int *params) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (loc_type) *loc_type = net->loc_type;
    if (roi_size) *roi_size = net->R;
    if (params) *params = net->params;
    return QCS_OK;
}

int qcs_learned_get_params(qcs_learned_net *net, float *h_params) {
    if (!net || !h_params) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaMemcpy(h_params, net->d_par, (size_t)net->params * sizeof(float), cudaMemcpyDeviceToHost),
             "read parameters");
    return QCS_OK;
}

int qcs_learned_set_params(qcs_learned_net *net, const float *h_params) {
    if (!net || !h_params) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaMemcpy(net->d_par, h_params, (size_t)net->params * sizeof(float), cudaMemcpyHostToDevice),
             "set parameters");
    net->version++;
    return QCS_OK;
}

int qcs_learned_features_device(const qcs_loc_para *p, const uint16_t *d_rois, int n, float *d_feat, float *d_scale,
                                void *stream) {
    if (!p || (!d_rois && n > 0) || !d_feat || !d_scale) return fail(QCS_ERR_ARG, "null argument");
    if (!L::shape_supported(p->LocType, p->ROISize))
        return fail(QCS_ERR_ROISIZE, "learned start points: GS2D or AS3D, ROISize 7, 9 or 11");
    if (n <= 0) return QCS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    QCS_CUDA(by_shape(QCS_LOCTYPE_GS2D, p->ROISize, [&](auto sh) -> cudaError_t {
                 L::features_kernel<decltype(sh)::R><<<blocks(n), 256, 0, s>>>(d_rois, n, p->Offset, p->KAdc, d_feat,
                                                                                d_scale);
                 return cudaGetLastError();
             }),
             "features");
    return QCS_OK;
}

int qcs_learned_targets_device(const qcs_loc_para *p, const uint16_t *d_rois, const float *d_rows,
                               const float *d_scale, int n, float *d_targets, float *d_valid, void *stream) {
    if (!p || !d_rois || !d_rows || !d_scale || !d_targets || !d_valid) return fail(QCS_ERR_ARG, "null argument");
    if (!L::shape_supported(p->LocType, p->ROISize))
        return fail(QCS_ERR_ROISIZE, "learned start points: GS2D or AS3D, ROISize 7, 9 or 11");
    if (n <= 0) return QCS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    QCS_CUDA(by_shape(p->LocType, p->ROISize, [&](auto sh) -> cudaError_t {
                 L::targets_kernel<decltype(sh)::R, decltype(sh)::LT>
                     <<<blocks(n), 256, 0, s>>>(d_rois, d_rows, d_scale, n, p->QE, d_targets, d_valid);
                 return cudaGetLastError();
             }),
             "targets");
    return QCS_OK;
}

int qcs_learned_forward_device(qcs_learned_net *net, const float *d_feat, int n, float *d_out, void *stream) {
    if (!net || !d_feat || !d_out) return fail(QCS_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int r0 = 0; r0 < n; r0 += net->batch) {
        const int rows = (n - r0) < net->batch ? (n - r0) : net->batch;
        QCS_CUDA(forward(net, d_feat + (size_t)r0 * net->kin, rows, net->d_z1, net->d_a1, net->d_z2, net->d_a2,
                         d_out + (size_t)r0 * net->nout, s),
                 "forward");
    }
    return QCS_OK;
}

int qcs_learned_gradient_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                const float *d_valid, int n, float *h_loss, void *stream) {
    return qcs_learned_gradient_counts_device(net, d_feat, d_targets, d_valid, nullptr, n, h_loss, stream);
}

int qcs_learned_gradient_counts_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                       const float *d_valid, const float *d_classes, int n, float *h_loss,
                                       void *stream) {
    if (!net || !d_feat || !d_targets || !d_valid) return fail(QCS_ERR_ARG, "null argument");
    if (n <= 0 || n > net->batch) return fail(QCS_ERR_CAPACITY, "gradient batch must be 1..batch rows");
    if (d_classes && net->loc_type != QCS_LOCTYPE_GS2D) return fail(QCS_ERR_ARG, "count classes: GS2D networks only");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    QCS_CUDA(cudaMemcpyAsync(net->d_x, d_feat, (size_t)n * net->kin * sizeof(float), cudaMemcpyDeviceToDevice, s),
             "copy features");
    QCS_CUDA(forward(net, net->d_x, n, net->d_z1, net->d_a1, net->d_z2, net->d_a2, net->d_y, s), "forward");
    QCS_CUDA(cudaMemsetAsync(net->d_loss, 0, sizeof(float), s), "clear loss");
    L::mse_kernel<<<blocks(n), 256, 0, s>>>(net->d_y, d_targets, d_valid, d_classes, n, net->nout,
                                            L::used_outputs(net->loc_type), L::weight_row(net->loc_type),
                                            1.0f / (float)n, net->d_dy, net->d_loss);
    QCS_CUDA(backward(net, n, s), "backward");
    if (h_loss) {
        QCS_CUDA(cudaMemcpyAsync(h_loss, net->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s), "read loss");
        QCS_CUDA(cudaStreamSynchronize(s), "gradient");
    }
    return QCS_OK;
}

int qcs_learned_get_grads(qcs_learned_net *net, float *h_grads) {
    if (!net || !h_grads) return fail(QCS_ERR_ARG, "null argument");
    QCS_CUDA(cudaMemcpy(h_grads, net->d_grad, (size_t)net->params * sizeof(float), cudaMemcpyDeviceToHost),
             "read gradients");
    return QCS_OK;
}

int qcs_learned_train_device(qcs_learned_net *net, const float *d_feat, const float *d_targets, const float *d_valid,
                             int n, int epochs, float lr, unsigned long long seed, float *h_epoch_loss, void *stream) {
    return qcs_learned_train_counts_device(net, d_feat, d_targets, d_valid, nullptr, n, epochs, lr, seed, h_epoch_loss,
                                           stream);
}

int qcs_learned_train_counts_device(qcs_learned_net *net, const float *d_feat, const float *d_targets,
                                    const float *d_valid, const float *d_classes, int n, int epochs, float lr,
                                    unsigned long long seed, float *h_epoch_loss, void *stream) {
    if (!net || !d_feat || !d_targets || !d_valid) return fail(QCS_ERR_ARG, "null argument");
    if (n < net->batch) return fail(QCS_ERR_ARG, "fewer training rows than one batch");
    if (d_classes && net->loc_type != QCS_LOCTYPE_GS2D) return fail(QCS_ERR_ARG, "count classes: GS2D networks only");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int B = net->batch;
    const int steps = n / B;
    const int kin = net->kin, nu = L::used_outputs(net->loc_type);
    int *h_perm = new int[n];
    int *d_perm = nullptr;
    float *d_vb = nullptr, *d_tb = nullptr;
    cudaError_t e = cudaMalloc((void **)&d_perm, (size_t)n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_vb, (size_t)B * 2 * sizeof(float));  // valid | classes
    float *d_cb = d_classes ? d_vb + B : nullptr;
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_tb, (size_t)B * nu * sizeof(float));
    unsigned long long state = seed ? seed : 0x2545F4914F6CDD1Dull;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        shuffle(h_perm, n, state);
        e = cudaMemcpyAsync(d_perm, h_perm, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(net->d_loss, 0, sizeof(float), s);
        for (int st = 0; st < steps && e == cudaSuccess; ++st) {
            const int *idx = d_perm + (size_t)st * B;
            L::gather_rows_kernel<<<blocks((long long)B * kin), 256, 0, s>>>(d_feat, idx, B, kin, net->d_x);
            L::gather_rows_kernel<<<blocks((long long)B * nu), 256, 0, s>>>(d_targets, idx, B, nu, d_tb);
            L::gather_rows_kernel<<<blocks(B), 256, 0, s>>>(d_valid, idx, B, 1, d_vb);
            if (d_cb) L::gather_rows_kernel<<<blocks(B), 256, 0, s>>>(d_classes, idx, B, 1, d_cb);
            e = forward(net, net->d_x, B, net->d_z1, net->d_a1, net->d_z2, net->d_a2, net->d_y, s);
            if (e != cudaSuccess) break;
            // per-batch mean loss and its gradient; the loss accumulates over the epoch
            L::mse_kernel<<<blocks(B), 256, 0, s>>>(net->d_y, d_tb, d_vb, d_cb, B, net->nout, nu,
                                                    L::weight_row(net->loc_type),
                                                    1.0f / (float)B, net->d_dy,
                                                    net->d_loss);
            e = backward(net, B, s);
            if (e != cudaSuccess) break;
            net->step++;
            const float c1 = 1.0f / (1.0f - powf(b1, (float)net->step));
            const float c2 = 1.0f / (1.0f - powf(b2, (float)net->step));
            L::adam_kernel<<<blocks(net->params), 256, 0, s>>>(net->d_par, net->d_grad, net->d_m, net->d_v,
                                                               net->params, lr, b1, b2, c1, c2, eps);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && h_epoch_loss) {
            e = cudaMemcpyAsync(h_epoch_loss + ep, net->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            h_epoch_loss[ep] /= (float)steps;
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    net->version++;
    cudaFree(d_perm);
    cudaFree(d_vb);
    cudaFree(d_tb);
    delete[] h_perm;
    if (e != cudaSuccess) return fail(QCS_ERR_CUDA, "training", e);
    return QCS_OK;
}

int qcs_learned_start_device(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                             float *d_start, float *d_work, void *stream) {
    if (!net || !p || !d_start || !d_work) return fail(QCS_ERR_ARG, "null argument");
    int st = check_shape(net, p);
    if (st) return st;
    if (n <= 0) return QCS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (net->use_tc) {
        QCS_CUDA(fused_start_points(net, p, d_rois, n, nullptr, d_start, nullptr, s), "fused start points");
        return QCS_OK;
    }
    float *feat = d_work, *scale = feat + (size_t)n * net->kin, *y = scale + 2 * (size_t)n;
    st = qcs_learned_features_device(p, d_rois, n, feat, scale, s);
    if (st) return st;
    st = qcs_learned_forward_device(net, feat, n, y, s);
    if (st) return st;
    QCS_CUDA(by_shape(net->loc_type, net->R, [&](auto sh) -> cudaError_t {
                 L::start_kernel<decltype(sh)::R, decltype(sh)::LT>
                     <<<blocks(n), 256, 0, s>>>(y, scale, n, d_start, nullptr, 0.0f);
                 return cudaGetLastError();
             }),
             "start points");
    return QCS_OK;
}

int qcs_learned_classes_device(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                               float *d_start, uint8_t *d_classes, void *stream) {
    if (!net || !p || !d_start || !d_classes) return fail(QCS_ERR_ARG, "null argument");
    int st = check_shape(net, p);
    if (st) return st;
    if (net->loc_type != QCS_LOCTYPE_GS2D) return fail(QCS_ERR_ARG, "count classes: GS2D networks only");
    if (n <= 0) return QCS_OK;
    if (!d_rois) return fail(QCS_ERR_ARG, "null ROI pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    QCS_CUDA(L::start_points(net, p, d_rois, n, d_start, s, d_classes), "start points and classes");
    return QCS_OK;
}

int qcs_learned_set_count_threshold(qcs_learned_net *net, float th) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (!(th >= 0.0f && th <= 1.0f)) return fail(QCS_ERR_ARG, "count threshold must be in [0, 1] (0: no routing)");
    if (th > 0.0f && net->loc_type != QCS_LOCTYPE_GS2D) return fail(QCS_ERR_ARG, "count classes: GS2D networks only");
    net->count_th = th;
    return QCS_OK;
}

float qcs_learned_count_threshold(const qcs_learned_net *net) { return net ? net->count_th : 0.0f; }

int qcs_learned_set_two_emitter(qcs_learned_net *net, qcs_learned_net *two, int iters, int bisections,
                                float dev_th, int fallback) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (!two) {
        if (net->two) net->two->owners--;
        net->two = nullptr;
        return QCS_OK;
    }
    if (net->loc_type != QCS_LOCTYPE_GS2D || two->loc_type != L::kTwo || two->R != net->R)
        return fail(QCS_ERR_ARG, "two-emitter start points: a QCS_LEARNED_GS2D_2E network of the GS2D network's ROI size");
    if (bisections <= 0) bisections = 11;
    if (!qcs::learned_2e_supported(net->R, iters, bisections))
        return fail(QCS_ERR_ARG, "two-emitter schedules: 3 or 4 iterations of 6 line-search steps, or 13 of 11");
    if (!(dev_th >= 0.0f)) return fail(QCS_ERR_ARG, "negative deviance bound");
    if (fallback != QCS_TWO_FALLBACK_3E && fallback != QCS_TWO_FALLBACK_PLAIN && fallback != QCS_TWO_FALLBACK_NONE)
        return fail(QCS_ERR_ARG, "fallback: QCS_TWO_FALLBACK_3E, QCS_TWO_FALLBACK_PLAIN or QCS_TWO_FALLBACK_NONE");
    net->two_to3e = fallback == QCS_TWO_FALLBACK_3E ? 1 : (fallback == QCS_TWO_FALLBACK_NONE ? 2 : 0);
    if (net->two != two) {
        if (net->two) net->two->owners--;
        two->owners++;
    }
    net->two = two;
    net->two_iters = iters;
    net->two_bisections = bisections;
    net->two_dev_th = dev_th;
    return QCS_OK;
}

int qcs_learned_set_three_emitter(qcs_learned_net *net, qcs_learned_net *three, int iters, int bisections,
                                  float dev_th) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (!three) {
        if (net->three) net->three->owners--;
        net->three = nullptr;
        return QCS_OK;
    }
    if (net->loc_type != QCS_LOCTYPE_GS2D || three->loc_type != L::kThree || three->R != net->R)
        return fail(QCS_ERR_ARG,
                    "three-emitter start points: a QCS_LEARNED_GS2D_3E network of the GS2D network's ROI size");
    if (bisections <= 0) bisections = 6;
    if (!qcs::learned_3e_supported(net->R, iters, bisections))
        return fail(QCS_ERR_ARG, "three-emitter schedules: 4 or 6 iterations of 6 line-search steps, or 16 of 11");
    if (dev_th != dev_th) return fail(QCS_ERR_ARG, "deviance bound is not a number");
    if (net->three != three) {
        if (net->three) net->three->owners--;
        three->owners++;
    }
    net->three = three;
    net->three_iters = iters;
    net->three_bisections = bisections;
    net->three_dev_th = dev_th;
    return QCS_OK;
}

int qcs_learned_set_single_refits(qcs_learned_net *net, int on) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    net->single_refits = on ? 1 : 0;
    return QCS_OK;
}

int qcs_learned_set_direct_two_emitter(qcs_learned_net *net, int on) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    if (on && net->loc_type != QCS_LOCTYPE_GS2D) return fail(QCS_ERR_ARG, "direct two-emitter routing: GS2D networks");
    net->direct_2e = on ? 1 : 0;
    return QCS_OK;
}

size_t qcs_learned_work_bytes(int n) {
    return (size_t)(n > 0 ? n : 0) * (L::in_width(11) + 2 + L::kOutMax) * sizeof(float);
}

int qcs_learned_set_inference(qcs_learned_net *net, int fused) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    net->use_tc = fused != 0;
    return QCS_OK;
}

int qcs_learned_fused_status(qcs_learned_net *net) {
    if (!net) return fail(QCS_ERR_ARG, "null network");
    int h = 0;
    QCS_CUDA(cudaDeviceSynchronize(), "fused inference");
    QCS_CUDA(cudaMemcpy(&h, net->d_err, sizeof(int), cudaMemcpyDeviceToHost), "read status");
    return h ? fail(QCS_ERR_CUDA, "fused inference: a tensor-core wait gave up") : QCS_OK;
}

}  // extern "C"

// Start points of n records into out: the fused kernel, or, with fused
// inference off, features and one GEMM per layer over all n rows in
// net-owned memory (grown, outside any capture, when n exceeds what the last
// call needed; not for concurrent calls).
cudaError_t qcs::learned::start_points(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n,
                                       float *out, cudaStream_t s, uint8_t *cls, const int *n_dev) {
    if (net->use_tc) return fused_start_points(net, p, d_rois, n, n_dev, out, cls, s);
    const int kin = net->kin;
    const size_t need = (size_t)n * (kin + 2 + 2 * L::kHidden + L::kOutMax);
    if (need > net->start_cap) {
        cudaFree(net->d_start);
        net->d_start = nullptr;
        net->start_cap = 0;
        cudaError_t e = cudaMalloc((void **)&net->d_start, need * sizeof(float));
        if (e != cudaSuccess) return e;
        net->start_cap = need;
    }
    float *feat = net->d_start, *scale = feat + (size_t)n * kin;
    float *h1 = scale + 2 * (size_t)n, *h2 = h1 + (size_t)n * L::kHidden, *y = h2 + (size_t)n * L::kHidden;
    const float th = class_threshold(net);
    // d_start holds one call's features and activations: a call on another stream waits until the call before it
    // has used them (outside stream capture: a graph holding this call must not run beside another call of the net)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e0 = cudaStreamIsCapturing(s, &cs);
    if (e0 != cudaSuccess) return e0;
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    if (!capturing && (e0 = cudaStreamWaitEvent(s, net->start_free, 0)) != cudaSuccess) return e0;
    e0 = by_shape(net->loc_type, net->R, [&](auto sh) -> cudaError_t {
        constexpr int R = decltype(sh)::R, LT = decltype(sh)::LT;
        L::features_kernel<R><<<blocks(n), 256, 0, s>>>(d_rois, n, p->Offset, p->KAdc, feat, scale);
        cudaError_t e = cudaSuccess;
        if (net->conv) {  // the conv net's activations hold one batch
            for (int r0 = 0; r0 < n && e == cudaSuccess; r0 += net->batch)
                e = forward(net, feat + (size_t)r0 * kin, n - r0 < net->batch ? n - r0 : net->batch, nullptr, nullptr,
                            nullptr, nullptr, y + (size_t)r0 * net->nout, s);
        } else {
            e = forward(net, feat, n, h1, h1, h2, h2, y, s);
        }
        if (e != cudaSuccess) return e;
        L::start_kernel<R, LT><<<blocks(n), 256, 0, s>>>(y, scale, n, out, LT == QCS_LOCTYPE_GS2D ? cls : nullptr, th);
        return cudaGetLastError();
    });
    if (e0 != cudaSuccess || capturing) return e0;
    return cudaEventRecord(net->start_free, s);
}
