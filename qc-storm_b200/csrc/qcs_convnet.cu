// Convolutional start-point network (QCS_LEARNED_ARCH_CONV): the R x R
// scaled pixels -> 3x3 conv, 32 channels, zero 'same' padding, ReLU -> 3x3
// conv, 64 channels, ReLU -> fully connected 256 over the flattened map
// (position major, channel minor) and the two scale features, ReLU -> the
// eight outputs of the MLP network (qcs_learned.cu), with the same features,
// targets, loss and start transform.  No counterpart in the reference.
//
// Parameters (FP32 master copies, row-major [in][out]): W1 [9][32] (tap
// t = 3 (dy + 1) + (dx + 1)), b1, W2 [9 * 32][64] (row t * 32 + input
// channel), b2, W3 [R*R*64 + 2][256], b3, W4 [256][8], b4.
//
// Training: im2col + tcgen05 GEMMs (qcs::learned::gemm), one batch at a time.
// Inference: two tcgen05 kernels per chunk of records.
//  * conv_tc_kernel: groups of T ROIs per CTA (records bulk-copied one
//    group ahead; one thread issues the MMAs).  The scaled pixels of the
//    group are laid out on a padded row grid in shared memory (row pitch
//    R + 1, one zero row after each ROI, a zero column at the end of each
//    row), so that the 3x3 neighbour (dy, dx) of grid row r is grid row
//    r + dy (R + 1) + dx for every interior position.  conv1 is one MMA
//    (M = 128 grid rows, N = 32, K = 16: nine taps and seven zeros) per tile
//    of rows; conv2 is nine MMAs pairs (K = 2 x 16 channels) per tile whose A
//    operands are the conv1 map shifted by each tap's row offset: a
//    descriptor start address moved by 16 bytes per row.  The epilogues add
//    the bias, apply the ReLU and round to BF16; conv2's writes each ROI's
//    64 x R*R map into the FC operand in global memory, already in the UMMA
//    K-major tile layout.
//  * fc_tc_kernel: one 128-ROI tile per CTA iteration; 64-deep K chunks of
//    the FC operand (16 KB) and of the W3 image (32 KB) arrive by bulk copy
//    into a four-stage ring, one thread issues four MMAs (M = 128, N = 256)
//    per chunk into tensor memory, the epilogue writes ReLU(FC) as the head's
//    A operand in shared memory, sixteen MMAs (N = 16) give the outputs, and
//    the start transform writes the start points (and the count class).
#include <cstdint>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_learned.h"
#include "qcs_tc.cuh"

namespace qcs {
namespace learned {
namespace conv {

constexpr int kC1 = 32, kC2 = 64, kFc = 256, kTaps = 9;
constexpr int kChunk = 65536;  // records per inference chunk (FC operand buffer)

__host__ __device__ constexpr int k0_of(int R) { return R * R * kC2; }       // flattened conv2 map
__host__ __device__ constexpr int kf_of(int R) { return R * R * kC2 + 64; }  // FC operand width (map, 2 scales, zeros)

struct Offsets {
    size_t W1, b1, W2, b2, W3, b3, W4, b4, total;
};
__host__ __device__ inline Offsets offsets(int R) {
    Offsets o;
    o.W1 = 0;
    o.b1 = o.W1 + kTaps * kC1;
    o.W2 = o.b1 + kC1;
    o.b2 = o.W2 + kTaps * kC1 * kC2;
    o.W3 = o.b2 + kC2;
    o.b3 = o.W3 + (size_t)(k0_of(R) + 2) * kFc;
    o.W4 = o.b3 + kFc;
    o.b4 = o.W4 + kFc * kOut;
    o.total = o.b4 + kOut;
    return o;
}

int param_count(int R) { return (int)offsets(R).total; }

// ------------------------------------------------------- training kernels
inline int nblk(long long n, int t = 256) { return (int)((n + t - 1) / t); }

// X1[b R^2 + p][t]: scaled pixel of feature row b at the tap's neighbour of p (0 outside)
__global__ void im2col1_kernel(const float *__restrict__ feat, int kin, int rows, int R, float *__restrict__ X1) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int PIX = R * R;
    if (i >= (long long)rows * PIX * kTaps) return;
    const long long row = i / kTaps;
    const int t = (int)(i - row * kTaps);
    const int b = (int)(row / PIX), p = (int)(row - (long long)b * PIX);
    const int yy = p / R + t / 3 - 1, xx = p % R + t % 3 - 1;
    X1[i] = (yy >= 0 && yy < R && xx >= 0 && xx < R) ? feat[(size_t)b * kin + yy * R + xx] : 0.0f;
}

// X2[b R^2 + p][t * 32 + c] = A1[b R^2 + neighbour][c] (0 outside)
__global__ void im2col2_kernel(const float *__restrict__ A1, int rows, int R, float *__restrict__ X2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int PIX = R * R;
    if (i >= (long long)rows * PIX * kTaps * kC1) return;
    const long long row = i / (kTaps * kC1);
    const int col = (int)(i - row * (kTaps * kC1));
    const int t = col / kC1, c = col - t * kC1;
    const int b = (int)(row / PIX), p = (int)(row - (long long)b * PIX);
    const int yy = p / R + t / 3 - 1, xx = p % R + t % 3 - 1;
    X2[i] = (yy >= 0 && yy < R && xx >= 0 && xx < R) ? A1[((size_t)b * PIX + yy * R + xx) * kC1 + c] : 0.0f;
}

// adjoint of im2col2: dA1[q][c] = sum over taps t of dX2[q - offset(t)][t * 32 + c], taps in order
__global__ void col2im2_kernel(const float *__restrict__ dX2, int rows, int R, float *__restrict__ dA1) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int PIX = R * R;
    if (i >= (long long)rows * PIX * kC1) return;
    const long long row = i / kC1;
    const int c = (int)(i - row * kC1);
    const int b = (int)(row / PIX), p = (int)(row - (long long)b * PIX);
    const int y = p / R, x = p % R;
    float s = 0.0f;
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
        const int sy = y - (t / 3 - 1), sx = x - (t % 3 - 1);
        if (sy >= 0 && sy < R && sx >= 0 && sx < R)
            s += dX2[((size_t)b * PIX + sy * R + sx) * (kTaps * kC1) + t * kC1 + c];
    }
    dA1[i] = s;
}

// Z (rows x cols) += bias; A = relu(Z) when relu (A may alias Z)
__global__ void bias_act_kernel(float *__restrict__ Z, const float *__restrict__ bias, long long rows, int cols,
                                float *__restrict__ A, int relu) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const float z = Z[i] + bias[i % cols];
    Z[i] = z;
    A[i] = relu ? fmaxf(z, 0.0f) : z;
}

// FC pre-activation: Z3 (GEMM over the conv2 map) + b3 + the two scale
// features' terms (BF16 operands, as the inference kernel multiplies them); A3 = relu
__global__ void fc_tail_kernel(float *__restrict__ Z3, const float *__restrict__ b3, const float *__restrict__ sfeat,
                               int kin, const float *__restrict__ W3tail, int rows, float *__restrict__ A3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * kFc) return;
    const int r = i / kFc, n = i - r * kFc;
    const float s0 = __bfloat162float(__float2bfloat16_rn(sfeat[(size_t)r * kin]));
    const float s1 = __bfloat162float(__float2bfloat16_rn(sfeat[(size_t)r * kin + 1]));
    const float w0 = __bfloat162float(__float2bfloat16_rn(W3tail[n]));
    const float w1 = __bfloat162float(__float2bfloat16_rn(W3tail[kFc + n]));
    const float z = Z3[i] + b3[n] + s0 * w0 + s1 * w1;
    Z3[i] = z;
    A3[i] = fmaxf(z, 0.0f);
}

__global__ void relu_back_kernel(float *__restrict__ d, const float *__restrict__ z, long long total) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total && !(z[i] > 0.0f)) d[i] = 0.0f;
}

// ----------------------------------------------------- inference kernels
// Shape of a conv_tc_kernel group for R x R ROIs: T ROIs per group on a
// padded grid of rows (pitch PR = R + 1, PB = PR^2 rows per ROI, front
// margin F), MT tiles of 128 rows, ROWS rows in all; shared-memory offsets.
// Threads: warps 0-3 stage records, build conv1 operands and run the
// epilogues (warp w reads tensor-memory lanes 32w..32w+31); one thread of
// warp 4 issues the MMAs and the record copies.
template <int R>
struct ConvTile {
    enum : int {
        T = R == 7 ? 14 : (R == 9 ? 8 : 6),
        PR = R + 1,
        PB = PR * PR,
        F = PR + 1,
        MT = (T * PB + 127) / 128,
        ROWS = F + MT * 128 + PR + 1,
        PIX = R * R,
        WHOLE = R * (R + 1),
        KG = kf_of(R) / 8,  // K groups of the FC operand
        SLOTS = 4,          // conv2 tiles in flight (64 accumulator columns each)
        THREADS = 160,
        REC_BYTES = (T * WHOLE * 2 + 15) / 16 * 16,
        OFF_A1 = 0,
        A1_BYTES = 4 * ROWS * 16,
        OFF_W2 = (OFF_A1 + A1_BYTES + 127) / 128 * 128,
        W2_BYTES = kTaps * 4 * kC2 * 16,
        OFF_W1 = OFF_W2 + W2_BYTES,
        W1_BYTES = 2 * kC1 * 16,
        OFF_C1 = OFF_W1 + W1_BYTES,
        C1_BYTES = 2 * 2 * 128 * 16,
        OFF_REC = OFF_C1 + C1_BYTES,
        OFF_X = OFF_REC + 2 * REC_BYTES,
        X_BYTES = T * PIX * 4,
        OFF_FS = (OFF_X + X_BYTES + 15) / 16 * 16,
        OFF_BIAS = OFF_FS + T * 8,
        OFF_BAR = (OFF_BIAS + (kC1 + kC2) * 4 + 15) / 16 * 16,  // conv1[2], conv2[4], records[2], drain; TMEM slot
        SMEM = OFF_BAR + 80 + 128,
    };
    static_assert(MT * 128 >= T * PB, "tiles cover the group");
    static_assert(SMEM <= 113 * 1024, "two CTAs per SM");
    static_assert(MT >= SLOTS, "conv2 ring");
};

// Weight images (BF16, UMMA K-major): W1 [2 K groups][32][8] (taps 9..15
// zero), W2 [9 taps][4 K groups][64][8], W4 [32 K groups][16][8] (outputs
// 8..15 zero), W3 [KF / 8 K groups][256][8] (rows k0 + 2 .. KF zero).
struct ImageOffsets {
    size_t w1, w2, w4, w3, total;  // bf16 elements
};
__host__ __device__ inline ImageOffsets image_offsets(int R) {
    ImageOffsets o;
    o.w1 = 0;
    o.w2 = o.w1 + 16 * kC1;
    o.w4 = o.w2 + (size_t)kTaps * kC1 * kC2;
    o.w3 = o.w4 + (size_t)kFc * 16;
    o.total = o.w3 + (size_t)kf_of(R) * kFc;
    return o;
}

__global__ void weight_image_kernel(const float *__restrict__ par, int R, __nv_bfloat16 *__restrict__ img) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const Offsets o = offsets(R);
    const ImageOffsets io = image_offsets(R);
    if (i >= (long long)io.total) return;
    float v = 0.0f;
    if (i < (long long)io.w2) {  // W1: n = channel, k = tap
        const int j = (int)i, kg = j / (kC1 * 8), rem = j - kg * kC1 * 8, n = rem / 8, k = kg * 8 + rem % 8;
        v = k < kTaps ? par[o.W1 + k * kC1 + n] : 0.0f;
    } else if (i < (long long)io.w4) {  // W2: per tap, n = output channel, k = input channel
        const int j = (int)(i - io.w2), t = j / (4 * kC2 * 8), rem = j - t * 4 * kC2 * 8;
        const int kg = rem / (kC2 * 8), r2 = rem - kg * kC2 * 8, n = r2 / 8, k = kg * 8 + r2 % 8;
        v = par[o.W2 + (size_t)(t * kC1 + k) * kC2 + n];
    } else if (i < (long long)io.w3) {  // W4: n = output, k = FC unit
        const int j = (int)(i - io.w4), kg = j / (16 * 8), rem = j - kg * 16 * 8, n = rem / 8, k = kg * 8 + rem % 8;
        v = n < kOut ? par[o.W4 + (size_t)k * kOut + n] : 0.0f;
    } else {  // W3: n = FC unit, k = operand column
        const long long j = i - (long long)io.w3, kg = j / (kFc * 8), rem = j - kg * kFc * 8;
        const int n = (int)(rem / 8);
        const long long k = kg * 8 + rem % 8;
        v = k < k0_of(R) + 2 ? par[o.W3 + (size_t)k * kFc + n] : 0.0f;
    }
    img[i] = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// records [c0, c0 + n) of the call (n counted from the chunk start; with
// n_dev, at most *n_dev - c0 of them)
__device__ __forceinline__ int chunk_count(int n, const int *n_dev, int c0) {
    if (!n_dev) return n;
    const int m = *n_dev - c0;
    return m < 0 ? 0 : (m < n ? m : n);
}

// records of group `grp` (T per group, the last one ragged) into shared
// memory by one bulk copy of their whole 16-byte blocks; returns the bytes copied
template <int R>
__device__ __forceinline__ uint32_t group_bytes(int grp, int n) {
    typedef ConvTile<R> L;
    const int cnt = min((int)L::T, n - grp * L::T);
    return (uint32_t)(cnt * L::WHOLE * 2) & ~15u;
}

template <int R>
__global__ void __launch_bounds__(160, 2)
    conv_tc_kernel(const uint16_t *__restrict__ rois, int n, const int *__restrict__ n_dev, int c0, float offset,
                   float kadc, const uint4 *__restrict__ w1img, const uint4 *__restrict__ w2img,
                   const float *__restrict__ b1, const float *__restrict__ b2, uint4 *__restrict__ fc_in,
                   float2 *__restrict__ scale, int bulk, int *__restrict__ err) {
    typedef ConvTile<R> L;
    enum { T = L::T, PR = L::PR, PB = L::PB, F = L::F, MT = L::MT, ROWS = L::ROWS, PIX = L::PIX, WHOLE = L::WHOLE,
           SLOTS = L::SLOTS };
    extern __shared__ uint8_t smem_raw[];
    n = chunk_count(n, n_dev, c0);
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t sbase = (raw + 127u) & ~127u;
    uint8_t *base = smem_raw + (sbase - raw);
    const uint32_t sA1 = sbase + L::OFF_A1, sW2 = sbase + L::OFF_W2, sW1 = sbase + L::OFF_W1, sC1 = sbase + L::OFF_C1;
    const uint32_t sRec = sbase + L::OFF_REC;
    const uint32_t sBar = sbase + L::OFF_BAR, bC1 = sBar, bC2 = sBar + 16, bRec = sBar + 48, bDrain = sBar + 64;
    const uint32_t sTmem = sBar + 72;
    float *xs = reinterpret_cast<float *>(base + L::OFF_X);
    float2 *fs = reinterpret_cast<float2 *>(base + L::OFF_FS);
    float *bias = reinterpret_cast<float *>(base + L::OFF_BIAS);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool worker = warp < 4, issuer = tid == 128;
    const int ngroups = (n + T - 1) / T;

    if (tid == 0) {
        for (int b = 0; b < 9; ++b) tc::mbar_init(sBar + 8 * b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights and biases; the conv1 map starts all zero (its margins, zero
    // rows and zero columns are never written)
    for (int i = tid; i < L::W2_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(base + L::OFF_W2)[i] = w2img[i];
    for (int i = tid; i < L::W1_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(base + L::OFF_W1)[i] = w1img[i];
    for (int i = tid; i < L::A1_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(base + L::OFF_A1)[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int i = tid; i < kC1 + kC2; i += blockDim.x) bias[i] = i < kC1 ? b1[i] : b2[i - kC1];
    if (warp == 0) tc::tmem_alloc(sTmem, 256);
    tc::fence_async_smem();
    tc::sync_tc();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(base + L::OFF_BAR + 72);
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    // phases: conv1 / conv2 barriers (waited by the workers), record buffers
    uint32_t ph1[2] = {0u, 0u}, ph2[SLOTS] = {0u, 0u, 0u, 0u};
    uint32_t rec_issued[2] = {0u, 0u}, rec_waited[2] = {0u, 0u};
    bool ok = true;
    auto fetch = [&](int grp, int buf) {  // issuer
        const uint32_t bytes = group_bytes<R>(grp, n);
        const uint32_t bar = bRec + 8 * buf;
        tc::mbar_arrive_expect(bar, bytes);
        if (bytes) tc::bulk_copy(sRec + buf * L::REC_BYTES, rois + (size_t)grp * T * WHOLE, bytes, bar);
        rec_issued[buf]++;
    };
    // conv1 operand of tile mt: the nine neighbours of each grid row (K = 16)
    auto build = [&](int mt) {  // workers
        const int row = mt * 128 + tid, j = row / PB, rem = row - j * PB, y = rem / PR, x = rem - y * PR;
        float v[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) v[t] = 0.0f;
        if (j < T && y < R && x < R) {
#pragma unroll
            for (int t = 0; t < kTaps; ++t) {
                const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
                v[t] = (yy >= 0 && yy < R && xx >= 0 && xx < R) ? xs[j * PIX + yy * R + xx] : 0.0f;
            }
        }
        uint8_t *c1 = base + L::OFF_C1 + (mt & 1) * 4096;
        *reinterpret_cast<uint4 *>(c1 + tid * 16) = tc::pack8(v);
        *reinterpret_cast<uint4 *>(c1 + (128 + tid) * 16) = tc::pack8(v + 8);
    };
    auto mma1 = [&](int mt) {  // issuer
        tc::mma_bf16(tmem + (mt & 1) * 32, tc::smem_desc(sC1 + (mt & 1) * 4096, 2048, 128),
                     tc::smem_desc(sW1, kC1 * 16, 128), tc::instr_desc(128, kC1), 0u);
        tc::mma_commit(bC1 + 8 * (mt & 1));
    };
    auto mma2 = [&](int mt) {  // issuer: nine shifted operand pairs into slot mt % SLOTS
        const uint32_t d = tmem + (mt % SLOTS) * kC2;
        const int row0 = F + mt * 128;
#pragma unroll
        for (int t = 0; t < kTaps; ++t) {
            const int off = (t / 3 - 1) * PR + (t % 3 - 1);
#pragma unroll
            for (int ks = 0; ks < 2; ++ks)
                tc::mma_bf16(d, tc::smem_desc(sA1 + (uint32_t)((2 * ks * ROWS + row0 + off) * 16), ROWS * 16, 128),
                             tc::smem_desc(sW2 + t * 4096 + 2 * ks * 1024, kC2 * 16, 128), tc::instr_desc(128, kC2),
                             (t > 0 || ks > 0) ? 1u : 0u);
        }
        tc::mma_commit(bC2 + 8 * (mt % SLOTS));
    };
    if (bulk && issuer && (int)blockIdx.x < ngroups) fetch(blockIdx.x, 0);

    int it = 0;
    for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x, ++it) {
        const int rb = it & 1, j0 = grp * T, cnt = min(T, n - j0);
        // the next group's records into the other buffer (consumed by the previous group)
        if (bulk && issuer && grp + (int)gridDim.x < ngroups) fetch(grp + gridDim.x, rb ^ 1);
        // (a) scaled pixels (BF16-rounded, as the MMA rounds them) and scale features
        if (worker) {
            const uint16_t *gsrc = rois + (size_t)j0 * WHOLE;
            const uint16_t *ssrc = reinterpret_cast<const uint16_t *>(base + L::OFF_REC + rb * L::REC_BYTES);
            int in_smem = 0;
            if (bulk) {
                ok = tc::mbar_wait(bRec + 8 * rb, rec_waited[rb] & 1u);
                in_smem = (int)group_bytes<R>(grp, n) / 2;
            }
            rec_waited[rb]++;
            for (int jj = warp; jj < T && ok; jj += 4) {
                const bool live = jj < cnt;
                float e[(PIX + 31) / 32];
                float lo = 1e30f, hi = -1e30f;
#pragma unroll
                for (int q = 0; q < (PIX + 31) / 32; ++q) {
                    const int k = lane + 32 * q, w = jj * WHOLE + k;
                    float v = 0.0f;
                    if (live && k < PIX) v = fmaxf(((float)(w < in_smem ? ssrc[w] : gsrc[w]) - offset) * kadc, 1.0f);
                    e[q] = v;
                    if (k < PIX) {
                        lo = fminf(lo, v);
                        hi = fmaxf(hi, v);
                    }
                }
#pragma unroll
                for (int m = 16; m > 0; m >>= 1) {
                    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, m));
                    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, m));
                }
                const float rng = fmaxf(hi - lo, 1.0f), inv = 1.0f / rng;
#pragma unroll
                for (int q = 0; q < (PIX + 31) / 32; ++q) {
                    const int k = lane + 32 * q;
                    if (k < PIX) xs[jj * PIX + k] = live ? bf16_round((e[q] - lo) * inv) : 0.0f;
                }
                if (lane == 0) {
                    fs[jj] = live ? make_float2(logf(rng) * 0.125f, logf(lo) * 0.125f) : make_float2(0.0f, 0.0f);
                    if (live) scale[j0 + jj] = make_float2(lo, rng);
                }
            }
        } else {
            rec_waited[rb]++;
        }
        ok = __syncthreads_and(ok);
        if (!ok) break;
        // (b) conv1: build tile mt + 1 and run the epilogue of tile mt while
        // the MMA of tile mt + 1 is queued; one barrier per tile
        if (worker) {
            build(0);
            tc::fence_async_smem();
        }
        tc::sync_tc();
        if (issuer) mma1(0);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            if (worker) {
                if (mt + 1 < MT) build(mt + 1);  // the buffer of tile mt - 1, whose MMA has ended
                ok = tc::mbar_wait(bC1 + 8 * (mt & 1), ph1[mt & 1]);
                ph1[mt & 1] ^= 1u;
                if (ok) {
                    tc::fence_after();
                    float v[32];
                    tc::tmem_ld32(lane_base + (mt & 1) * 32, v);
                    const int row = mt * 128 + tid, j = row / PB, rem = row - j * PB, y = rem / PR, x = rem - y * PR;
                    if (j < T && y < R && x < R) {
#pragma unroll
                        for (int c = 0; c < kC1; ++c) v[c] = fmaxf(v[c] + bias[c], 0.0f);
#pragma unroll
                        for (int kg = 0; kg < 4; ++kg)
                            *reinterpret_cast<uint4 *>(base + L::OFF_A1 + (size_t)(kg * ROWS + F + row) * 16) =
                                tc::pack8(v + 8 * kg);
                    }
                }
                tc::fence_async_smem();
            }
            tc::fence_before();
            ok = __syncthreads_and(ok);
            tc::fence_after();
            if (!ok) break;
            if (issuer && mt + 1 < MT) mma1(mt + 1);
        }
        if (!ok) break;
        // (c) conv2: SLOTS tiles in flight; the epilogue (bias, ReLU, BF16)
        // writes each ROI's map into the FC operand
        if (issuer)
            for (int q = 0; q < SLOTS; ++q) mma2(q);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int sl = mt % SLOTS;
            if (worker) {
                ok = tc::mbar_wait(bC2 + 8 * sl, ph2[sl]);
                ph2[sl] ^= 1u;
                if (ok) {
                    tc::fence_after();
                    float v[kC2];
                    tc::tmem_ld32(lane_base + sl * kC2, v);
                    tc::tmem_ld32(lane_base + sl * kC2 + 32, v + 32);
                    const int row = mt * 128 + tid, j = row / PB, rem = row - j * PB, y = rem / PR, x = rem - y * PR;
                    if (j < cnt && y < R && x < R) {
                        const int g = j0 + j;  // record within the chunk
                        uint4 *dst = fc_in + ((size_t)(g >> 7) * L::KG + (size_t)(y * R + x) * 8) * 128 + (g & 127);
#pragma unroll
                        for (int c = 0; c < kC2; ++c) v[c] = fmaxf(v[c] + bias[kC1 + c], 0.0f);
#pragma unroll
                        for (int kg = 0; kg < 8; ++kg) dst[(size_t)kg * 128] = tc::pack8(v + 8 * kg);
                    }
                }
            }
            tc::fence_before();
            ok = __syncthreads_and(ok);
            tc::fence_after();
            if (!ok) break;
            if (issuer && mt + SLOTS < MT) mma2(mt + SLOTS);
        }
        if (!ok) break;
        // (d) the two scale features and the zero padding after the map
        if (tid < cnt) {
            const int g = j0 + tid;
            uint4 *dst = fc_in + ((size_t)(g >> 7) * L::KG + (size_t)PIX * 8) * 128 + (g & 127);
            float v[8] = {bf16_round(fs[tid].x), bf16_round(fs[tid].y), 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            dst[0] = tc::pack8(v);
#pragma unroll
            for (int q = 1; q < 8; ++q) dst[(size_t)q * 128] = make_uint4(0u, 0u, 0u, 0u);
        }
        __syncthreads();
    }
    // every MMA this CTA issued and every record copy it started end before
    // its memory is released (bounded waits)
    if (issuer) {
        for (int b = 0; b < 2; ++b)
            while (rec_waited[b] < rec_issued[b]) {
                if (!tc::mbar_wait(bRec + 8 * b, rec_waited[b] & 1u)) break;
                rec_waited[b]++;
            }
        tc::mma_commit(bDrain);
    }
    const bool drained = __syncthreads_and(tc::mbar_wait(bDrain, 0));
    tc::sync_tc();
    if (warp == 0) tc::tmem_free(tmem, 256);
    if ((!ok || !drained) && tid == 0) atomicExch(err, 1);
}

template <int R>
struct FcTile {
    enum : int {
        S = 4,                        // ring stages
        KG = kf_of(R) / 8,            // K groups
        NCH = kf_of(R) / 64,          // K chunks
        A_BYTES = 128 * 64 * 2,       // one chunk of the FC operand
        W_BYTES = kFc * 64 * 2,       // one chunk of the W3 image
        STAGE = A_BYTES + W_BYTES,
        OFF_W4 = S * STAGE,
        W4_BYTES = kFc * 16 * 2,
        OFF_BAR = OFF_W4 + W4_BYTES,  // full[S], empty[S], acc, head, drain, tmem slot
        SMEM = OFF_BAR + 96 + 128,
        HEAD_BYTES = 128 * kFc * 2,   // head A operand (aliases the ring after the K loop)
    };
    static_assert(HEAD_BYTES <= OFF_W4, "head operand inside the ring");
};

template <int R, int LT>
__global__ void __launch_bounds__(128, 1)
    fc_tc_kernel(const uint8_t *__restrict__ fc_in, int n, const int *__restrict__ n_dev, int c0,
                 const uint8_t *__restrict__ w3img, const uint4 *__restrict__ w4img, const float *__restrict__ b3,
                 const float *__restrict__ b4, const float2 *__restrict__ scale, float *__restrict__ start,
                 uint8_t *__restrict__ cls, float count_th, int *__restrict__ err) {
    typedef FcTile<R> L;
    enum { S = L::S, NCH = L::NCH, NST = start_width(LT) };
    extern __shared__ uint8_t smem_raw[];
    n = chunk_count(n, n_dev, c0);
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t sbase = (raw + 127u) & ~127u;
    uint8_t *base = smem_raw + (sbase - raw);
    const uint32_t sBar = sbase + L::OFF_BAR;
    const uint32_t sFull = sBar, sEmpty = sBar + 8 * S, sAcc = sBar + 16 * S, sHead = sAcc + 8, sDrain = sAcc + 16;
    const uint32_t sTmem = sAcc + 24;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ntiles = (n + 127) / 128;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(sFull + 8 * s, 1);
            tc::mbar_init(sEmpty + 8 * s, 1);
        }
        tc::mbar_init(sAcc, 1);
        tc::mbar_init(sHead, 1);
        tc::mbar_init(sDrain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < L::W4_BYTES / 16; i += blockDim.x) reinterpret_cast<uint4 *>(base + L::OFF_W4)[i] = w4img[i];
    if (warp == 0) tc::tmem_alloc(sTmem, 512);
    tc::fence_async_smem();
    tc::sync_tc();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(base + (sTmem - sbase));
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    // ring state (thread 0), per stage: copy phases waited for, copies
    // issued, MMA commits issued (the k-th commit completes phase k)
    uint32_t full_done[S], issued[S], commits[S];
#pragma unroll
    for (int s = 0; s < S; ++s) full_done[s] = issued[s] = commits[s] = 0u;
    uint32_t acc_ph = 0u, head_ph = 0u;
    bool ok = true;
    int tile = blockIdx.x;
    for (; tile < ntiles; tile += gridDim.x) {
        if (tid == 0) {
            const uint8_t *a_src = fc_in + (size_t)tile * L::KG * 128 * 16;
            auto fetch = [&](int c) {
                const int s = c % S;
                const uint32_t dst = sbase + s * L::STAGE;
                tc::mbar_arrive_expect(sFull + 8 * s, L::STAGE);
                tc::bulk_copy(dst, a_src + (size_t)c * L::A_BYTES, L::A_BYTES, sFull + 8 * s);
                tc::bulk_copy(dst + L::A_BYTES, w3img + (size_t)c * L::W_BYTES, L::W_BYTES, sFull + 8 * s);
                issued[s]++;
            };
            for (int c = 0; c < S && c < NCH; ++c) fetch(c);
            for (int c = 0; c < NCH; ++c) {
                const int s = c % S;
                if (!tc::mbar_wait(sFull + 8 * s, full_done[s] & 1u)) {
                    ok = false;
                    break;
                }
                full_done[s]++;
                tc::fence_after();
                const uint32_t a0 = sbase + s * L::STAGE, w0 = a0 + L::A_BYTES;
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma_bf16(tmem, tc::smem_desc(a0 + ks * 2 * 2048, 2048, 128),
                                 tc::smem_desc(w0 + ks * 2 * kFc * 16, kFc * 16, 128), tc::instr_desc(128, kFc),
                                 (c > 0 || ks > 0) ? 1u : 0u);
                tc::mma_commit(sEmpty + 8 * s);
                commits[s]++;
                // refill the stage chunk c - 1 used once its MMAs are done
                // (chunk c's are queued behind them); its commit is the latest on that stage
                if (c >= 1 && c - 1 + S < NCH) {
                    const int sp = (c - 1) % S;
                    if (!tc::mbar_wait(sEmpty + 8 * sp, (commits[sp] - 1u) & 1u)) {
                        ok = false;
                        break;
                    }
                    fetch(c - 1 + S);
                }
            }
            tc::mma_commit(sAcc);
        }
        ok = __syncthreads_and(ok && tc::mbar_wait(sAcc, acc_ph));
        acc_ph ^= 1u;
        if (!ok) break;
        tc::fence_after();
        // FC epilogue: ReLU(D + b3) -> the head's A operand (over the ring)
#pragma unroll 1
        for (int c0f = 0; c0f < kFc; c0f += 16) {
            float v[16];
            tc::tmem_ld16(lane_base + c0f, v);
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = fmaxf(v[q] + __ldg(b3 + c0f + q), 0.0f);
            *reinterpret_cast<uint4 *>(base + (size_t)((c0f / 8) * 128 + tid) * 16) = tc::pack8(v);
            *reinterpret_cast<uint4 *>(base + (size_t)((c0f / 8 + 1) * 128 + tid) * 16) = tc::pack8(v + 8);
        }
        tc::fence_async_smem();
        tc::sync_tc();
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < kFc / 16; ++ks)
                tc::mma_bf16(tmem + kFc, tc::smem_desc(sbase + ks * 2 * 2048, 2048, 128),
                             tc::smem_desc(sbase + L::OFF_W4 + ks * 2 * 16 * 16, 16 * 16, 128), tc::instr_desc(128, 16),
                             ks > 0 ? 1u : 0u);
            tc::mma_commit(sHead);
        }
        ok = __syncthreads_and(tc::mbar_wait(sHead, head_ph));
        head_ph ^= 1u;
        if (!ok) break;
        tc::fence_after();
        float y[16];
        tc::tmem_ld16(lane_base + kFc, y);
        const int g = tile * 128 + tid;
        if (g < n) {
#pragma unroll
            for (int j = 0; j < kOut; ++j) y[j] += __ldg(b4 + j);
            const float2 sc = scale[g];
            start_from_outputs<R, LT>(y, sc.x, sc.y, start + (size_t)g * NST);
            if (LT == QCS_LOCTYPE_GS2D && cls)
                cls[g] = (uint8_t)count_class(y[kCount0], y[kCount0 + 1], y[kCount0 + 2], count_th);
        }
        tc::sync_tc();  // accumulators and the ring are free for the next tile
    }
    // error path: copies still landing and MMAs still running end before the
    // memory is released (bounded waits); the CTA's remaining records get NaN
    // start points, so their fits are rejected and refitted from the plain start
    if (tid == 0) {
        for (int s = 0; s < S; ++s)
            while (full_done[s] < issued[s]) {
                if (!tc::mbar_wait(sFull + 8 * s, full_done[s] & 1u)) break;
                full_done[s]++;
            }
        tc::mma_commit(sDrain);
    }
    const bool drained = __syncthreads_and(tc::mbar_wait(sDrain, 0));
    tc::sync_tc();
    if (warp == 0) tc::tmem_free(tmem, 512);
    if (!ok || !drained) {
        for (int t = tile; t < ntiles; t += gridDim.x) {
            const int g = t * 128 + tid;
            if (g < n) {
#pragma unroll
                for (int j = 0; j < NST; ++j) start[(size_t)g * NST + j] = __int_as_float(0x7fc00000);
                if (LT == QCS_LOCTYPE_GS2D && cls) cls[g] = 0;
            }
        }
        if (tid == 0) atomicExch(err, 1);
    }
}


// -------------------------------------------------------------- host side
struct State {
    int R = 7, batch = 0;
    // training activations of one batch (P = batch * R * R positions)
    float *x1 = nullptr, *z1 = nullptr, *a1 = nullptr, *x2 = nullptr, *z2 = nullptr, *a2 = nullptr;
    float *z3 = nullptr, *a3 = nullptr, *d3 = nullptr, *part = nullptr;
    // inference: weight images, FC operand and scales of one chunk
    __nv_bfloat16 *img = nullptr;
    uint8_t *fc_in = nullptr;
    float2 *scale = nullptr;
    unsigned img_version = 0;
    cudaEvent_t img_ready = nullptr;
    cudaEvent_t scratch_free = nullptr;  // recorded after the last inference call's use of fc_in and scale
    int sms = 148;
};

void destroy(State *st) {
    if (!st) return;
    cudaFree(st->x1);
    cudaFree(st->img);
    cudaFree(st->fc_in);
    if (st->img_ready) cudaEventDestroy(st->img_ready);
    if (st->scratch_free) cudaEventDestroy(st->scratch_free);
    delete st;
}

cudaError_t create(int R, int batch, State **out) {
    *out = nullptr;
    State *st = new State();
    st->R = R;
    st->batch = batch;
    const size_t P = (size_t)batch * R * R;
    const size_t fl = P * (kTaps + 2 * kC1 + kTaps * kC1 + 2 * kC2) + (size_t)batch * 3 * kFc +
                      (size_t)kColsumSplits * kFc;
    cudaError_t e = cudaMalloc((void **)&st->x1, fl * sizeof(float));
    if (e == cudaSuccess) {
        float *a = st->x1 + P * kTaps;
        st->z1 = a;
        a += P * kC1;
        st->a1 = a;
        a += P * kC1;
        st->x2 = a;
        a += P * kTaps * kC1;
        st->z2 = a;
        a += P * kC2;
        st->a2 = a;
        a += P * kC2;
        st->z3 = a;
        a += (size_t)batch * kFc;
        st->a3 = a;
        a += (size_t)batch * kFc;
        st->d3 = a;
        a += (size_t)batch * kFc;
        st->part = a;
    }
    const size_t tiles = kChunk / 128;
    if (e == cudaSuccess) e = cudaMalloc((void **)&st->img, image_offsets(R).total * sizeof(__nv_bfloat16));
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&st->fc_in, tiles * (size_t)kf_of(R) * 128 * 2 + (size_t)kChunk * sizeof(float2));
    if (e == cudaSuccess) st->scale = reinterpret_cast<float2 *>(st->fc_in + tiles * (size_t)kf_of(R) * 128 * 2);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->img_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->scratch_free, cudaEventDisableTiming);
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&st->sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        destroy(st);
        return e;
    }
    *out = st;
    return cudaSuccess;
}

// He-style uniform initialisation (variance 2 / fan_in; 1 / fan_in for the head)
void init_params(float *h, int R, unsigned long long seed) {
    const Offsets o = offsets(R);
    unsigned long long st = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto uni = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (float)((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0f - 1.0f;
    };
    memset(h, 0, o.total * sizeof(float));
    for (size_t i = o.W1; i < o.b1; ++i) h[i] = uni() * sqrtf(6.0f / kTaps);
    for (size_t i = o.W2; i < o.b2; ++i) h[i] = uni() * sqrtf(6.0f / (kTaps * kC1));
    for (size_t i = o.W3; i < o.b3; ++i) h[i] = uni() * sqrtf(6.0f / (float)(k0_of(R) + 2));
    for (size_t i = o.W4; i < o.b4; ++i) h[i] = uni() * sqrtf(3.0f / kFc);
}

cudaError_t forward(State *st, const float *par, const float *feat, int rows, int kin, float *y, cudaStream_t s,
                    float *ws, size_t wsf, int *err) {
    const int R = st->R;
    const Offsets o = offsets(R);
    const long long P = (long long)rows * R * R;
    const int K0 = k0_of(R);
    cudaError_t e;
    im2col1_kernel<<<nblk(P * kTaps), 256, 0, s>>>(feat, kin, rows, R, st->x1);
    if ((e = gemm((int)P, kC1, kTaps, st->x1, kTaps, 1, par + o.W1, kC1, 1, st->z1, kC1, 0.0f, s, ws, wsf, err))) return e;
    bias_act_kernel<<<nblk(P * kC1), 256, 0, s>>>(st->z1, par + o.b1, P, kC1, st->a1, 1);
    im2col2_kernel<<<nblk(P * kTaps * kC1), 256, 0, s>>>(st->a1, rows, R, st->x2);
    if ((e = gemm((int)P, kC2, kTaps * kC1, st->x2, kTaps * kC1, 1, par + o.W2, kC2, 1, st->z2, kC2, 0.0f, s, ws, wsf,
                  err)))
        return e;
    bias_act_kernel<<<nblk(P * kC2), 256, 0, s>>>(st->z2, par + o.b2, P, kC2, st->a2, 1);
    if ((e = gemm(rows, kFc, K0, st->a2, K0, 1, par + o.W3, kFc, 1, st->z3, kFc, 0.0f, s, ws, wsf, err))) return e;
    fc_tail_kernel<<<nblk((long long)rows * kFc), 256, 0, s>>>(st->z3, par + o.b3, feat + R * R, kin,
                                                                par + o.W3 + (size_t)K0 * kFc, rows, st->a3);
    if ((e = gemm(rows, kOut, kFc, st->a3, kFc, 1, par + o.W4, kOut, 1, y, kOut, 0.0f, s, ws, wsf, err))) return e;
    bias_act_kernel<<<nblk((long long)rows * kOut), 256, 0, s>>>(y, par + o.b4, rows, kOut, y, 0);
    return cudaGetLastError();
}

cudaError_t backward(State *st, const float *par, float *grad, const float *feat, int rows, int kin, const float *dy,
                     cudaStream_t s, float *ws, size_t wsf, int *err) {
    const int R = st->R;
    const Offsets o = offsets(R);
    const long long P = (long long)rows * R * R;
    const int K0 = k0_of(R);
    cudaError_t e;
    // head
    if ((e = gemm(kFc, kOut, rows, st->a3, 1, kFc, dy, kOut, 1, grad + o.W4, kOut, 0.0f, s, ws, wsf, err))) return e;
    if ((e = column_sums(dy, rows, kOut, grad + o.b4, st->part, s))) return e;
    if ((e = gemm(rows, kFc, kOut, dy, kOut, 1, par + o.W4, 1, kOut, st->d3, kFc, 0.0f, s, ws, wsf, err))) return e;
    relu_back_kernel<<<nblk((long long)rows * kFc), 256, 0, s>>>(st->d3, st->z3, (long long)rows * kFc);
    // FC: map rows and the two scale rows of W3
    if ((e = gemm(K0, kFc, rows, st->a2, 1, K0, st->d3, kFc, 1, grad + o.W3, kFc, 0.0f, s, ws, wsf, err))) return e;
    if ((e = gemm(2, kFc, rows, feat + R * R, 1, kin, st->d3, kFc, 1, grad + o.W3 + (size_t)K0 * kFc, kFc, 0.0f, s, ws,
                  wsf, err)))
        return e;
    if ((e = column_sums(st->d3, rows, kFc, grad + o.b3, st->part, s))) return e;
    // dA2 = d3 W3[map rows]^T, over a2 (no longer needed)
    if ((e = gemm(rows, K0, kFc, st->d3, kFc, 1, par + o.W3, 1, kFc, st->a2, K0, 0.0f, s, ws, wsf, err))) return e;
    relu_back_kernel<<<nblk(P * kC2), 256, 0, s>>>(st->a2, st->z2, P * kC2);
    // conv2
    if ((e = gemm(kTaps * kC1, kC2, (int)P, st->x2, 1, kTaps * kC1, st->a2, kC2, 1, grad + o.W2, kC2, 0.0f, s, ws, wsf,
                  err)))
        return e;
    if ((e = column_sums(st->a2, P, kC2, grad + o.b2, st->part, s))) return e;
    // dX2 = dZ2 W2^T over x2, then dA1 over a1
    if ((e = gemm((int)P, kTaps * kC1, kC2, st->a2, kC2, 1, par + o.W2, 1, kC2, st->x2, kTaps * kC1, 0.0f, s, ws, wsf,
                  err)))
        return e;
    col2im2_kernel<<<nblk(P * kC1), 256, 0, s>>>(st->x2, rows, R, st->a1);
    relu_back_kernel<<<nblk(P * kC1), 256, 0, s>>>(st->a1, st->z1, P * kC1);
    // conv1
    if ((e = gemm(kTaps, kC1, (int)P, st->x1, 1, kTaps, st->a1, kC1, 1, grad + o.W1, kC1, 0.0f, s, ws, wsf, err)))
        return e;
    if ((e = column_sums(st->a1, P, kC1, grad + o.b1, st->part, s))) return e;
    return cudaGetLastError();
}

template <int R, int LT>
static cudaError_t launch_chunks(State *st, const float *par, const qcs_loc_para *p, const uint16_t *rois, int n,
                                 const int *n_dev, float *out, uint8_t *cls, float th, cudaStream_t s, int *err) {
    typedef ConvTile<R> CT;
    typedef FcTile<R> FT;
    const Offsets o = offsets(R);
    const ImageOffsets io = image_offsets(R);
    auto k1 = conv_tc_kernel<R>;
    auto k2 = fc_tc_kernel<R, LT>;
    cudaError_t e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CT::SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FT::SMEM);
    if (e != cudaSuccess) return e;
    const uint4 *img = reinterpret_cast<const uint4 *>(st->img);
    // records reach shared memory by bulk copy when they start on a 16-byte boundary
    const bool bulk = (reinterpret_cast<uintptr_t>(rois) & 15) == 0;
    for (int c0 = 0; c0 < n; c0 += kChunk) {
        const int cn = n - c0 < kChunk ? n - c0 : kChunk;
        const int groups = (cn + CT::T - 1) / CT::T, tiles = (cn + 127) / 128;
        const int g1 = groups < 2 * st->sms ? groups : 2 * st->sms;
        const int g2 = tiles < st->sms ? tiles : st->sms;
        k1<<<g1, CT::THREADS, CT::SMEM, s>>>(rois + (size_t)c0 * R * (R + 1), cn, n_dev, c0, p->Offset, p->KAdc,
                                             img + io.w1 / 8, img + io.w2 / 8, par + o.b1, par + o.b2,
                                             reinterpret_cast<uint4 *>(st->fc_in), st->scale, bulk ? 1 : 0, err);
        k2<<<g2, 128, FT::SMEM, s>>>(st->fc_in, cn, n_dev, c0, reinterpret_cast<const uint8_t *>(st->img + io.w3),
                                     img + io.w4 / 8, par + o.b3, par + o.b4, st->scale,
                                     out + (size_t)c0 * start_width(LT), cls ? cls + c0 : nullptr, th, err);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t start_points(State *st, const float *par, unsigned version, int loc_type, const qcs_loc_para *p,
                         const uint16_t *rois, int n, const int *n_dev, float *out, uint8_t *cls, float th,
                         cudaStream_t s, int *err) {
    if (n <= 0) return cudaSuccess;
    // the weight images are rebuilt only after a parameter change (rules as the MLP's fused path)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return e;
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    if (st->img_version != version) {
        weight_image_kernel<<<nblk((long long)image_offsets(st->R).total), 256, 0, s>>>(par, st->R, st->img);
        if (!capturing) {
            e = cudaEventRecord(st->img_ready, s);
            if (e != cudaSuccess) return e;
            st->img_version = version;
        }
    } else if (!capturing) {
        e = cudaStreamWaitEvent(s, st->img_ready, 0);
        if (e != cudaSuccess) return e;
    } else if (cudaEventQuery(st->img_ready) != cudaSuccess) {
        return cudaErrorNotReady;
    }
    // fc_in and scale hold one call's intermediate results: a call on another stream waits until the call before
    // it has used them (outside stream capture: a graph holding this call must not run beside another call of the
    // same network)
    if (!capturing && (e = cudaStreamWaitEvent(s, st->scratch_free, 0)) != cudaSuccess) return e;
    const int R = st->R;
    e = cudaErrorInvalidValue;
#define QCS_CONV_CASE(RR, LTT) \
    else if (R == RR && loc_type == LTT) e = launch_chunks<RR, LTT>(st, par, p, rois, n, n_dev, out, cls, th, s, err);
    if (false) {
    }
    QCS_CONV_CASE(7, QCS_LOCTYPE_GS2D)
    QCS_CONV_CASE(9, QCS_LOCTYPE_GS2D)
    QCS_CONV_CASE(11, QCS_LOCTYPE_GS2D)
    QCS_CONV_CASE(7, QCS_LOCTYPE_AS3D)
    QCS_CONV_CASE(9, QCS_LOCTYPE_AS3D)
    QCS_CONV_CASE(11, QCS_LOCTYPE_AS3D)
    QCS_CONV_CASE(7, kTwo)
    QCS_CONV_CASE(9, kTwo)
    QCS_CONV_CASE(11, kTwo)
#undef QCS_CONV_CASE
    if (e != cudaSuccess || capturing) return e;
    return cudaEventRecord(st->scratch_free, s);
}

}  // namespace conv
}  // namespace learned
}  // namespace qcs
