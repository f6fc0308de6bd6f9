// ROI extraction (LDROIExtractData_TypeDef, reference directory
// MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/SubregionExtraction/) on the
// device, with no host synchronisation per batch of frames:
//
//   background_kernel  9x9 ring-minimum background, averaged over the left and
//                      right neighbour inside each aligned 32-column group,
//                      subtracted and clamped at 0
//                      (LDROIExtraction_ImageFiltering.cu:125-267)
//   variance_kernel    mean and mean square of the 4-quadrant minimum over the
//                      central patch (LDROIExtraction.cu:140-177,
//                      _ImageFiltering.cu:503-533)
//   detect_kernel      separable 5-tap Gaussian (horizontal then vertical, each
//                      pass truncated to uint16 like the reference's
//                      intermediate images) fused with the 3x3 local-maximum
//                      test (_ImageFiltering.cu:85-121, 286-454;
//                      LDROIExtraction_ROIExtraction.cu:25-164); GS2D with
//                      multi-emitter fitting detects on the background-removed
//                      image itself, as the reference does (its sharpen step
//                      writes into a scratch image nothing reads,
//                      _ImageFiltering.cu:96-104, 675)
//   scan_kernel        exclusive scan of detections per 4096-pixel chunk
//   compact_kernel     ordered compaction of the detections into sorted keys
//   cut_kernel         single/multi classification, ROI cut and header, one
//                      warp per record (_ROIExtraction.cu:181-302)
//   WLE pre-pass       launch_wle_presorted over the batch's records and keys
//                      (LDROIExtraction.cu:124-132)
//
// Differences from the reference that a caller can see, each deliberate:
//   * records of a batch come in pixel order (y * width + x over the stacked
//     batch); the reference appends them in atomicAdd arrival order;
//   * the variance is formed from exact integer sums, each mean rounded once
//     to float; the reference adds float terms with atomics in GPU arrival
//     order, so its value varies in the last bits from run to run;
//   * more than QCS_MAX_POINT_NUM detections in one batch, or more records
//     than the context holds, are dropped and counted instead of written past
//     the end of the buffers;
//   * frames already in device memory (QCS_IMAGE_SOURCE_GPU) are read in
//     place; the reference rejects that source.
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"
#include "qcs_kernels.h"

namespace qcs {
namespace {

constexpr int kChunk = 4096;         // pixels per ordering chunk (one compaction block)
constexpr int kCompactThreads = 256; // 16 pixels per thread
constexpr int kBgPairs = 128;        // column pairs per block (two columns per thread)
constexpr int kBgThreads = 2 * kBgPairs; // two row halves
constexpr int kBgCols = 2 * kBgPairs, kBgRows = 32, kBgWords = kBgCols / 2 + 4;
constexpr int kDetTX = 128, kDetTY = 32, kDetThreads = 256;
constexpr int kVarBlocks = 64, kVarThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kCutThreads = 256;     // one warp per record

// Device state words of an extraction context.
enum { kStAccum = 0, kStBase = 1, kStBatchN = 2, kStDropped = 3, kStDetected = 4, kStNum = 8 };

// Position-image flags written by detect_kernel.
enum : uint8_t { kMarked = 1, kCandidate = 2 };

struct Taps {
    float t[5];
};

struct DetectPara {
    int W, H0, Hb, half, low_th;
};

struct EmitPara {
    int W, H0, R, multi, start_frame, npx;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// Exact int <-> float conversions on the FMA pipe (the conversion pipe runs
// at a quarter of its rate).  For 0 <= u < 2^23 the float with bits
// 0x4B000000 | u is 2^23 + u, so subtracting 2^23 gives (float)u exactly.
// For 0 <= v < 2^23, v + 2^23 rounded toward zero is 2^23 + floor(v): its low
// 23 bits are floor(v), the truncating conversion of the reference's
// float -> unsigned short stores (saturated at 65535 first).
__device__ __forceinline__ float u2f(uint32_t u) { return __fsub_rn(__uint_as_float(0x4B000000u | u), 8388608.0f); }
__device__ __forceinline__ uint32_t trunc_u16(float v) {
    return __float_as_uint(__fadd_rz(fminf(v, 65535.0f), 8388608.0f)) - 0x4B000000u;
}
// trunc_u16 as a float (the value a uint16 intermediate image would hold)
__device__ __forceinline__ float trunc_u16f(float v) { return __fsub_rn(__fadd_rz(fminf(v, 65535.0f), 8388608.0f), 8388608.0f); }

// dst[r * COLS + c] = (float) src pixel (clamp(gx0 + c), clamp(gy0 + r)) for a
// ROWS x COLS tile.  Every load of a thread is issued before the first store,
// so the loads of a thread overlap instead of each waiting out the latency.
template <int ROWS, int COLS, int THREADS>
__device__ __forceinline__ void load_tile_clamped_f(float *dst, const uint16_t *__restrict__ src, int W, int H, int gx0,
                                                    int gy0) {
    constexpr int N = ROWS * COLS, PER = (N + THREADS - 1) / THREADS;
    uint16_t v[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * THREADS;
        if (i < N) {
            const int r = i / COLS, c = i - r * COLS;
            v[j] = src[(size_t)clampi(gy0 + r, 0, H - 1) * W + clampi(gx0 + c, 0, W - 1)];
        }
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * THREADS;
        if (i < N) dst[i] = u2f(v[j]);
    }
}

// Background removal, two adjacent columns per thread with the pixel pairs
// packed in 32-bit words (16-bit SIMD minima).  Per output pixel (x, y) the
// ring sum is sum_i min(P(x-4+i, y-4), P(x+4, y-4+i), P(x+4-i, y+4),
// P(x-4, y+4-i)), i = 0..7 (the four points of each quarter turn of the 9x9
// border); the right and left border columns slide down the strip in
// registers.  All sums are integers, so the float steps that follow (ring
// sum / 8, three-neighbour sum, / 3) round exactly as the reference's.
__global__ void __launch_bounds__(kBgThreads) background_kernel(const uint16_t *__restrict__ raw,
                                                                uint16_t *__restrict__ bg, int W, int H) {
    // t[r][k]: pixels (x0 - 4 + 2k, x0 - 3 + 2k) of row y0 - 4 + r (clamped), low half first
    __shared__ uint32_t t[kBgRows + 8][kBgWords];
    const int x0 = blockIdx.x * kBgCols, y0 = blockIdx.y * kBgRows;
    const uintptr_t align = reinterpret_cast<uintptr_t>(raw);
    if ((W & 3) == 0 && (align & 7) == 0 && x0 >= 4 && x0 - 4 + 2 * kBgWords <= W && y0 >= 4 && y0 + kBgRows + 4 <= H) {
        // interior tile: 8-byte loads (x0 - 4 and W are multiples of 4 pixels)
        constexpr int kQ = kBgWords / 2, N = (kBgRows + 8) * kQ, PER = (N + kBgThreads - 1) / kBgThreads;
        uint2 v[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kBgThreads;
            if (i < N) {
                const int r = i / kQ, k = i - r * kQ;
                v[j] = *reinterpret_cast<const uint2 *>(raw + (size_t)(y0 - 4 + r) * W + x0 - 4 + 4 * k);
            }
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kBgThreads;
            if (i < N) {
                const int r = i / kQ, k = i - r * kQ;
                t[r][2 * k] = v[j].x;
                t[r][2 * k + 1] = v[j].y;
            }
        }
    } else {
        constexpr int N = (kBgRows + 8) * kBgWords, PER = (N + kBgThreads - 1) / kBgThreads;
        uint32_t v[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kBgThreads;
            if (i < N) {
                const int r = i / kBgWords, k = i - r * kBgWords;
                const uint16_t *row = raw + (size_t)clampi(y0 - 4 + r, 0, H - 1) * W;
                const int gx = x0 - 4 + 2 * k;
                v[j] = (uint32_t)row[clampi(gx, 0, W - 1)] | ((uint32_t)row[clampi(gx + 1, 0, W - 1)] << 16);
            }
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kBgThreads;
            if (i < N) {
                const int r = i / kBgWords, k = i - r * kBgWords;
                t[r][k] = v[j];
            }
        }
    }
    __syncthreads();
    const int q = threadIdx.x % kBgPairs;  // word of the left border column
    const int r0 = (threadIdx.x / kBgPairs) * (kBgRows / 2), r1 = r0 + kBgRows / 2;
    const int x = x0 + 2 * q;              // even column; the thread also owns x + 1
    const int g = q & 15;                  // pair index inside the aligned 32-column group
    uint32_t rc[8], lc[8];                 // right column rows r..r+7, left column rows r+1..r+8
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        rc[i] = t[r0 + i][q + 4];
        lc[i] = t[r0 + 1 + i][q];
    }
    const bool store_wide = ((W & 1) == 0) && ((reinterpret_cast<uintptr_t>(bg) & 3) == 0);
    for (int r = r0; r < r1; ++r) {
        uint32_t tw[5], bw[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            tw[k] = t[r][q + k];
            bw[k] = t[r + 8][q + k];
        }
        int se = 0, so = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t top = (i & 1) ? __byte_perm(tw[(i - 1) / 2], tw[(i + 1) / 2], 0x5432) : tw[i / 2];
            const uint32_t bot = (i & 1) ? __byte_perm(bw[(7 - i) / 2], bw[(9 - i) / 2], 0x5432) : bw[4 - i / 2];
            const uint32_t m = __vminu2(__vminu2(top, rc[i]), __vminu2(bot, lc[7 - i]));
            se += (int)(m & 0xFFFFu);
            so += (int)(m >> 16);
        }
        // neighbours inside the aligned 32-column group
        const int so_prev = __shfl_up_sync(0xffffffffu, so, 1);
        const int se_next = __shfl_down_sync(0xffffffffu, se, 1);
        const int sum_e = (g == 0 ? se : so_prev) + se + so;
        const int sum_o = se + so + (g == 15 ? so : se_next);
        const float mean_e = __fdiv_rn(__fmul_rn(u2f((uint32_t)sum_e), 0.125f), 3.0f);
        const float mean_o = __fdiv_rn(__fmul_rn(u2f((uint32_t)sum_o), 0.125f), 3.0f);
        const uint32_t cw = t[r + 4][q + 2];
        const uint32_t ve = trunc_u16(fmaxf(__fsub_rn(u2f(cw & 0xFFFFu), mean_e), 0.0f));
        const uint32_t vo = trunc_u16(fmaxf(__fsub_rn(u2f(cw >> 16), mean_o), 0.0f));
        const int y = y0 + r;
        if (y < H) {
            uint16_t *out = bg + (size_t)y * W;
            if (store_wide && x + 1 < W) {
                *reinterpret_cast<uint32_t *>(out + x) = ve | (vo << 16);
            } else {
                if (x < W) out[x] = (uint16_t)ve;
                if (x + 1 < W) out[x + 1] = (uint16_t)vo;
            }
        }
        if (r + 1 < r1) {
#pragma unroll
            for (int i = 0; i < 7; ++i) {
                rc[i] = rc[i + 1];
                lc[i] = lc[i + 1];
            }
            rc[7] = t[r + 8][q + 4];
            lc[7] = t[r + 9][q];
        }
    }
}

// Exact sums of the 4-quadrant minimum over the S x S patch whose corner is
// (cx, cy), accumulated over blocks with 64-bit integer atomics (the result
// does not depend on their order).  The last block to finish forms
// var[0] = mean square - mean^2 (at least 100) and clears acc[0..2].
__global__ void __launch_bounds__(kVarThreads) variance_kernel(const uint16_t *__restrict__ bg, int W, int cx, int cy,
                                                               int S, unsigned long long *__restrict__ acc,
                                                               float *__restrict__ var) {
    unsigned long long s1 = 0, s2 = 0;
    const int total = S * S;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const int X = cx + g % S, Y = cy + g / S;
        const unsigned d1 = bg[(size_t)Y * W + X], d2 = bg[(size_t)Y * W + X - S];
        const unsigned d3 = bg[(size_t)(Y - S) * W + X], d4 = bg[(size_t)(Y - S) * W + X - S];
        const unsigned d = min(min(d1, d2), min(d3, d4));
        s1 += d;
        s2 += (unsigned long long)d * d;
    }
    for (int o = 16; o; o >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    __shared__ unsigned long long w1[kVarThreads / 32], w2[kVarThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        w1[warp] = s1;
        w2[warp] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0, b = 0;
        for (int i = 0; i < kVarThreads / 32; ++i) {
            a += w1[i];
            b += w2[i];
        }
        atomicAdd(&acc[0], a);
        atomicAdd(&acc[1], b);
        __threadfence();
        const unsigned long long ticket = atomicAdd(&acc[2], 1ull);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            const unsigned long long A = atomicAdd(&acc[0], 0ull), B = atomicAdd(&acc[1], 0ull);
            const double T = (double)total;
            const float mx = (float)__ddiv_rn((double)A, T);
            const float mx2 = (float)__ddiv_rn((double)B, T);
            float v = __fsub_rn(mx2, __fmul_rn(mx, mx));
            if (v < 100.0f) v = 100.0f;
            var[0] = v;
            acc[0] = 0;
            acc[1] = 0;
            acc[2] = 0;
        }
    }
}

// Smoothing and detection on float tiles holding integer values (every
// intermediate image of the reference is uint16, so each pass ends with the
// truncation to uint16, kept in float).
template <bool SMOOTH>
__global__ void __launch_bounds__(kDetThreads) detect_kernel(const uint16_t *__restrict__ bg, uint8_t *__restrict__ pos,
                                                             int *__restrict__ chunk_count, const float *__restrict__ var,
                                                             Taps taps, DetectPara dp) {
    constexpr int kIn = SMOOTH ? (kDetTY + 6) * (kDetTX + 6) : (kDetTY + 2) * (kDetTX + 2);
    // background-removed tile, then (same storage) the smoothed tile
    __shared__ float buf[kIn];
    __shared__ float ht[SMOOTH ? (kDetTY + 6) * (kDetTX + 2) : 1];
    const int W = dp.W, Hb = dp.Hb;
    const int x0 = blockIdx.x * kDetTX, y0 = blockIdx.y * kDetTY;
    float *sm = buf;  // sm[r * (kDetTX + 2) + c] is pixel (x0 - 1 + c, y0 - 1 + r)
    if (SMOOTH) {
        // halo 3, coordinates clamped like every read of the reference's filters
        load_tile_clamped_f<kDetTY + 6, kDetTX + 6, kDetThreads>(buf, bg, W, Hb, x0 - 3, y0 - 3);
        __syncthreads();
        // horizontal pass: ht[r][c] is column x0 - 1 + c of row clamp(y0 - 3 + r)
        for (int i = threadIdx.x; i < (kDetTY + 6) * (kDetTX + 2); i += kDetThreads) {
            const int r = i / (kDetTX + 2), c = i - r * (kDetTX + 2);
            const float *row = buf + r * (kDetTX + 6) + c;
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 5; ++k) acc = __fmaf_rn(row[k], taps.t[k], acc);
            ht[i] = trunc_u16f(acc);
        }
        __syncthreads();
        // vertical pass into buf
        for (int i = threadIdx.x; i < (kDetTY + 2) * (kDetTX + 2); i += kDetThreads) {
            const float *col = ht + i;
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 5; ++k) acc = __fmaf_rn(col[k * (kDetTX + 2)], taps.t[k], acc);
            sm[i] = trunc_u16f(acc);
        }
    } else {
        load_tile_clamped_f<kDetTY + 2, kDetTX + 2, kDetThreads>(buf, bg, W, Hb, x0 - 1, y0 - 1);
    }
    __syncthreads();
    const float sd = __fsqrt_rn(var[0]);
    const float th = __fmul_rn(dp.low_th ? 8.5f : 9.5f, sd);
    const float th1 = __fmul_rn(dp.low_th ? 3.5f : 3.8f, sd);
    // one column per thread, rows r0, r0 + kRowStep, ...: the row inside the
    // frame advances without a division per pixel
    constexpr int kRowStep = kDetThreads / kDetTX, L = kDetTX + 2;
    const int c = threadIdx.x % kDetTX, r0 = threadIdx.x / kDetTX;
    const int x = x0 + c;
    const bool col_in = x >= dp.half && x < W - dp.half;
    int y = y0 + r0;
    int ry = y % dp.H0;
    for (int r = r0; r < kDetTY; r += kRowStep, y += kRowStep) {
        if (y >= Hb) break;
        if (x < W) {
            uint8_t flag = 0;
            if (col_in && ry >= dp.half && ry < dp.H0 - dp.half) {
                const float *p = sm + r * L + c;
                const float C = p[L + 1];
                if (C >= th) {
                    const float v00 = p[0], v01 = p[1], v02 = p[2];
                    const float v10 = p[L], v12 = p[L + 2];
                    const float v20 = p[2 * L], v21 = p[2 * L + 1], v22 = p[2 * L + 2];
                    const int j1 = (v00 > th1) + (v01 > th1) + (v02 > th1) + (v10 > th1) + (v12 > th1) + (v20 > th1) +
                                   (v21 > th1) + (v22 > th1);
                    const int ji = (C > v01) + (C >= v12) + (C >= v21) + (C > v10);
                    const int jo = (C > v00) + (C > v02) + (C > v20) + (C > v22);
                    if (j1 >= 7 && ji == 4 && jo >= 3) {
                        flag = kMarked;
                        if (jo == 4) {
                            flag |= kCandidate;
                            atomicAdd(&chunk_count[(y * W + x) / kChunk], 1);
                        }
                    }
                }
            }
            pos[(size_t)y * W + x] = flag;
        }
        ry += kRowStep;
        if (ry >= dp.H0) ry -= dp.H0;
    }
}

// Inclusive scan over the block; returns the exclusive prefix, *total = sum.
template <int THREADS>
__device__ __forceinline__ int block_exclusive_scan(int v, int *total) {
    __shared__ int warp_sums[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < THREADS / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < THREADS / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    const int before = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[THREADS / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// Chunk counts -> exclusive chunk offsets (in place); decides how many of the
// batch's detections are kept and where they start in the record buffer.
__global__ void __launch_bounds__(kScanThreads) scan_kernel(int *__restrict__ chunk, int nchunks,
                                                            int *__restrict__ state, int batch_cap, int capacity) {
    const int per = (nchunks + kScanThreads - 1) / kScanThreads;
    const int b = threadIdx.x * per, e = min(b + per, nchunks);
    int sum = 0;
    for (int i = b; i < e; ++i) sum += chunk[i];
    int total = 0;
    int run = block_exclusive_scan<kScanThreads>(sum, &total);
    for (int i = b; i < e; ++i) {
        const int c = chunk[i];
        chunk[i] = run;
        run += c;
    }
    if (threadIdx.x == 0) {
        const int acc = state[kStAccum];
        int n = min(total, batch_cap);
        n = min(n, capacity - acc);
        if (n < 0) n = 0;
        state[kStBase] = acc;
        state[kStBatchN] = n;
        state[kStAccum] = acc + n;
        state[kStDropped] += total - n;
        state[kStDetected] = total;
    }
}

// Ordered compaction: the k-th detection of the batch in pixel order gets
// record base + k; its key frame << 32 | y << 16 | x goes to keys[base + k].
__global__ void __launch_bounds__(kCompactThreads) compact_kernel(const uint8_t *__restrict__ pos,
                                                                  const int *__restrict__ chunk_off,
                                                                  const int *__restrict__ state,
                                                                  unsigned long long *__restrict__ keys, EmitPara ep) {
    const int p0 = blockIdx.x * kChunk + threadIdx.x * 16;
    uint8_t f[16];
    if (p0 + 16 <= ep.npx) {
        const uint4 v = *reinterpret_cast<const uint4 *>(pos + p0);
        memcpy(f, &v, 16);
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) f[j] = (p0 + j < ep.npx) ? pos[p0 + j] : 0;
    }
    int cnt = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) cnt += (f[j] & kCandidate) ? 1 : 0;
    int total;
    int k = chunk_off[blockIdx.x] + block_exclusive_scan<kCompactThreads>(cnt, &total);
    if (cnt == 0) return;
    const int base = state[kStBase], n = state[kStBatchN];
    for (int j = 0; j < 16; ++j) {
        if (!(f[j] & kCandidate)) continue;
        if (k < n) {
            const int p = p0 + j;
            const int yb = p / ep.W, x = p - yb * ep.W;
            const int fb = yb / ep.H0, y = yb - fb * ep.H0;
            const unsigned long long frame = (unsigned long long)(ep.start_frame + fb);
            keys[base + k] = (frame << 32) | ((unsigned long long)y << 16) | (unsigned long long)x;
        }
        ++k;
    }
}

// One warp per record: single/multi classification from the position image
// (LDROIExtraction_ROIExtraction.cu:181-243), the R x R cut of the raw frame
// and the 5 header words (_ROIExtraction.cu:257-302).
__global__ void __launch_bounds__(kCutThreads) cut_kernel(const unsigned long long *__restrict__ keys,
                                                          const int *__restrict__ state, const uint8_t *__restrict__ pos,
                                                          const uint16_t *__restrict__ raw, uint16_t *__restrict__ rois,
                                                          EmitPara ep) {
    const int base = state[kStBase], n = state[kStBatchN];
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (kCutThreads / 32);
    const int R = ep.R, half = R / 2, RR = R * R, whole = R * (R + 1), W = ep.W;
    for (int k = blockIdx.x * (kCutThreads / 32) + (threadIdx.x >> 5); k < n; k += warps) {
        const unsigned long long key = keys[base + k];
        const int x = (int)(key & 0xFFFF), y = (int)((key >> 16) & 0xFFFF);
        const int frame = (int)(key >> 32);
        const int yb = (frame - ep.start_frame) * ep.H0 + y;
        int type = QCS_ROITYPE_SINGLE;
        if (ep.multi) {
            int nb = 0, nb3 = 0;
            for (int i = lane; i < RR; i += 32) {
                const int r = i / R, c = i - r * R;
                const int m = pos[(size_t)(yb + r - half) * W + (x + c - half)] & kMarked;
                nb += m;
                if (r >= half - 1 && r <= half + 1 && c >= half - 1 && c <= half + 1) nb3 += m;
            }
            for (int o = 16; o; o >>= 1) {
                nb += __shfl_xor_sync(0xffffffffu, nb, o);
                nb3 += __shfl_xor_sync(0xffffffffu, nb3, o);
            }
            type = (nb - nb3 > 0) ? QCS_ROITYPE_MULTI : QCS_ROITYPE_SINGLE;
        }
        uint16_t *rec = rois + (size_t)(base + k) * whole;
        for (int i = lane; i < RR; i += 32) {
            const int r = i / R, c = i - r * R;
            rec[i] = raw[(size_t)(yb - half + r) * W + (x - half + c)];
        }
        if (lane < 5) {
            const uint16_t h[5] = {(uint16_t)x, (uint16_t)y, (uint16_t)(frame % 65536), (uint16_t)(frame / 65536),
                                   (uint16_t)type};
            rec[RR + lane] = h[lane];
        }
    }
}

// The smoothing taps of LDROIExtractData_TypeDef::FilterInit
// (LDROIExtraction_ImageFiltering.cu:22-67), computed on the host as there
// (host code is built with -ffp-contract=off: every operation rounded).
void filter_taps(int R, int loc_type, int multi, float *taps) {
    float sigma = 0.5f + (R - 7) * (1.0f - 0.5f) / (11 - 7);
    if (sigma < 0.5f) sigma = 0.5f;
    if (loc_type == QCS_LOCTYPE_AS3D)
        sigma *= 1.5f;
    else if (multi == 0 && loc_type == QCS_LOCTYPE_GS2D)
        sigma *= 1.2f;
    const float neg = -1 / (2 * sigma * sigma);
    const float center = (float)(5 / 2);
    for (int c = 0; c < 5; ++c) taps[c] = expf((c - center) * (c - center) * neg);
    float sum = 0;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) sum += taps[i] * taps[j];
    sum = sqrtf(1.0f / sum);
    for (int c = 0; c < 5; ++c) taps[c] = taps[c] * sum;
}

}  // namespace
}  // namespace qcs

using qcs::fail;

struct qcs_extract_data {
    qcs_loc_para para;
    int W, H0, R, whole, max_batch, capacity;
    long long max_px;
    int nchunks_max;
    qcs::Taps taps;
    uint16_t *d_raw = nullptr, *d_bg = nullptr;
    uint8_t *d_pos = nullptr;
    int *d_chunk = nullptr, *d_state = nullptr;
    float *d_var = nullptr;
    unsigned long long *d_var_acc = nullptr;
    unsigned long long *d_keys = nullptr;
    uint16_t *d_rois = nullptr;
    float *d_wle = nullptr;
    uint16_t *h_rois = nullptr;
    float *h_wle = nullptr;
    int *h_state = nullptr;
    int h_copied = 0;
    cudaStream_t stream = nullptr, last = nullptr;
    cudaEvent_t done = nullptr;  // recorded after the work of each call
    int first_frame = -1, end_frame = -1;
    // host frames: two device buffers filled in turn on a copy stream, so the
    // copy of one batch overlaps the kernels of the batch before it
    uint16_t *d_raw2 = nullptr;
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr};    // a buffer's frames have arrived
    cudaEvent_t consumed[2] = {nullptr, nullptr};  // the kernels that read a buffer are done
    bool used[2] = {false, false};
    int next_raw = 0;
};

namespace {

// Orders a call on stream s after the context's previous work (which may
// have been issued on another stream).
cudaError_t order_after_last(qcs_extract_data *c, cudaStream_t s) {
    if (s == c->last) return cudaSuccess;
    return cudaStreamWaitEvent(s, c->done, 0);
}

cudaError_t mark_done(qcs_extract_data *c, cudaStream_t s) {
    c->last = s;
    return cudaEventRecord(c->done, s);
}

// Brings the device state words into h_state (waits for the last call).
int read_state(qcs_extract_data *c) {
    QCS_CUDA(cudaMemcpyAsync(c->h_state, c->d_state, qcs::kStNum * sizeof(int), cudaMemcpyDeviceToHost, c->last),
             "read extraction counters");
    QCS_CUDA(cudaStreamSynchronize(c->last), "extraction");
    return QCS_OK;
}

}  // namespace

extern "C" {

int qcs_extract_max_batched_num(int image_width, int image_high) {
    if (image_width + image_high <= 0) return 1;
    int n = 2048 * 2 / (image_width + image_high);
    n = n / 2 * 2;
    return n < 1 ? 1 : n;
}

int qcs_extract_deinit(qcs_extract_data *c) {
    if (!c) return QCS_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->last && c->last != c->stream) cudaStreamSynchronize(c->last);
    cudaFree(c->d_raw);
    cudaFree(c->d_bg);
    cudaFree(c->d_pos);
    cudaFree(c->d_chunk);
    cudaFree(c->d_state);
    cudaFree(c->d_var);
    cudaFree(c->d_var_acc);
    cudaFree(c->d_keys);
    cudaFree(c->d_rois);
    cudaFree(c->d_wle);
    cudaFreeHost(c->h_rois);
    cudaFreeHost(c->h_wle);
    cudaFreeHost(c->h_state);
    if (c->done) cudaEventDestroy(c->done);
    if (c->copy) cudaStreamSynchronize(c->copy);
    cudaFree(c->d_raw2);
    for (int b = 0; b < 2; ++b) {
        if (c->copied[b]) cudaEventDestroy(c->copied[b]);
        if (c->consumed[b]) cudaEventDestroy(c->consumed[b]);
    }
    if (c->copy) cudaStreamDestroy(c->copy);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return QCS_OK;
}

int qcs_extract_init_ex(const qcs_loc_para *p, int max_batched_num, int capacity, qcs_extract_data **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    if (!p) return fail(QCS_ERR_ARG, "null parameter struct");
    const int R = p->ROISize;
    if (R < 5 || R > 17 || (R & 1) == 0) return fail(QCS_ERR_ROISIZE, "ROISize must be odd, 5..17");
    if (p->ImageWidth < 16 || p->ImageHigh < 16 || p->ImageWidth > 65535 || p->ImageHigh > 65535)
        return fail(QCS_ERR_ARG, "image width and height must be 16..65535");
    if (max_batched_num <= 0) max_batched_num = qcs_extract_max_batched_num(p->ImageWidth, p->ImageHigh);
    if (capacity <= 0) capacity = QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_extract_data *c = new qcs_extract_data();
    c->para = *p;
    c->W = p->ImageWidth;
    c->H0 = p->ImageHigh;
    c->R = R;
    c->whole = R * (R + 1);
    c->max_batch = max_batched_num;
    c->capacity = capacity;
    c->max_px = (long long)c->W * c->H0 * max_batched_num;
    if (c->max_px > (1ll << 31) - qcs::kChunk) {
        delete c;
        return fail(QCS_ERR_CAPACITY, "frames per batch x frame size above 2^31 pixels");
    }
    c->nchunks_max = (int)((c->max_px + qcs::kChunk - 1) / qcs::kChunk);
    qcs::filter_taps(R, p->LocType, p->MultiEmitterFitEn, c->taps.t);
    const size_t px = (size_t)c->max_px, px_pad = (size_t)c->nchunks_max * qcs::kChunk;
    cudaError_t e = cudaMalloc((void **)&c->d_raw, px * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_bg, px * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_pos, px_pad);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_chunk, (size_t)c->nchunks_max * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_state, qcs::kStNum * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_var, 4 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_var_acc, 4 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_keys, (size_t)capacity * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_rois, (size_t)capacity * c->whole * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_wle, (size_t)capacity * QCS_WLE_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_rois, (size_t)capacity * c->whole * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_wle, (size_t)capacity * QCS_WLE_PARA_NUM * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_state, qcs::kStNum * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_raw2, px * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaEventCreateWithFlags(&c->copied[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->consumed[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_state, 0, qcs::kStNum * sizeof(int), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_var_acc, 0, 4 * sizeof(unsigned long long), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        qcs_extract_deinit(c);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_extract_init", e);
    }
    memset(c->h_state, 0, qcs::kStNum * sizeof(int));
    c->last = c->stream;
    *out = c;
    return QCS_OK;
}

int qcs_extract_init(const qcs_loc_para *p, qcs_extract_data **out) { return qcs_extract_init_ex(p, 0, 0, out); }

int qcs_extract_molecules(qcs_extract_data *c, const uint16_t *img, int image_source, const qcs_loc_para *p,
                          int start_frame, int batched_num, void *stream) {
    if (!c || !p || !img) return fail(QCS_ERR_ARG, "null argument");
    if (p->ROISize != c->R) return fail(QCS_ERR_ROISIZE, "ROISize differs from the one the context was created with");
    if (batched_num < 1) return fail(QCS_ERR_ARG, "batched_num must be >= 1");
    const int W = p->ImageWidth, H0 = p->ImageHigh;
    if (W < 16 || H0 < 16 || W > 65535 || H0 > 65535) return fail(QCS_ERR_ARG, "image width and height must be 16..65535");
    const long long npx = (long long)W * H0 * batched_num;
    if (npx > c->max_px) return fail(QCS_ERR_CAPACITY, "batch larger than the context's frame buffer");
    if (start_frame < 0) return fail(QCS_ERR_ARG, "negative start frame");
    if (p->LocType < QCS_LOCTYPE_GS2D || p->LocType > QCS_LOCTYPE_DH3D) return fail(QCS_ERR_ARG, "LocType out of range");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    QCS_CUDA(order_after_last(c, s), "order after the previous call");
    const uint16_t *raw = nullptr;
    int buf = -1;  // the device frame buffer this call reads, for host frames outside a capture
    if (image_source == QCS_IMAGE_SOURCE_CPU_PINNED || image_source == QCS_IMAGE_SOURCE_CPU_NORMAL) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        QCS_CUDA(cudaStreamIsCapturing(s, &cs), "capture status");
        if (cs != cudaStreamCaptureStatusNone) {
            // under capture the copy stays on the captured stream
            QCS_CUDA(cudaMemcpyAsync(c->d_raw, img, (size_t)npx * sizeof(uint16_t), cudaMemcpyHostToDevice, s),
                     "copy frames");
            raw = c->d_raw;
        } else {
            // the copy waits only for the kernels that last read its buffer (two
            // calls ago), so it runs under the previous call's kernels
            buf = c->next_raw;
            c->next_raw ^= 1;
            uint16_t *dst = buf ? c->d_raw2 : c->d_raw;
            if (c->used[buf]) QCS_CUDA(cudaStreamWaitEvent(c->copy, c->consumed[buf], 0), "frame buffer reuse");
            QCS_CUDA(cudaMemcpyAsync(dst, img, (size_t)npx * sizeof(uint16_t), cudaMemcpyHostToDevice, c->copy),
                     "copy frames");
            QCS_CUDA(cudaEventRecord(c->copied[buf], c->copy), "frames copied");
            QCS_CUDA(cudaStreamWaitEvent(s, c->copied[buf], 0), "wait for the frames");
            raw = dst;
        }
    } else if (image_source == QCS_IMAGE_SOURCE_GPU) {
        raw = img;
    } else {
        return fail(QCS_ERR_ARG, "unknown image source");
    }
    // first batch of an accumulation opens the frame range (LDROIExtraction.cu:37-46)
    if (c->first_frame < 0 && c->end_frame < 0) {
        c->first_frame = start_frame;
        c->end_frame = start_frame + batched_num - 1;
    } else {
        c->end_frame += batched_num;
    }
    const int Hb = H0 * batched_num;
    const int nchunks = (int)((npx + qcs::kChunk - 1) / qcs::kChunk);
    QCS_CUDA(cudaMemsetAsync(c->d_chunk, 0, (size_t)nchunks * sizeof(int), s), "clear chunk counts");
    dim3 gbg((W + qcs::kBgCols - 1) / qcs::kBgCols, (Hb + qcs::kBgRows - 1) / qcs::kBgRows);
    qcs::background_kernel<<<gbg, qcs::kBgThreads, 0, s>>>(raw, c->d_bg, W, Hb);
    // central patch of the stacked batch (LDROIExtraction.cu:142-157)
    int sw = W / 2 - 5, sh = Hb / 2 - 5;
    sw = sw > 256 ? 256 : sw;
    sh = sh > 256 ? 256 : sh;
    sw = sw < 1 ? 1 : sw;
    sh = sh < 1 ? 1 : sh;
    const int S = sw < sh ? sw : sh;
    int vblocks = (S * S + qcs::kVarThreads * 4 - 1) / (qcs::kVarThreads * 4);
    vblocks = vblocks < 1 ? 1 : (vblocks > qcs::kVarBlocks ? qcs::kVarBlocks : vblocks);
    qcs::variance_kernel<<<vblocks, qcs::kVarThreads, 0, s>>>(c->d_bg, W, W / 2, Hb / 2, S, c->d_var_acc, c->d_var);
    const int multi = p->MultiEmitterFitEn;
    qcs::DetectPara dp{W, H0, Hb, c->R / 2,
                       (p->LocType == QCS_LOCTYPE_AS3D || (multi == 0 && p->LocType == QCS_LOCTYPE_GS2D)) ? 1 : 0};
    dim3 gdet((W + qcs::kDetTX - 1) / qcs::kDetTX, (Hb + qcs::kDetTY - 1) / qcs::kDetTY);
    if (p->LocType == QCS_LOCTYPE_GS2D && multi > 0)
        qcs::detect_kernel<false><<<gdet, qcs::kDetThreads, 0, s>>>(c->d_bg, c->d_pos, c->d_chunk, c->d_var, c->taps, dp);
    else
        qcs::detect_kernel<true><<<gdet, qcs::kDetThreads, 0, s>>>(c->d_bg, c->d_pos, c->d_chunk, c->d_var, c->taps, dp);
    qcs::scan_kernel<<<1, qcs::kScanThreads, 0, s>>>(c->d_chunk, nchunks, c->d_state, QCS_MAX_POINT_NUM, c->capacity);
    qcs::EmitPara ep{W, H0, c->R, multi, start_frame, (int)npx};
    qcs::compact_kernel<<<nchunks, qcs::kCompactThreads, 0, s>>>(c->d_pos, c->d_chunk, c->d_state, c->d_keys, ep);
    const int batch_max = QCS_MAX_POINT_NUM < c->capacity ? QCS_MAX_POINT_NUM : c->capacity;
    int cut_blocks = (batch_max + qcs::kCutThreads / 32 - 1) / (qcs::kCutThreads / 32);
    cut_blocks = cut_blocks > 148 * 8 ? 148 * 8 : cut_blocks;
    qcs::cut_kernel<<<cut_blocks, qcs::kCutThreads, 0, s>>>(c->d_keys, c->d_state, c->d_pos, raw, c->d_rois, ep);
    QCS_CUDA(cudaGetLastError(), "extraction kernels");
    // WLE rows of this batch's records (device range state[1], state[2])
    QCS_CUDA(qcs::launch_wle_presorted(c->d_rois, c->d_keys, c->d_state + qcs::kStBase, batch_max, c->R, p->LocType,
                                       c->d_wle, s),
             "WLE pre-pass");
    if (buf >= 0) {
        QCS_CUDA(cudaEventRecord(c->consumed[buf], s), "frame buffer read");
        c->used[buf] = true;
    }
    QCS_CUDA(mark_done(c, s), "record completion");
    return QCS_OK;
}

int qcs_extract_accumulated_roi_num(qcs_extract_data *c, int *n) {
    if (!c || !n) return fail(QCS_ERR_ARG, "null argument");
    const int st = read_state(c);
    if (st) return st;
    *n = c->h_state[qcs::kStAccum];
    return QCS_OK;
}

int qcs_extract_reset_roi_num(qcs_extract_data *c, void *stream) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->last;
    QCS_CUDA(order_after_last(c, s), "order after the previous call");
    QCS_CUDA(cudaMemsetAsync(c->d_state, 0, qcs::kStNum * sizeof(int), s), "reset counters");
    QCS_CUDA(mark_done(c, s), "record completion");
    c->h_copied = 0;
    c->first_frame = -1;
    c->end_frame = -1;
    return QCS_OK;
}

static int copy_to_host(qcs_extract_data *c) {
    const int st = read_state(c);
    if (st) return st;
    const int n = c->h_state[qcs::kStAccum];
    if (n > c->h_copied) {
        const size_t a = (size_t)c->h_copied, m = (size_t)(n - c->h_copied);
        QCS_CUDA(cudaMemcpyAsync(c->h_rois + a * c->whole, c->d_rois + a * c->whole, m * c->whole * sizeof(uint16_t),
                                 cudaMemcpyDeviceToHost, c->last),
                 "read records");
        QCS_CUDA(cudaMemcpyAsync(c->h_wle + a * QCS_WLE_PARA_NUM, c->d_wle + a * QCS_WLE_PARA_NUM,
                                 m * QCS_WLE_PARA_NUM * sizeof(float), cudaMemcpyDeviceToHost, c->last),
                 "read WLE rows");
        QCS_CUDA(cudaStreamSynchronize(c->last), "read records");
        c->h_copied = n;
    }
    return QCS_OK;
}

const uint16_t *qcs_extract_h_image_roi(qcs_extract_data *c) {
    if (!c || copy_to_host(c) != QCS_OK) return nullptr;
    return c->h_rois;
}

const float *qcs_extract_h_wle_para(qcs_extract_data *c) {
    if (!c || copy_to_host(c) != QCS_OK) return nullptr;
    return c->h_wle;
}

const uint16_t *qcs_extract_d_image_roi(const qcs_extract_data *c) { return c ? c->d_rois : nullptr; }
const float *qcs_extract_d_wle_para(const qcs_extract_data *c) { return c ? c->d_wle : nullptr; }
const int *qcs_extract_device_roi_num(const qcs_extract_data *c) { return c ? c->d_state + qcs::kStAccum : nullptr; }

int qcs_extract_frame_range(const qcs_extract_data *c, int *first_frame, int *end_frame) {
    if (!c) return fail(QCS_ERR_ARG, "null context");
    if (first_frame) *first_frame = c->first_frame;
    if (end_frame) *end_frame = c->end_frame;
    return QCS_OK;
}

int qcs_extract_dropped_num(qcs_extract_data *c, int *n) {
    if (!c || !n) return fail(QCS_ERR_ARG, "null argument");
    const int st = read_state(c);
    if (st) return st;
    *n = c->h_state[qcs::kStDropped];
    return QCS_OK;
}

}  // extern "C"
