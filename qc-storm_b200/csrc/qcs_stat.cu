// Localization statistics (FluoStatisticData_TypeDef::GetStatisticalInf,
// StatisticsInfo/statisticsInfo_top.cu:61-255; kernels statisticsInfo.cu:18-88,
// statisticsInfo_densityCalc.cu:17-103; host helpers statisticsInfo_rc.cu:18-115):
// per call, histograms of total photons, localization precision, peak SNR and
// PSF width over the rows that pass the reference's sanity window, their means,
// the activation density from the fraction of rows with no / one neighbour in
// the same frame, and time series of the means.
//
// The reference counts neighbours frame by frame: per frame, a kernel gathers
// the frame's rows and a second compares every pair, with two host
// synchronisations per frame.  Here every row of every frame in the range is
// handled in one pass: rows are sorted by (frame, row of a grid of cells as
// wide as the neighbour radius) and each row looks at the rows of its own and
// the two adjacent cell rows of its frame only, so the cost is independent of
// the number of frames and close to linear in rows.  Counts, histograms and
// bins equal the reference's (same comparisons, separate roundings as its host
// build); the four sums are reduced per block and then in block order
// (deterministic; the reference adds them with float atomics in any order).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <vector>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"

using qcs::fail;

namespace {

constexpr int kTPB = 256;
constexpr int kLen = 400;
constexpr int kLenMax = QCS_STAT_HIST_LEN;  // StatInf_Hist_DatLenMax
constexpr float kGapPhoton = 10000.0f / kLen;
constexpr float kGapPrec = 60.0f / kLen;
constexpr float kGapSNR = 50.0f / kLen;
constexpr float kGapPSF = 5.0f / kLen;
constexpr uint64_t kKeyNone = ~0ull;

__device__ __forceinline__ int bin(float v, float gap) {
    int b = (int)__fdiv_rn(v, gap);
    return min(max(b, 0), kLenMax - 1);
}

// CalcLocResultStatInf: histograms (int atomics) and per-block sums of
// [valid count, precision, SNR, width, background] in a fixed order.
__global__ void __launch_bounds__(kTPB) hist_kernel(const float *__restrict__ rows, int n, int *__restrict__ hist,
                                                    float *__restrict__ part) {
    const int i = blockIdx.x * kTPB + threadIdx.x;
    float v[5] = {0, 0, 0, 0, 0};
    if (i < n) {
        const float *q = rows + (size_t)i * 12;
        const float tp = q[QCS_POS_TPHO], bg = q[QCS_POS_BAKG];
        const float psf = __fdiv_rn(__fadd_rn(q[QCS_POS_SIGX], q[QCS_POS_SIGY]), 2.0f);
        const float snr = q[QCS_POS_PSNR];
        const float px = q[QCS_POS_CRBX], py = q[QCS_POS_CRBY];
        const float pxy = __fsqrt_rn(__fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py)));
        if ((tp > 30.0f) && (bg > 2.0f) && (snr >= 3.0f) && (psf >= 0.01f) && (pxy > 0.01f) && (pxy < 55.0f)) {
            atomicAdd(hist + bin(tp, kGapPhoton), 1);
            atomicAdd(hist + kLenMax + bin(pxy, kGapPrec), 1);
            atomicAdd(hist + 2 * kLenMax + bin(snr, kGapSNR), 1);
            atomicAdd(hist + 3 * kLenMax + bin(psf, kGapPSF), 1);
            v[0] = 1.0f;
            v[1] = pxy;
            v[2] = snr;
            v[3] = psf;
            v[4] = bg;
        }
    }
    __shared__ float ws[kTPB / 32][5];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0) ws[warp][k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        float s = 0;
        for (int w = 0; w < kTPB / 32; ++w) s += ws[w][threadIdx.x];
        part[(size_t)blockIdx.x * 5 + threadIdx.x] = s;
    }
}

// block partial sums -> sums[5], in block order
__global__ void sum_kernel(const float *__restrict__ part, int nblocks, float *__restrict__ sums) {
    if (threadIdx.x >= 5) return;
    float s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * 5 + threadIdx.x];
    sums[threadIdx.x] = s;
}

// GetFirstFrame / GetLastFrame (bfgsMLE_Loc_top/bfgs_top.cu:345-381): index of
// the first row with a nonzero frame, and of the last such row after row 0.
__global__ void frame_ends_kernel(const float *__restrict__ rows, int n, int *__restrict__ ends) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if ((int)rows[(size_t)i * 12 + QCS_POS_FRME] != 0) {
        atomicMin(ends, i);
        if (i > 0) atomicMax(ends + 1, i);
    }
}

__device__ __forceinline__ uint64_t cell_key(int frame, int cell) {
    return ((uint64_t)(uint32_t)frame << 32) | (uint64_t)((uint32_t)cell ^ 0x80000000u);
}

// FillerMoleculesInCurFrame's selection for every frame of [fs, fe] at once:
// rows at least 5 px inside the image get a (frame, cell row) key, others none.
__global__ void density_keys_kernel(const float *__restrict__ rows, int n, int fs, int fe, int W, int H, float rad,
                                    uint64_t *__restrict__ keys, int *__restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *q = rows + (size_t)i * 12;
    const int xp = (int)q[QCS_POS_XPOS], yp = (int)q[QCS_POS_YPOS], f = (int)q[QCS_POS_FRME];
    const bool sel = xp >= 5 && xp < W - 5 && yp >= 5 && yp < H - 5 && f >= fs && f <= fe;
    keys[i] = sel ? cell_key(f, (int)floorf(__fdiv_rn(q[QCS_POS_YPOS], rad))) : kKeyNone;
    vals[i] = i;
}

__device__ __forceinline__ int lower_bound(const uint64_t *__restrict__ a, int n, uint64_t k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// CalcOverlapFluoNum: rows with no / one other selected row of their frame
// within the radius (squared distance with separate roundings, <= rad^2).
__global__ void density_count_kernel(const float *__restrict__ rows, int n, const uint64_t *__restrict__ skeys,
                                     const int *__restrict__ svals, float rad, int *__restrict__ cnt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t key = skeys[j];
    if (key == kKeyNone) return;
    const int me = svals[j];
    const int frame = (int)(key >> 32);
    const int cell = (int)((uint32_t)key ^ 0x80000000u);
    const float cx = rows[(size_t)me * 12 + QCS_POS_XPOS], cy = rows[(size_t)me * 12 + QCS_POS_YPOS];
    const float th2 = __fmul_rn(rad, rad);
    int nb = 0;
    const uint64_t khi = cell_key(frame, cell + 1);
    for (int k = lower_bound(skeys, n, cell_key(frame, cell - 1)); k < n && skeys[k] <= khi && nb < 2; ++k) {
        const int o = svals[k];
        if (o == me) continue;
        const float dx = __fsub_rn(rows[(size_t)o * 12 + QCS_POS_XPOS], cx);
        const float dy = __fsub_rn(rows[(size_t)o * 12 + QCS_POS_YPOS], cy);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), 0.0f);
        nb += (d2 <= th2);
    }
    if (nb == 0) atomicAdd(cnt, 1);
    if (nb == 1) atomicAdd(cnt + 1, 1);
    atomicAdd(cnt + 2, 1);
}

inline int blocks(int n) { return (n + kTPB - 1) / kTPB; }

// host helpers of statisticsInfo_rc.cu (float arithmetic, separate roundings)
float activation_density(float r0, float r1, float radius_um) {
    const float PI = 3.14159f;
    if (r0 <= 0.001f) r0 = 0.001f;
    if (r1 <= 0.001f) r1 = 0.001f;
    if (r0 > 1) r0 = 1;
    if (r1 > 1) r1 = 1;
    const float ratio0 = logf(r0);
    const float ratio1 = logf(r1 / PI / radius_um / radius_um);
    const float density0 = -ratio0 / PI / radius_um / radius_um;
    const float density1 = -ratio1 / PI / radius_um / radius_um;
    return r0 * density0 + (1.0f - r0) * density1;
}

float hist_mean(const int *h, int len, float pct) {
    int mx = h[0];
    for (int i = 0; i < len; ++i) mx = h[i] > mx ? h[i] : mx;
    pct = pct * mx;
    float ws = 0, os = 0;
    for (int i = 0; i < len; ++i) {
        const float v = (float)h[i];
        if (v >= pct) {
            ws += v * (i + 0.5f);
            os += v;
        }
    }
    if (os == 0) os = 1;
    return ws / os;
}

float series_mean(const std::vector<float> &v) {
    float mean = 0;
    if (v.size() > 2) {
        float tot = 0;
        int k = 0;
        for (size_t i = 1; i < v.size() - 1; ++i) {
            tot += v[i];
            k++;
        }
        if (k <= 0) k = 1;
        mean = tot / k;
    }
    return mean;
}

// The on-time curve fit of UpdateOntimeRatio (statisticsInfo_top.cu:30-35):
// least squares of y = a * exp(b * i) over the on-time ratios by the reference's
// BFGSOptimizer<float, 2, 4, 11> with ExpFit_PreFitting / ExpFit_TargerF (BFGS
// for curve fitting/BFGSOptimizer.h:120-533, CurveFitting.cpp:27-58).  The
// parameters are searched divided by max(|start|, 1); each of the 4 steps
// normalises the direction to a mean |component| of 1 and brackets the step
// length in [1e-5, 1] (the lower end scored at 1e-4, as the reference does),
// halving the bracket 11 times towards the lower loss; gradients are central
// differences of 0.002 in the scaled coordinates; the inverse Hessian takes the
// BFGS update (I - s y'/y's) H (I - y s'/y's) + s s'/y's.  A 10-point host
// problem: every float operation is rounded separately in the reference's order
// (host build, no contraction), so the result equals the reference's.
struct DecayFit {
    const float *y;
    int n;
    float scale[2];

    float loss(const float *u) const {
        const float a = u[0] * scale[0], b = u[1] * scale[1];
        float e = 0;
        for (int i = 0; i < n; ++i) {
            const float r = a * expf(b * (float)i) - y[i];
            e += r * r;
        }
        return e;
    }
    float loss_along(const float *p, const float *d, float t) const {
        const float u[2] = {d[0] * t + p[0], d[1] * t + p[1]};
        return loss(u);
    }
    void gradient(const float *p, float *g) const {
        float u[2] = {p[0], p[1]};
        for (int k = 0; k < 2; ++k) {
            u[k] = u[k] - 0.002f;
            const float below = loss(u);
            u[k] = u[k] + 0.004f;
            const float above = loss(u);
            g[k] = (above - below) * 250.0f;
            u[k] = u[k] - 0.002f;  // not exactly p[k] again: the next component sees it
        }
    }
};

void fit_decay(const float *y, int n, float *a, float *b) {
    DecayFit f{y, n, {1.0f, 1.0f}};
    float p[2];
    p[0] = y[0];
    p[1] = ((double)y[0] > 0.01 && (double)y[1] > 0.01) ? logf(y[1] / y[0]) : 0.0f;
    for (int k = 0; k < 2; ++k) {
        f.scale[k] = std::fabs(p[k]) > 1.0f ? std::fabs(p[k]) : 1.0f;
        p[k] = p[k] / f.scale[k];
    }
    float g[2], d[2];
    float h[2][2] = {{1.0f, 0.0f}, {0.0f, 1.0f}};
    f.gradient(p, g);
    d[0] = -g[0];
    d[1] = -g[1];
    constexpr int kSteps = 4, kHalvings = 11;
    for (int step = 0; step < kSteps; ++step) {
        float mean_abs = 0;
        mean_abs += std::fabs(d[0]);
        mean_abs += std::fabs(d[1]);
        mean_abs = mean_abs / 2;
        d[0] = d[0] / mean_abs;
        d[1] = d[1] / mean_abs;
        float lo = 0.00001f, hi = 1.0f;
        float f_lo = f.loss_along(p, d, 0.0001f), f_hi = f.loss_along(p, d, 1.0f);
        for (int k = 0; k < kHalvings; ++k) {
            const float mid = (lo + hi) * 0.5f;
            const bool last = k == kHalvings - 1;
            if (f_lo < f_hi) {
                hi = mid;
                if (!last) f_hi = f.loss_along(p, d, hi);
            } else {
                lo = mid;
                if (!last) f_lo = f.loss_along(p, d, lo);
            }
        }
        const float t = (lo + hi) * 0.5f;
        const float s[2] = {d[0] * t, d[1] * t};
        p[0] = p[0] + s[0];
        p[1] = p[1] + s[1];
        if (step == kSteps - 1) break;
        const float g0[2] = {g[0], g[1]};
        f.gradient(p, g);
        const float yk[2] = {g[0] - g0[0], g[1] - g0[1]};
        float sy = 0;
        sy += s[0] * yk[0];
        sy += s[1] * yk[1];
        const float inv = 1.0f / sy;
        const float yi[2] = {yk[0] * inv, yk[1] * inv}, si[2] = {s[0] * inv, s[1] * inv};
        float left[2][2], ss[2][2], lh[2][2];
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                left[r][c] = (r == c ? 1.0f : 0.0f) - s[r] * yi[c];  // I - s y' / y's
                ss[r][c] = s[r] * si[c];
            }
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                float acc = 0;
                for (int k = 0; k < 2; ++k) acc += left[r][k] * h[k][c];
                lh[r][c] = acc;
            }
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                float acc = 0;
                for (int k = 0; k < 2; ++k) acc += lh[r][k] * left[c][k];  // right factor: the transpose
                h[r][c] = acc + ss[r][c];
            }
        for (int r = 0; r < 2; ++r) {
            float acc = 0;
            for (int c = 0; c < 2; ++c) acc -= h[r][c] * g[c];
            d[r] = acc;
        }
    }
    *a = p[0] * f.scale[0];
    *b = p[1] * f.scale[1];
}

}  // namespace

struct qcs_stat {
    int capacity = 0;
    float *d_rows = nullptr;  // capacity x 12 (host rows are copied here)
    int *d_hist = nullptr;    // 4 x 1600
    float *d_part = nullptr;  // per-block sums
    float *d_sums = nullptr;  // 5
    int *d_ints = nullptr;    // frame ends (2), neighbour counts (3)
    uint64_t *d_keys = nullptr, *d_skeys = nullptr;
    int *d_vals = nullptr, *d_svals = nullptr;
    void *d_sort = nullptr;
    size_t sort_bytes = 0;
    int *h_hist = nullptr;    // pinned, 4 x 1600: the last call's histograms
    float *h_sums = nullptr;  // pinned, 5
    int *h_ints = nullptr;    // pinned, 5
    float means[QCS_STAT_MEANS] = {0};
    float mean_ontime = 0;
    float ontime[QCS_ONTIME_BINS] = {0};
    std::vector<float> series[QCS_STAT_SERIES];
    cudaStream_t stream = nullptr;
};

namespace {

int stat_run(qcs_stat *st, const float *d_rows, int n, const qcs_loc_para *p, cudaStream_t s) {
    // CalcLocResultStatInf, then the histograms to the host and cleared
    const int nb = blocks(n);
    hist_kernel<<<nb, kTPB, 0, s>>>(d_rows, n, st->d_hist, st->d_part);
    sum_kernel<<<1, 32, 0, s>>>(st->d_part, nb, st->d_sums);
    const int init[2] = {0x7fffffff, -1};
    QCS_CUDA(cudaMemcpyAsync(st->d_ints, init, sizeof(init), cudaMemcpyHostToDevice, s), "frame ends");
    frame_ends_kernel<<<blocks(n), kTPB, 0, s>>>(d_rows, n, st->d_ints);
    QCS_CUDA(cudaGetLastError(), "statistics kernels");
    QCS_CUDA(cudaMemcpyAsync(st->h_hist, st->d_hist, 4 * kLenMax * sizeof(int), cudaMemcpyDeviceToHost, s), "histograms");
    QCS_CUDA(cudaMemcpyAsync(st->h_sums, st->d_sums, 5 * sizeof(float), cudaMemcpyDeviceToHost, s), "sums");
    QCS_CUDA(cudaMemcpyAsync(st->h_ints, st->d_ints, 2 * sizeof(int), cudaMemcpyDeviceToHost, s), "frame ends");
    QCS_CUDA(cudaMemsetAsync(st->d_hist, 0, 4 * kLenMax * sizeof(int), s), "clear histograms");
    QCS_CUDA(cudaStreamSynchronize(s), "statistics");
    float vnum = st->h_sums[0];
    if (vnum <= 0) vnum = 1;
    // GetFirstFrame / GetLastFrame from the row indices found on the device
    float fr[2] = {0, 0};
    if (st->h_ints[0] < n)
        QCS_CUDA(cudaMemcpy(&fr[0], d_rows + (size_t)st->h_ints[0] * 12 + QCS_POS_FRME, sizeof(float),
                            cudaMemcpyDeviceToHost),
                 "first frame");
    if (st->h_ints[1] > 0)
        QCS_CUDA(cudaMemcpy(&fr[1], d_rows + (size_t)st->h_ints[1] * 12 + QCS_POS_FRME, sizeof(float),
                            cudaMemcpyDeviceToHost),
                 "last frame");
    const int sf = (int)fr[0], ef = (int)fr[1];
    // CalcLocalizationDensity2D
    const float rad = (p->LocType == QCS_LOCTYPE_GS2D) ? 10.0f : 20.0f;
    const float rad_um = rad * p->PixelSize / 1000;
    int fs = sf, fe = ef;
    if (ef - sf + 1 > 3) {
        fs = sf + 1;
        fe = ef - 1;
    }
    int total = 0, c0 = 0, c1 = 0;
    if (fs <= fe) {
        density_keys_kernel<<<blocks(n), kTPB, 0, s>>>(d_rows, n, fs, fe, p->ImageWidth, p->ImageHigh, rad, st->d_keys,
                                                       st->d_vals);
        size_t tb = st->sort_bytes;
        QCS_CUDA(cub::DeviceRadixSort::SortPairs(st->d_sort, tb, st->d_keys, st->d_skeys, st->d_vals, st->d_svals, n, 0,
                                                 64, s),
                 "sort rows by frame and cell");
        QCS_CUDA(cudaMemsetAsync(st->d_ints + 2, 0, 3 * sizeof(int), s), "neighbour counts");
        density_count_kernel<<<blocks(n), kTPB, 0, s>>>(d_rows, n, st->d_skeys, st->d_svals, rad, st->d_ints + 2);
        QCS_CUDA(cudaGetLastError(), "density kernels");
        QCS_CUDA(cudaMemcpyAsync(st->h_ints + 2, st->d_ints + 2, 3 * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "neighbour counts");
        QCS_CUDA(cudaStreamSynchronize(s), "density");
        c0 = st->h_ints[2];
        c1 = st->h_ints[3];
        total = st->h_ints[4];
    }
    float *m = st->means;
    if (total > 50) {
        const float r0 = (float)c0 / total, r1 = (float)c1 / total;
        float d = activation_density(r0, r1, rad_um);
        if (p->MultiEmitterFitEn)
            d = d * d * 0.5098f + d * 0.6364f;
        else
            d = d * d * 0.8082f + d * 0.519f;
        m[QCS_STAT_MEAN_DENSITY] = d;
    }
    // UpdateStatDat
    m[QCS_STAT_MEAN_PHOTON] = kGapPhoton * hist_mean(st->h_hist, kLenMax, 0.1f);
    m[QCS_STAT_MEAN_PREC] = st->h_sums[1] / vnum;
    m[QCS_STAT_MEAN_SNR] = st->h_sums[2] / vnum;
    m[QCS_STAT_MEAN_BKG] = st->h_sums[4] / vnum;
    m[QCS_STAT_MEAN_PSF] = st->h_sums[3] / vnum;
    m[QCS_STAT_MEAN_PSF_CTL] = m[QCS_STAT_MEAN_PSF] * (-m[QCS_STAT_MEAN_SNR]);
    st->series[QCS_STAT_SERIES_PHOTON].push_back(m[QCS_STAT_MEAN_PHOTON]);
    st->series[QCS_STAT_SERIES_PREC].push_back(m[QCS_STAT_MEAN_PREC]);
    st->series[QCS_STAT_SERIES_SNR].push_back(m[QCS_STAT_MEAN_SNR]);
    st->series[QCS_STAT_SERIES_BKG].push_back(m[QCS_STAT_MEAN_BKG]);
    st->series[QCS_STAT_SERIES_PSF].push_back(m[QCS_STAT_MEAN_PSF]);
    st->series[QCS_STAT_SERIES_PSF_CTL].push_back(m[QCS_STAT_MEAN_PSF_CTL]);
    st->series[QCS_STAT_SERIES_DENSITY].push_back(m[QCS_STAT_MEAN_DENSITY]);
    m[QCS_STAT_TV_PHOTON] = series_mean(st->series[QCS_STAT_SERIES_PHOTON]);
    m[QCS_STAT_TV_PREC] = series_mean(st->series[QCS_STAT_SERIES_PREC]);
    m[QCS_STAT_TV_SNR] = series_mean(st->series[QCS_STAT_SERIES_SNR]);
    return QCS_OK;
}

}  // namespace

extern "C" {

int qcs_stat_deinit(qcs_stat *st) {
    if (!st) return QCS_OK;
    if (st->stream) cudaStreamSynchronize(st->stream);
    cudaFree(st->d_rows);
    cudaFree(st->d_hist);
    cudaFree(st->d_part);
    cudaFree(st->d_keys);
    cudaFree(st->d_sort);
    cudaFreeHost(st->h_hist);
    if (st->stream) cudaStreamDestroy(st->stream);
    delete st;
    return QCS_OK;
}

int qcs_stat_init(int capacity, qcs_stat **out) {
    if (!out) return fail(QCS_ERR_ARG, "null output handle");
    *out = nullptr;
    if (capacity <= 0) capacity = 2 * QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_stat *st = new qcs_stat();
    st->capacity = capacity;
    const size_t cap = (size_t)capacity;
    const size_t nb = (size_t)blocks(capacity);
    cudaError_t e = cudaMalloc((void **)&st->d_rows, cap * 12 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&st->d_hist, 4 * kLenMax * sizeof(int) + 16 * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&st->d_part, (nb * 5 + 8) * sizeof(float));
    // keys, sorted keys, values, sorted values, each from a 256-byte boundary
    const size_t bk = (cap * sizeof(uint64_t) + 255) / 256 * 256, bv = (cap * sizeof(int) + 255) / 256 * 256;
    if (e == cudaSuccess) e = cudaMalloc((void **)&st->d_keys, 2 * bk + 2 * bv);
    if (e == cudaSuccess) {
        st->d_ints = st->d_hist + 4 * kLenMax;
        st->d_sums = st->d_part + nb * 5;
        char *b = reinterpret_cast<char *>(st->d_keys);
        st->d_skeys = reinterpret_cast<uint64_t *>(b + bk);
        st->d_vals = reinterpret_cast<int *>(b + 2 * bk);
        st->d_svals = reinterpret_cast<int *>(b + 2 * bk + bv);
        e = cub::DeviceRadixSort::SortPairs(nullptr, st->sort_bytes, st->d_keys, st->d_skeys, st->d_vals, st->d_svals,
                                            capacity, 0, 64);
    }
    if (e == cudaSuccess) e = cudaMalloc(&st->d_sort, st->sort_bytes > 0 ? st->sort_bytes : 1);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&st->h_hist, (4 * kLenMax + 16) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(st->d_hist, 0, 4 * kLenMax * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        qcs_stat_deinit(st);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_stat_init", e);
    }
    memset(st->h_hist, 0, (4 * kLenMax + 16) * sizeof(int));
    st->h_ints = st->h_hist + 4 * kLenMax;
    st->h_sums = reinterpret_cast<float *>(st->h_ints + 8);
    *out = st;
    return QCS_OK;
}

int qcs_stat_reset_all(qcs_stat *st) {
    if (!st) return fail(QCS_ERR_ARG, "null statistics");
    QCS_CUDA(cudaMemsetAsync(st->d_hist, 0, 4 * kLenMax * sizeof(int), st->stream), "clear histograms");
    QCS_CUDA(cudaStreamSynchronize(st->stream), "clear histograms");
    for (auto &v : st->series) v.clear();
    for (float &m : st->means) m = 0;
    return QCS_OK;
}

int qcs_stat_get_statistical_inf(qcs_stat *st, const float *h_rows, int n, const qcs_loc_para *p, void *stream) {
    if (!st || !p) return fail(QCS_ERR_ARG, "null argument");
    if (n > st->capacity) return fail(QCS_ERR_CAPACITY, "more rows than the statistics' capacity");
    if (n <= 0) return QCS_OK;
    if (!h_rows) return fail(QCS_ERR_ARG, "null rows");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : st->stream;
    QCS_CUDA(cudaMemcpyAsync(st->d_rows, h_rows, (size_t)n * 12 * sizeof(float), cudaMemcpyHostToDevice, s),
             "copy rows");
    return stat_run(st, st->d_rows, n, p, s);
}

int qcs_stat_get_statistical_inf_device(qcs_stat *st, const float *d_rows, int n, const qcs_loc_para *p,
                                        void *stream) {
    if (!st || !p) return fail(QCS_ERR_ARG, "null argument");
    if (n > st->capacity) return fail(QCS_ERR_CAPACITY, "more rows than the statistics' capacity");
    if (n <= 0) return QCS_OK;
    if (!d_rows) return fail(QCS_ERR_ARG, "null rows");
    return stat_run(st, d_rows, n, p, stream ? static_cast<cudaStream_t>(stream) : st->stream);
}

int qcs_stat_histograms(const qcs_stat *st, int *out) {
    if (!st || !out) return fail(QCS_ERR_ARG, "null argument");
    memcpy(out, st->h_hist, 4 * kLenMax * sizeof(int));
    return QCS_OK;
}

int qcs_stat_means(const qcs_stat *st, float *out) {
    if (!st || !out) return fail(QCS_ERR_ARG, "null argument");
    memcpy(out, st->means, sizeof(st->means));
    return QCS_OK;
}

int qcs_stat_update_ontime_ratio(qcs_stat *st, const float *ratios) {
    if (!st || !ratios) return fail(QCS_ERR_ARG, "null argument");
    float *r = st->ontime;
    memcpy(r, ratios, sizeof(st->ontime));
    float a = 0, b = 0;
    fit_decay(r, QCS_ONTIME_BINS, &a, &b);
    const float k1 = -logf(1 - a), k2 = -b;
    st->mean_ontime = 2 / (k1 + k2);
    for (int i = 4; i < QCS_ONTIME_BINS; ++i) r[3] += r[i];
    for (int i = 0; i < 4; ++i) {
        r[i] = fminf(fmaxf(r[i], 0.0f), 1.0f);
        st->series[QCS_STAT_SERIES_ONTIME_F1 + i].push_back(r[i]);
    }
    return QCS_OK;
}

int qcs_stat_ontime(const qcs_stat *st, float *mean_ontime, float *ratios) {
    if (!st) return fail(QCS_ERR_ARG, "null statistics");
    if (mean_ontime) *mean_ontime = st->mean_ontime;
    if (ratios) memcpy(ratios, st->ontime, sizeof(st->ontime));
    return QCS_OK;
}

int qcs_stat_series(const qcs_stat *st, int which, float *out, int max_n) {
    if (!st || which < 0 || which >= QCS_STAT_SERIES) return fail(QCS_ERR_ARG, "bad series");
    const std::vector<float> &v = st->series[which];
    const int n = (int)v.size();
    for (int i = 0; out && i < n && i < max_n; ++i) out[i] = v[(size_t)i];
    return n;
}

}  // extern "C"
