// Super-resolution render: every localization row adds a 7x7 Gaussian, its
// width the row's CRLB, into a float image SRImageWidth x SRImageHigh (and,
// for 3D types, z times the same weights into a colour map), and updates the
// running display maximum and histogram.  ImageRenderData_TypeDef's device
// part (ImgRender/ImageRender_top.cu:29-60, 223-292):
//   FluoRenderWithPrec_2D   ImgRender/ImageRender_2d.cu:25-155
//   FluoRenderWithPrec_3D   ImgRender/ImageRender_3d.cu:29-148
//   ResetFillMaxVal         ImgRender/ImageRender_top.cu:68-102
// The reference runs one thread per row with 49 serial atomics and copies the
// rows from the host first.  Here one warp renders a row (its lanes add the
// 49 pixels as fire-and-forget reductions), the display histogram collects in
// shared memory per block, the running maximum is raised only when a centre
// exceeds it, rows can come straight from a localization on the device with
// their count in device memory (no host round trip), and the periodic
// histogram rescale runs on the device instead of through the host.  The
// float sums, the maximum and the histogram depend on the order of the
// atomic adds, as in the reference.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"
#include "qcs_error.h"

using qcs::fail;

namespace {

constexpr int kW = 7, kHalf = 3, kPix = kW * kW;
constexpr long long kRescaleAfter = 20ll * QCS_MAX_POINT_NUM;  // rows between histogram rescales

struct RenderArgs {
    int width, high, mode;
    float zoom, pixel, snr_th, zth, fixed_prec;
};

// FluoRenderTop's bookkeeping before a batch: after every 20 x MaxPointNum
// rows the histogram is rescaled to 200 / hist[0] (ResetFillMaxVal(1)).
__global__ void render_prepare_kernel(const int *__restrict__ d_n, int n, long long *__restrict__ count,
                                      int *__restrict__ hist) {
    const int rows = d_n ? min(max(*d_n, 0), n) : n;
    if (rows <= 0) return;
    long long c = *count + rows;
    if (c > kRescaleAfter) {
        c = 0;
        int nd = hist[0];
        if (nd <= 1) nd = 1;
        for (int i = 0; i < QCS_RENDER_HIST_LEN; ++i) hist[i] = hist[i] * 200 / nd;
    }
    *count = c;
}

// Device-scope relaxed load: the value at L2, never a stale L1 copy.
__device__ __forceinline__ int load_relaxed_gpu(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <bool IS2D>
__global__ void __launch_bounds__(256) render_kernel(const float *__restrict__ rows, const int *__restrict__ d_n,
                                                     int n, RenderArgs a, float *__restrict__ img,
                                                     float *__restrict__ cmap, int *__restrict__ maxv,
                                                     int *__restrict__ hist) {
    __shared__ int s_hist[QCS_RENDER_HIST_LEN];
    for (int k = threadIdx.x; k < QCS_RENDER_HIST_LEN; k += blockDim.x) s_hist[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int count = d_n ? min(max(*d_n, 0), n) : n;
    for (int i = warp; i < count; i += nwarps) {
        const float *r = rows + (size_t)i * QCS_OUT_PARA_NUM;
        float PeakPhoton = __ldg(r + QCS_POS_PPHO);
        const float X = __fmul_rn(__ldg(r + QCS_POS_XPOS), a.zoom);
        const float Y = __fmul_rn(__ldg(r + QCS_POS_YPOS), a.zoom);
        const float Z = __ldg(r + QCS_POS_ZPOS);
        float CurSNR = __ldg(r + QCS_POS_PSNR);
        float LocPrec = IS2D ? __ldg(r + QCS_POS_CRBX)
                             : __fdiv_rn(__fadd_rn(__ldg(r + QCS_POS_CRBX), __ldg(r + QCS_POS_CRBY)), 2.0f);
        CurSNR = isnan(LocPrec) ? 0.0f : CurSNR;
        PeakPhoton = isnan(LocPrec) ? 0.0f : PeakPhoton;
        PeakPhoton = (LocPrec <= 0.0f) ? 0.0f : PeakPhoton;
        bool valid = (CurSNR >= a.snr_th) && (PeakPhoton > 1.0f) && (X > (float)kW) &&
                     (X < (float)(a.width - 1 - kW)) && (Y > (float)kW) && (Y < (float)(a.high - 1 - kW));
        if (!IS2D) valid = valid && (fabsf(Z) < a.zth);
        if (!valid) continue;  // uniform over the warp
        if (a.mode == QCS_RENDER_1PHOTON_CRLB || a.mode == QCS_RENDER_1PHOTON_FIXED) PeakPhoton = 1.0f;
        if (a.mode == QCS_RENDER_1PHOTON_FIXED) LocPrec = a.fixed_prec;
        if (IS2D && LocPrec > 30.0f) {  // coarser than 30 nm: not rendered
            LocPrec = 30.0f;
            PeakPhoton = 0.0f;
        }
        const float px = __fdiv_rn(a.pixel, a.zoom);
        LocPrec = fmaxf(LocPrec, __fdiv_rn(px, 2.0f));
        const float sigma = __fdiv_rn(LocPrec, px);
        const float S = __fdiv_rn(-0.5f, __fmul_rn(sigma, sigma));
        const int ix = (int)X, iy = (int)Y;
        const float fx = __fadd_rn(__fsub_rn(X, (float)ix), (float)kHalf);
        const float fy = __fadd_rn(__fsub_rn(Y, (float)iy), (float)kHalf);
        if (IS2D && a.mode == QCS_RENDER_FITTED_PHOTON_1PIXEL) {
            if (lane == 0) atomicAdd(&img[(size_t)a.width * iy + ix], PeakPhoton);
        } else {
            for (int k = lane; k < kPix; k += 32) {
                const int rc = k / kW, cc = k - rc * kW;
                const float dx = __fsub_rn((float)cc, fx), dy = __fsub_rn((float)rc, fy);
                const float v = __expf(__fmul_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), S));
                const size_t off = (size_t)a.width * (iy - kHalf + rc) + (ix - kHalf + cc);
                const float w = __fmul_rn(PeakPhoton, v);
                atomicAdd(&img[off], w);
                if (!IS2D) atomicAdd(&cmap[off], __fmul_rn(__fmul_rn(Z, PeakPhoton), v));
            }
        }
        __syncwarp();
        if (lane == 0) {
            // the centre after this row's adds (atomic read: the value at L2)
            const float centre = atomicAdd(&img[(size_t)a.width * iy + ix], 0.0f);
            const int c = (int)centre;
            // the running maximum: read first, raised atomically only when
            // this centre exceeds it (every row raising one shared word
            // serialises at L2)
            int m = load_relaxed_gpu(maxv);
            if (c > m) {
                const int old = atomicMax(maxv, c);
                m = old > c ? old : c;
            }
            if (m != 0) {
                const int pos = c * QCS_RENDER_HIST_LEN / m;
                if (pos >= 0 && pos < QCS_RENDER_HIST_LEN) atomicAdd(&s_hist[pos], 1);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < QCS_RENDER_HIST_LEN; k += blockDim.x)
        if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

}  // namespace

struct qcs_render_data {
    int width = 0, high = 0, capacity = 0;
    bool is2d = true;
    float *d_img = nullptr, *d_cmap = nullptr, *d_rows = nullptr;
    int *d_max = nullptr, *d_hist = nullptr;
    long long *d_count = nullptr;
    cudaStream_t stream = nullptr;
};

static int render_launch(qcs_render_data *r, const float *d_rows, const int *d_n, int max_n, const qcs_loc_para *p,
                         int mode, float fixed_prec, cudaStream_t s) {
    if (p->SRImageWidth != r->width || p->SRImageHigh != r->high)
        return fail(QCS_ERR_ARG, "SRImageWidth / SRImageHigh differ from the render context's");
    if ((p->LocType == QCS_LOCTYPE_GS2D) != r->is2d)
        return fail(QCS_ERR_ARG, "2D / 3D localization type differs from the render context's");
    if (mode < QCS_RENDER_FITTED_PHOTON_CRLB || mode > QCS_RENDER_FITTED_PHOTON_1PIXEL)
        return fail(QCS_ERR_ARG, "unknown rendering mode");
    if (max_n <= 0) return QCS_OK;
    RenderArgs a;
    a.width = r->width;
    a.high = r->high;
    a.mode = mode;
    a.zoom = p->PixelZoom;
    a.pixel = p->PixelSize;
    a.snr_th = p->SNR_th;
    a.zth = 5.0f * fmaxf(fabsf(p->MinZDepth), fabsf(p->MaxZDepth));
    a.fixed_prec = fixed_prec;
    render_prepare_kernel<<<1, 1, 0, s>>>(d_n, max_n, r->d_count, r->d_hist);
    const long long warps_needed = max_n;
    long long blocks = (warps_needed + 7) / 8;  // 8 warps per block
    if (blocks > 148 * 16) blocks = 148 * 16;   // a few rows per warp: latency hidden, block histogram shared
    if (r->is2d)
        render_kernel<true><<<(int)blocks, 256, 0, s>>>(d_rows, d_n, max_n, a, r->d_img, nullptr, r->d_max, r->d_hist);
    else
        render_kernel<false><<<(int)blocks, 256, 0, s>>>(d_rows, d_n, max_n, a, r->d_img, r->d_cmap, r->d_max,
                                                         r->d_hist);
    QCS_CUDA(cudaGetLastError(), "render kernels");
    return QCS_OK;
}

extern "C" {

int qcs_render_deinit(qcs_render_data *r) {
    if (!r) return QCS_OK;
    if (r->stream) cudaStreamSynchronize(r->stream);
    cudaFree(r->d_img);
    cudaFree(r->d_cmap);
    cudaFree(r->d_rows);
    cudaFree(r->d_max);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return QCS_OK;
}

int qcs_render_init(const qcs_loc_para *p, int capacity, qcs_render_data **out) {
    if (!out || !p) return fail(QCS_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->SRImageWidth <= 0 || p->SRImageHigh <= 0) return fail(QCS_ERR_ARG, "SRImageWidth / SRImageHigh not set");
    if (capacity <= 0) capacity = QCS_MAX_POINT_NUM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QCS_ERR_CUDA, "no CUDA device: qcstorm_b200 has no CPU fallback");
    qcs_render_data *r = new qcs_render_data();
    r->width = p->SRImageWidth;
    r->high = p->SRImageHigh;
    r->capacity = capacity;
    r->is2d = p->LocType == QCS_LOCTYPE_GS2D;
    const size_t px = (size_t)r->width * r->high;
    cudaError_t e = cudaMalloc((void **)&r->d_img, px * sizeof(float));
    if (e == cudaSuccess && !r->is2d) e = cudaMalloc((void **)&r->d_cmap, px * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&r->d_rows, (size_t)capacity * QCS_OUT_PARA_NUM * sizeof(float));
    // maximum, histogram and row count in one block
    if (e == cudaSuccess) e = cudaMalloc((void **)&r->d_max, 256 + QCS_RENDER_HIST_LEN * sizeof(int) + 256);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        qcs_render_deinit(r);
        return fail(e == cudaErrorMemoryAllocation ? QCS_ERR_NOMEM : QCS_ERR_CUDA, "qcs_render_init", e);
    }
    r->d_hist = reinterpret_cast<int *>(reinterpret_cast<char *>(r->d_max) + 256);
    r->d_count = reinterpret_cast<long long *>(reinterpret_cast<char *>(r->d_hist) + QCS_RENDER_HIST_LEN * sizeof(int));
    int st = qcs_render_reset(r, nullptr);
    if (!st) st = qcs_render_reset_max(r, nullptr);
    if (st) {
        qcs_render_deinit(r);
        return st;
    }
    QCS_CUDA(cudaStreamSynchronize(r->stream), "qcs_render_init");
    *out = r;
    return QCS_OK;
}

int qcs_render_reset(qcs_render_data *r, void *stream) {
    if (!r) return fail(QCS_ERR_ARG, "null render context");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    const size_t px = (size_t)r->width * r->high;
    QCS_CUDA(cudaMemsetAsync(r->d_img, 0, px * sizeof(float), s), "reset image");
    if (r->d_cmap) QCS_CUDA(cudaMemsetAsync(r->d_cmap, 0, px * sizeof(float), s), "reset colour map");
    return QCS_OK;
}

int qcs_render_reset_max(qcs_render_data *r, void *stream) {
    if (!r) return fail(QCS_ERR_ARG, "null render context");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    QCS_CUDA(cudaMemsetAsync(r->d_max, 0, 256 + QCS_RENDER_HIST_LEN * sizeof(int) + 256, s), "reset display state");
    return QCS_OK;
}

int qcs_render_rows(qcs_render_data *r, const float *h_rows, const qcs_loc_para *p, int mode, float fixed_prec, int n,
                    void *stream) {
    if (!r || !p) return fail(QCS_ERR_ARG, "null argument");
    if (n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (n > r->capacity) return fail(QCS_ERR_CAPACITY, "row count above the render context's capacity");
    if (n == 0) return QCS_OK;
    if (!h_rows) return fail(QCS_ERR_ARG, "null rows");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    QCS_CUDA(cudaMemcpyAsync(r->d_rows, h_rows, (size_t)n * QCS_OUT_PARA_NUM * sizeof(float), cudaMemcpyHostToDevice,
                             s),
             "copy rows");
    return render_launch(r, r->d_rows, nullptr, n, p, mode, fixed_prec, s);
}

int qcs_render_rows_device(qcs_render_data *r, const float *d_rows, const int *d_n, int max_n, const qcs_loc_para *p,
                           int mode, float fixed_prec, void *stream) {
    if (!r || !p) return fail(QCS_ERR_ARG, "null argument");
    if (max_n < 0) return fail(QCS_ERR_ARG, "negative row count");
    if (max_n > 0 && !d_rows) return fail(QCS_ERR_ARG, "null rows");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    return render_launch(r, d_rows, d_n, max_n, p, mode, fixed_prec, s);
}

float *qcs_render_d_image(qcs_render_data *r) { return r ? r->d_img : nullptr; }
float *qcs_render_d_colormap(qcs_render_data *r) { return r ? r->d_cmap : nullptr; }

int qcs_render_read(qcs_render_data *r, float *h_img, float *h_colormap, int *h_max, int *h_hist, void *stream) {
    if (!r) return fail(QCS_ERR_ARG, "null render context");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    const size_t px = (size_t)r->width * r->high;
    if (h_img) QCS_CUDA(cudaMemcpyAsync(h_img, r->d_img, px * sizeof(float), cudaMemcpyDeviceToHost, s), "read image");
    if (h_colormap && r->d_cmap)
        QCS_CUDA(cudaMemcpyAsync(h_colormap, r->d_cmap, px * sizeof(float), cudaMemcpyDeviceToHost, s),
                 "read colour map");
    if (h_max) QCS_CUDA(cudaMemcpyAsync(h_max, r->d_max, sizeof(int), cudaMemcpyDeviceToHost, s), "read maximum");
    if (h_hist)
        QCS_CUDA(cudaMemcpyAsync(h_hist, r->d_hist, QCS_RENDER_HIST_LEN * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "read histogram");
    QCS_CUDA(cudaStreamSynchronize(s), "read render");
    return QCS_OK;
}

}  // extern "C"
