// Device-side orchestration of LDLocData_TypeDef::BFGS_MLELocalization
// (bfgs_top.cu:26-204): classify -> single-emitter fit -> 2E fit -> 3E fit
// (GS2D) -> CRLB, entirely on one stream with no host round trip.  The
// reference reads the queue lengths back to the host between the stages
// (five synchronisations per batch) and fills the queues with atomics; here
// every queue is built by an order-preserving compaction kernel and every
// fit launch reads its length from device memory, so the result (including
// the order of appended second emitters) is deterministic: ascending ROI
// order for the queues, queue order for appended rows.
#include <cstdint>
#include <cuda_runtime.h>

#include "qcs_cascade.h"
#include "qcs_fit_math.cuh"
#include "qcs_kernels.h"

namespace qcs {
namespace {

constexpr int kScanThreads = 1024;

// Block-wide exclusive scan of one predicate per thread (kScanThreads =
// 1024 = 32 warps); returns the prefix, *total (shared) receives the total.
__device__ __forceinline__ int block_scan(int pred, int *total) {
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ballot = __ballot_sync(0xffffffffu, pred);
    const int in_warp = __popc(ballot & ((1u << lane) - 1u));
    __syncthreads();  // previous call's readers are done with warp_sums / *total
    if (lane == 0) warp_sums[warp] = __popc(ballot);
    __syncthreads();
    if (warp == 0) {
        const int v = warp_sums[lane];
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        warp_sums[lane] = x - v;
        if (lane == 31) *total = x;
    }
    __syncthreads();
    return warp_sums[warp] + in_warp;
}

// Split records by WLE molecule type into the single-emitter queue
// (MLEFit, WLEFit) and the two-emitter queue (MultiFit), both ascending
// (bfgs_top_MoleculeClasify.cu:26-92).  With a predicted emitter-count class
// per record (pred, learned path only: 0 one emitter, 1 the two-emitter
// stage, 2 the three-emitter stage), class 2 goes straight to the 3E queue
// and class 1 to the 2E queue, so neither pays for the fits that would have
// rejected it; pred == null is the reference's split.
__global__ void __launch_bounds__(kScanThreads) classify_queues_kernel(const float *__restrict__ wle, int n,
                                                                       const int *__restrict__ n_dev, int multi,
                                                                       const uint8_t *__restrict__ pred,
                                                                       CascadeState st) {
    __shared__ int tot;
    if (n_dev) n = min(max(*n_dev, 0), n);
    int n1 = 0, n2 = 0, n3 = 0;
    for (int base = 0; base < n; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const int valid = i < n;
        const int type = valid ? (int)wle[(size_t)i * QCS_WLE_PARA_NUM + 5] : 0;
        const int cls = (valid && pred) ? pred[i] : 0;
        const int to_3e = valid && multi && cls == 2;
        const int to_multi = valid && multi && !to_3e && (type > QCS_MOLECULE_WLEFIT || cls == 1);
        const int to_single = valid && !to_multi && !to_3e;
        int p1 = block_scan(to_single, &tot);
        const int t1 = tot;
        if (to_single) st.q_single[n1 + p1] = i;
        int p2 = block_scan(to_multi, &tot);
        const int t2 = tot;
        if (to_multi) st.q2[n2 + p2] = i;
        int p3 = block_scan(to_3e, &tot);
        const int t3 = tot;
        if (to_3e) st.q3[n3 + p3] = i;
        n1 += t1;
        n2 += t2;
        n3 += t3;
    }
    if (threadIdx.x == 0) {
        st.counters[kCntSingle] = n1;
        st.counters[kCnt2E] = n2;
        st.counters[kCnt2EClassify] = n2;
        st.counters[kCnt3E] = n3;
        st.counters[kCnt3EClassify] = n3;
        st.counters[kCntRejected] = 0;
        st.counters[kCntRows] = n;
    }
}

// Append single-emitter rejects with SNR > 6 to the two-emitter queue, in
// single-queue order (bfgsMLE_GS2D_core.h:279-298).
__global__ void __launch_bounds__(kScanThreads) append_2e_kernel(CascadeState st) {
    __shared__ int tot;
    const int ns = st.counters[kCntSingle];
    int n2 = st.counters[kCnt2E];
    for (int base = 0; base < ns; base += kScanThreads) {
        const int k = base + threadIdx.x;
        int id = 0, pred = 0;
        if (k < ns) {
            id = st.q_single[k];
            pred = st.to2e[id];
        }
        const int p = block_scan(pred, &tot);
        if (pred) st.q2[n2 + p] = id;
        n2 += tot;
    }
    if (threadIdx.x == 0) st.counters[kCnt2E] = n2;
}

// Walk the multi-emitter queue slots in order: append second emitters after
// the current rows, and route rejections to the next queue (3E) or the
// rejected count.  stage 2 = after the 2E fit, 3 = after the 3E fit.
__global__ void __launch_bounds__(kScanThreads) compact_multi_kernel(CascadeState st, float *__restrict__ loc,
                                                                     int stage, int route_rejects_to_3e,
                                                                     int max_rows) {
    __shared__ int tot;
    const int nslots = (stage == 2) ? st.counters[kCnt2E] : st.counters[kCnt3E];
    const int8_t *res = (stage == 2) ? st.res2 : st.res3;
    const float *extra = (stage == 2) ? st.extra2 : st.extra3;
    const int *queue = (stage == 2) ? st.q2 : st.q3;
    int rows = st.counters[kCntRows];
    // after the 2E stage, rejects follow the records classified straight to 3E
    int n3 = (stage == 2) ? st.counters[kCnt3E] : 0, rejected = st.counters[kCntRejected];
    for (int base = 0; base < nslots; base += kScanThreads) {
        const int k = base + threadIdx.x;
        const int r = (k < nslots) ? res[k] : -1;
        const int is2 = (r == 2);
        const int is0 = (r == 0);
        const int p2 = block_scan(is2, &tot);
        const int t2 = tot;
        if (is2) {
            const int dst = rows + p2;
            if (dst < max_rows) {
                const float4 *s = reinterpret_cast<const float4 *>(extra + (size_t)k * 12);
                float4 *d = reinterpret_cast<float4 *>(loc + (size_t)dst * 12);
                d[0] = s[0];
                d[1] = s[1];
                d[2] = s[2];
            }
        }
        rows += t2;
        const int p0 = block_scan(is0 && route_rejects_to_3e, &tot);
        const int t0 = tot;
        if (is0 && route_rejects_to_3e) st.q3[n3 + p0] = queue[k];
        n3 += t0;
        if (!route_rejects_to_3e) {
            const int pr = block_scan(is0, &tot);
            (void)pr;
            rejected += tot;
        }
    }
    if (threadIdx.x == 0) {
        st.counters[kCntRows] = rows;
        st.counters[kCntRejected] = rejected;
        if (stage == 2) st.counters[kCnt3E] = n3;
        st.counters[kCntValid] = rows < max_rows ? rows : max_rows;
    }
}

__global__ void init_counters_kernel(CascadeState st, int n, const int *__restrict__ n_dev) {
    if (n_dev) n = min(max(*n_dev, 0), n);
    st.counters[kCntSingle] = n;
    st.counters[kCnt2E] = 0;
    st.counters[kCnt2EClassify] = 0;
    st.counters[kCnt3E] = 0;
    st.counters[kCnt3EClassify] = 0;
    st.counters[kCntRejected] = 0;
    st.counters[kCntRows] = n;
}

__global__ void finish_kernel(CascadeState st, int max_rows) {
    const int rows = st.counters[kCntRows];
    st.counters[kCntValid] = rows < max_rows ? rows : max_rows;
}

}  // namespace

cudaError_t cascade_classify(const CascadeArgs &a, const CascadeState &st) {
    if (a.para.MultiEmitterFitEn)
        classify_queues_kernel<<<1, kScanThreads, 0, a.stream>>>(a.wle, a.n, a.n_dev, 1, a.pred, st);
    else
        init_counters_kernel<<<1, 1, 0, a.stream>>>(st, a.n, a.n_dev);
    return cudaGetLastError();
}

FitLaunch cascade_single_launch(const CascadeArgs &a, const CascadeState &st) {
    const int multi = a.para.MultiEmitterFitEn;
    FitLaunch f;
    f.rois = a.rois;
    f.wle = a.wle;
    f.loc = a.loc;
    f.para = core_para(a.para);
    f.stream = a.stream;
    f.mo = MultiOut{nullptr, nullptr};
    // Single emitter over the classify queue (identity when multi-emitter
    // fitting is off, as in the reference); its length is on the device.
    f.q = Queue{multi ? st.q_single : nullptr, st.counters + kCntSingle, 0};
    f.max_count = a.n;
    f.to2e = multi ? st.to2e : nullptr;
    return f;
}

cudaError_t cascade_tail(const CascadeArgs &a, const CascadeState &st) {
    const qcs_loc_para &p = a.para;
    const int n = a.n;
    const int R = p.ROISize;
    const int multi = p.MultiEmitterFitEn;
    const bool as3d = (p.LocType == QCS_LOCTYPE_AS3D);
    cudaError_t e;
    FitLaunch f = cascade_single_launch(a, st);
    if (multi) {
        append_2e_kernel<<<1, kScanThreads, 0, a.stream>>>(st);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const bool has2e = (p.LocType == QCS_LOCTYPE_GS2D) || as3d;
        if (has2e) {
            f.q = Queue{st.q2, st.counters + kCnt2E, 0};
            f.max_count = n;
            f.to2e = nullptr;
            f.mo = MultiOut{st.res2, st.extra2};
            if ((e = launch_fit(as3d ? kAS3D2E : k2E, R, f)) != cudaSuccess) return e;
            compact_multi_kernel<<<1, kScanThreads, 0, a.stream>>>(st, a.loc, 2, as3d ? 0 : 1, a.max_rows);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            if (p.LocType == QCS_LOCTYPE_GS2D) {
                f.q = Queue{st.q3, st.counters + kCnt3E, 0};
                f.mo = MultiOut{st.res3, st.extra3};
                if ((e = launch_fit(k3E, R, f)) != cudaSuccess) return e;
                compact_multi_kernel<<<1, kScanThreads, 0, a.stream>>>(st, a.loc, 3, 0, a.max_rows);
                if ((e = cudaGetLastError()) != cudaSuccess) return e;
            }
        }
    }
    finish_kernel<<<1, 1, 0, a.stream>>>(st, a.max_rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_crlb(a.loc, st.counters + kCntValid, 0, multi ? a.max_rows : n, p.LocType, p.ReadNoise_e, p.QE,
                       p.PixelSize, a.stream);
}

cudaError_t run_cascade(const CascadeArgs &a, const CascadeState &st) {
    cudaError_t e = cascade_classify(a, st);
    if (e != cudaSuccess) return e;
    const bool as3d = (a.para.LocType == QCS_LOCTYPE_AS3D);
    if ((e = launch_fit(as3d ? kAS3D : kGS2D, a.para.ROISize, cascade_single_launch(a, st))) != cudaSuccess) return e;
    return cascade_tail(a, st);
}

}  // namespace qcs
