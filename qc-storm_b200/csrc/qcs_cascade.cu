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

// The records' split (bfgs_top_MoleculeClasify.cu:26-92): by WLE molecule
// type into the single-emitter queue (MLEFit, WLEFit) and the two-emitter
// queue (MultiFit), both ascending.  With a predicted emitter-count class per
// record (pred, learned path only: 0 one emitter, 1 the two-emitter stage, 2
// the three-emitter stage), class 2 goes straight to the 3E queue and class 1
// to the 2E queue, so neither pays for the fits that would have rejected it;
// pred == null is the reference's split.  After the single-emitter fit its
// rejects with SNR > 6 follow the classified records in the 2E queue, in
// single-queue order (bfgsMLE_GS2D_core.h:279-298); after each multi-emitter
// fit the queue slots are walked in order, second emitters appended after the
// current rows and rejections routed to the next queue (3E) or counted.  All
// three are order-preserving compactions (ClassifyStage, Append2EStage,
// CompactStage below).

// ---- order-preserving compaction over many blocks --------------------------
// The queues above are built by one block walking all records, 1,024 at a
// time (~100 serial steps for 100,000 records).  The same compactions run here
// over one block per 1,024-element tile in two launches: every tile counts its
// selected elements; then every tile adds the counts of the tiles before it to
// its own prefix sums and scatters, and the last tile writes the totals.  The
// positions are the one-block walk's exactly (ascending element order).  A
// stage S gives the element count (on the device), NP predicates per element,
// where a selected element goes, and the counters after the last element;
// counters it reads and later overwrites are copied first (snapshot, by tile
// 0 of the counting launch) so that no tile reads a value the last tile has
// already replaced.  scan: kScanSnap snapshot ints, then NP counts per tile.
constexpr int kScanSnap = 4;

template <class S>
__global__ void __launch_bounds__(kScanThreads) tile_count_kernel(S s, int *__restrict__ scan) {
    const int n = s.count();
    if (blockIdx.x == 0 && threadIdx.x == 0) s.snapshot(scan);
    const int i = blockIdx.x * kScanThreads + threadIdx.x;
    int f[S::NP];
    s.flags(i, n, f);
#pragma unroll
    for (int p = 0; p < S::NP; ++p) {
        const int c = __syncthreads_count(f[p]);
        if (threadIdx.x == 0) scan[kScanSnap + blockIdx.x * S::NP + p] = c;
    }
}

template <class S>
__global__ void __launch_bounds__(kScanThreads) tile_scatter_kernel(S s, const int *__restrict__ scan) {
    __shared__ int base[S::NP];
    __shared__ int tot;
    if (threadIdx.x < 32) {
        int acc[S::NP];
#pragma unroll
        for (int p = 0; p < S::NP; ++p) acc[p] = 0;
        for (int t = threadIdx.x; t < (int)blockIdx.x; t += 32)
#pragma unroll
            for (int p = 0; p < S::NP; ++p) acc[p] += scan[kScanSnap + t * S::NP + p];
#pragma unroll
        for (int p = 0; p < S::NP; ++p) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[p] += __shfl_down_sync(0xffffffffu, acc[p], o);
            if (threadIdx.x == 0) base[p] = acc[p];
        }
    }
    __syncthreads();
    const int n = s.count();
    const int i = blockIdx.x * kScanThreads + threadIdx.x;
    int f[S::NP];
    s.flags(i, n, f);
    int total[S::NP];
#pragma unroll
    for (int p = 0; p < S::NP; ++p) {
        const int pre = block_scan(f[p], &tot);
        if (f[p]) s.emit(p, i, base[p] + pre, scan);
        total[p] = base[p] + tot;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) s.finish(total, scan, n);
}

// the classify split
struct ClassifyStage {
    enum { NP = 3 };
    const float *wle;
    int n;
    const int *n_dev;
    const uint8_t *pred;
    CascadeState st;
    __device__ int count() const { return n_dev ? min(max(*n_dev, 0), n) : n; }
    __device__ void snapshot(int *) const {}
    __device__ void flags(int i, int cnt, int (&f)[NP]) const {
        const int valid = i < cnt;
        const int type = valid ? (int)wle[(size_t)i * QCS_WLE_PARA_NUM + 5] : 0;
        const int cls = (valid && pred) ? pred[i] : 0;
        const int to_3e = valid && cls == 2;
        const int to_multi = valid && !to_3e && (type > QCS_MOLECULE_WLEFIT || cls == 1);
        f[0] = valid && !to_multi && !to_3e;
        f[1] = to_multi;
        f[2] = to_3e;
    }
    __device__ void emit(int p, int i, int pos, const int *) const {
        if (p == 0) st.q_single[pos] = i;
        else if (p == 1) st.q2[pos] = i;
        else st.q3[pos] = i;
    }
    __device__ void finish(const int (&t)[NP], const int *, int cnt) const {
        st.counters[kCntSingle] = t[0];
        st.counters[kCnt2E] = t[1];
        st.counters[kCnt2EClassify] = t[1];
        st.counters[kCnt3E] = t[2];
        st.counters[kCnt3EClassify] = t[2];
        st.counters[kCntRejected] = 0;
        st.counters[kCntRefit3E] = 0;
        st.counters[kCntRows] = cnt;
    }
};

// single-emitter rejects to the 2E queue
struct Append2EStage {
    enum { NP = 1 };
    CascadeState st;
    __device__ int count() const { return st.counters[kCntSingle]; }
    __device__ void snapshot(int *snap) const { snap[0] = st.counters[kCnt2E]; }
    __device__ void flags(int k, int cnt, int (&f)[NP]) const { f[0] = k < cnt ? st.to2e[st.q_single[k]] : 0; }
    __device__ void emit(int, int k, int pos, const int *snap) const { st.q2[snap[0] + pos] = st.q_single[k]; }
    __device__ void finish(const int (&t)[NP], const int *snap, int) const { st.counters[kCnt2E] = snap[0] + t[0]; }
};

// second emitters appended, rejects routed on
struct CompactStage {
    enum { NP = 2 };
    CascadeState st;
    float *loc;
    int stage, route, max_rows;
    __device__ int count() const { return stage == 2 ? st.counters[kCnt2E] : st.counters[kCnt3E]; }
    __device__ void snapshot(int *snap) const {
        snap[0] = st.counters[kCntRows];
        snap[1] = stage == 2 ? st.counters[kCnt3E] : 0;
        snap[2] = st.counters[kCntRejected];
    }
    __device__ void flags(int k, int cnt, int (&f)[NP]) const {
        const int r = k < cnt ? (stage == 2 ? st.res2[k] : st.res3[k]) : -1;
        f[0] = r == 2;
        f[1] = r == 0;
    }
    __device__ void emit(int p, int k, int pos, const int *snap) const {
        if (p == 0) {
            const int dst = snap[0] + pos;
            if (dst < max_rows) {
                const float4 *src = reinterpret_cast<const float4 *>((stage == 2 ? st.extra2 : st.extra3) + (size_t)k * 12);
                float4 *d = reinterpret_cast<float4 *>(loc + (size_t)dst * 12);
                d[0] = src[0];
                d[1] = src[1];
                d[2] = src[2];
            }
        } else if (route) {
            st.q3[snap[1] + pos] = (stage == 2 ? st.q2 : st.q3)[k];
        }
    }
    __device__ void finish(const int (&t)[NP], const int *snap, int) const {
        const int rows = snap[0] + t[0];
        st.counters[kCntRows] = rows;
        st.counters[kCntRejected] = snap[2] + (route ? 0 : t[1]);
        if (stage == 2) st.counters[kCnt3E] = snap[1] + (route ? t[1] : 0);
        st.counters[kCntValid] = rows < max_rows ? rows : max_rows;
    }
};

template <class S>
cudaError_t launch_compaction(const S &s, int max_count, const CascadeState &st, cudaStream_t stream) {
    const int tiles = max_count > 0 ? (max_count + kScanThreads - 1) / kScanThreads : 1;
    tile_count_kernel<S><<<tiles, kScanThreads, 0, stream>>>(s, st.scan);
    tile_scatter_kernel<S><<<tiles, kScanThreads, 0, stream>>>(s, st.scan);
    return cudaGetLastError();
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
    st.counters[kCntRefit3E] = 0;
}

// Likelihood-ratio selection of each record's model (run_cascade_lr); the
// chosen model's first row replaces loc[i], its second emitter (if any) goes
// to extra2[i] with res2[i] = 1 or 2 (0: no model accepted), which the
// cascade's append compaction then reads as a two-emitter stage over all
// records.
__global__ void lr_select_kernel(CascadeState st, float *__restrict__ loc, LrScratch lr, int n,
                                 const int *__restrict__ n_dev) {
    __shared__ int cnt[3];
    if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
    __syncthreads();
    if (n_dev) n = min(max(*n_dev, 0), n);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const bool a1 = loc[(size_t)i * 12] > 0.0f, a2 = st.res2[i] >= 1, a3 = st.res3[i] >= 1;
        const double l1 = lr.ll1[i], l2 = lr.ll2[i], l3 = lr.ll3[i];
        const double th = lr.threshold;
        int best = a1 ? 1 : 0;
        double lb = l1;
        if (a2 && (best == 0 || 2.0 * (l2 - lb) > th * (2 - best))) {
            best = 2;
            lb = l2;
        }
        if (a3 && (best == 0 || 2.0 * (l3 - lb) > th * (3 - best))) best = 3;
        float4 *dst = reinterpret_cast<float4 *>(loc + (size_t)i * 12);
        if (best >= 2) {
            const float4 *src = reinterpret_cast<const float4 *>((best == 2 ? lr.loc2 : lr.loc3) + (size_t)i * 12);
            dst[0] = src[0];
            dst[1] = src[1];
            dst[2] = src[2];
        }
        if (best == 3) {
            const float4 *src = reinterpret_cast<const float4 *>(st.extra3 + (size_t)i * 12);
            float4 *x = reinterpret_cast<float4 *>(st.extra2 + (size_t)i * 12);
            x[0] = src[0];
            x[1] = src[1];
            x[2] = src[2];
        }
        st.res2[i] = (int8_t)(best == 0 ? 0 : (best == 1 ? 1 : (best == 2 ? st.res2[i] : st.res3[i])));
        if (best > 0) atomicAdd(&cnt[best - 1], 1);
    }
    __syncthreads();
    if (threadIdx.x < 3 && cnt[threadIdx.x]) atomicAdd(st.counters + kCntSel1 + threadIdx.x, cnt[threadIdx.x]);
}

// counters of run_cascade_lr: every record is in each stage's (identity) queue
__global__ void lr_counters_kernel(CascadeState st, int n, const int *__restrict__ n_dev) {
    if (n_dev) n = min(max(*n_dev, 0), n);
    st.counters[kCntSingle] = n;
    st.counters[kCnt2E] = n;
    st.counters[kCnt2EClassify] = 0;
    st.counters[kCnt3E] = n;
    st.counters[kCnt3EClassify] = 0;
    st.counters[kCntRejected] = 0;
    st.counters[kCntRows] = n;
    st.counters[kCntSel1] = 0;
    st.counters[kCntSel2] = 0;
    st.counters[kCntSel3] = 0;
}

__global__ void finish_kernel(CascadeState st, int max_rows) {
    const int rows = st.counters[kCntRows];
    st.counters[kCntValid] = rows < max_rows ? rows : max_rows;
}

}  // namespace

cudaError_t cascade_classify(const CascadeArgs &a, const CascadeState &st) {
    if (a.para.MultiEmitterFitEn) return launch_compaction(ClassifyStage{a.wle, a.n, a.n_dev, a.pred, st}, a.n, st, a.stream);
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
        if (a.starts_ready && (e = cudaStreamWaitEvent(a.stream, a.starts_ready, 0)) != cudaSuccess) return e;
        if ((e = launch_compaction(Append2EStage{st}, n, st, a.stream)) != cudaSuccess) return e;
        const bool has2e = (p.LocType == QCS_LOCTYPE_GS2D) || as3d;
        if (has2e) {
            f.q = Queue{st.q2, st.counters + kCnt2E, 0};
            f.max_count = n;
            f.to2e = nullptr;
            f.mo = MultiOut{st.res2, st.extra2};
            f.group_limit = a.group_limit2;
            if (a.two && !as3d) {
                // learned starts; the plain refits write into the (still unused) 3E stage's arrays and are
                // merged back into their slots
                const TwoEmitterStart &t = *a.two;
                if ((e = launch_fit_learned_2e(R, t.iters, t.bisections, f, t.start, t.dev_th, t.refit,
                                               t.to3e == 1 ? 1 : 0)) != cudaSuccess)
                    return e;
                if (!t.to3e && (e = launch_flag_slots(t.refit, st.counters + kCnt2E, n, st.q2, t.slots, t.ids,
                                           st.counters + kCntRefit2E, a.stream)) != cudaSuccess)
                    return e;
                if (t.to3e) {  // to the 3E fit, or no refit
                    if ((e = cudaMemsetAsync(st.counters + kCntRefit2E, 0, sizeof(int), a.stream)) != cudaSuccess)
                        return e;
                } else {
                    FitLaunch g = f;
                    g.q = Queue{t.ids, st.counters + kCntRefit2E, 0};
                    g.mo = MultiOut{st.res3, st.extra3};
                    if ((e = launch_fit(k2E, R, g)) != cudaSuccess) return e;
                    if ((e = launch_merge_refit(t.slots, st.counters + kCntRefit2E, n, st.res3, st.extra3, st.res2,
                                                st.extra2, a.stream)) != cudaSuccess)
                        return e;
                }
            } else if ((e = launch_fit(as3d ? kAS3D2E : k2E, R, f)) != cudaSuccess) {
                return e;
            }
            if ((e = launch_compaction(CompactStage{st, a.loc, 2, as3d ? 0 : 1, a.max_rows}, n, st, a.stream)) !=
                cudaSuccess)
                return e;
            if (p.LocType == QCS_LOCTYPE_GS2D) {
                f.q = Queue{st.q3, st.counters + kCnt3E, 0};
                f.mo = MultiOut{st.res3, st.extra3, a.params3};
                f.group_limit = a.group_limit3;
                if (a.three) {
                    // learned starts; the plain refits write into the 2E stage's arrays (consumed by its
                    // compaction above) and are merged back into their slots
                    const ThreeEmitterStart &t = *a.three;
                    const bool refits = t.dev_th >= 0.0f;
                    if ((e = launch_fit_learned_3e(R, t.iters, t.bisections, f, t.start, refits ? t.dev_th : 0.0f,
                                                   t.refit)) != cudaSuccess)
                        return e;
                    if (!refits) {
                        if ((e = cudaMemsetAsync(st.counters + kCntRefit3E, 0, sizeof(int), a.stream)) != cudaSuccess)
                            return e;
                    } else if ((e = launch_flag_slots(t.refit, st.counters + kCnt3E, n, st.q3, t.slots, t.ids,
                                               st.counters + kCntRefit3E, a.stream)) != cudaSuccess)
                        return e;
                    if (refits) {
                        FitLaunch g = f;
                        g.q = Queue{t.ids, st.counters + kCntRefit3E, 0};
                        g.mo = MultiOut{st.res2, st.extra2};
                        if ((e = launch_fit(k3E, R, g)) != cudaSuccess) return e;
                        if ((e = launch_merge_refit(t.slots, st.counters + kCntRefit3E, n, st.res2, st.extra2, st.res3,
                                                    st.extra3, a.stream)) != cudaSuccess)
                            return e;
                    }
                } else if ((e = launch_fit(k3E, R, f)) != cudaSuccess) {
                    return e;
                }
                if ((e = launch_compaction(CompactStage{st, a.loc, 3, 0, a.max_rows}, n, st, a.stream)) != cudaSuccess)
                    return e;
            }
        }
    }
    finish_kernel<<<1, 1, 0, a.stream>>>(st, a.max_rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_crlb(a.loc, st.counters + kCntValid, 0, multi ? a.max_rows : n, p.LocType, p.ReadNoise_e, p.QE,
                       p.PixelSize, a.stream);
}

cudaError_t run_cascade_lr(const CascadeArgs &a, const CascadeState &st, const LrScratch &lr) {
    const qcs_loc_para &p = a.para;
    const int n = a.n, R = p.ROISize;
    cudaError_t e;
    lr_counters_kernel<<<1, 1, 0, a.stream>>>(st, n, a.n_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    FitLaunch f;
    f.rois = a.rois;
    f.wle = a.wle;
    f.q = Queue{nullptr, st.counters + kCntSingle, 0};  // identity over the call's records
    f.max_count = n;
    f.loc = a.loc;
    f.to2e = nullptr;
    f.mo = MultiOut{nullptr, nullptr};
    f.para = core_para(p);
    f.stream = a.stream;
    f.ll = lr.ll1;
    if ((e = launch_fit(kGS2D, R, f)) != cudaSuccess) return e;
    // every record goes through the 2E and 3E fits: throughput-bound queues, one thread per ROI
    f.thread_per_roi = 1;
    f.loc = lr.loc2;
    f.mo = MultiOut{st.res2, st.extra2};
    f.ll = lr.ll2;
    if ((e = launch_fit(k2E, R, f)) != cudaSuccess) return e;
    f.loc = lr.loc3;
    f.mo = MultiOut{st.res3, st.extra3};
    f.ll = lr.ll3;
    if ((e = launch_fit(k3E, R, f)) != cudaSuccess) return e;
    if (n > 0) lr_select_kernel<<<(n + 255) / 256, 256, 0, a.stream>>>(st, a.loc, lr, n, a.n_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // second emitters appended after the records, in record order; records with no model counted as rejected
    if ((e = launch_compaction(CompactStage{st, a.loc, 2, 0, a.max_rows}, n, st, a.stream)) != cudaSuccess) return e;
    finish_kernel<<<1, 1, 0, a.stream>>>(st, a.max_rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_crlb(a.loc, st.counters + kCntValid, 0, a.max_rows, p.LocType, p.ReadNoise_e, p.QE, p.PixelSize,
                       a.stream);
}

cudaError_t run_cascade(const CascadeArgs &a, const CascadeState &st) {
    cudaError_t e = cascade_classify(a, st);
    if (e != cudaSuccess) return e;
    const bool as3d = (a.para.LocType == QCS_LOCTYPE_AS3D);
    const int kind = as3d ? kAS3D : kGS2D;
    // the lane-group kernel gives the one-thread kernel's rows bit for bit; which is faster depends on the batch
    if (a.lanes > 1 && group_fit_supported(kind, a.para.ROISize))
        e = launch_fit_group(kind, a.para.ROISize, (kind == kGS2D && a.para.ROISize == 7) ? a.lanes : 8,
                             cascade_single_launch(a, st));
    else
        e = launch_fit(kind, a.para.ROISize, cascade_single_launch(a, st));
    if (e != cudaSuccess) return e;
    return cascade_tail(a, st);
}

}  // namespace qcs
