// Fit kernels: single-emitter GS2D / AS3D and multi-emitter GS2D-2E, GS2D-3E,
// AS3D-2E.  One thread per ROI; a block stages its ROIs' pixels into shared
// memory in a [pixel][thread] layout (conflict-free: thread t reads column t),
// each thread then pre-estimates, fits with the fixed schedule of
// qcs_fit_math.cuh and writes its 12-float row.  Queues come from device
// memory, so the whole single -> 2E -> 3E cascade runs without host syncs.
//
// Reference kernels re-expressed (MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/bfgsMLE_dll/):
//   bfgsMLE_Loc_LD/bfgsMLE_GS2D_core.h:57-310, 522-575   bfgsMLELoc_Gauss2D, PreEstimation_GS2D
//   bfgsMLE_Loc_LD/bfgsMLE_AS3D_core.h:58-337, 548-607   bfgsMLELoc_AS3D, PreEstimation_AS3D
//   bfgsMLE_Loc_HD/bfgsMLE_GS2D_2Emitter_core.h:75-371, 596-698
//   bfgsMLE_Loc_HD/bfgsMLE_GS2D_3Emitter_core.h:77-362, 593-710
//   bfgsMLE_Loc_HD/bfgsMLE_AS3D_2Emitter_core.h:78-422, 648-750
// Differences in layout only: the reference writes second emitters through
// an atomic counter (arbitrary order) and queues ROIs with atomics; here each
// multi-emitter queue slot records its outcome and a compaction kernel
// appends rows in queue order (qcs_cascade.cu), which is deterministic.
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>
#include <utility>

#include "qcs_device.cuh"
#include "qcs_fit_math.cuh"
#include "qcs_kernels.h"

#define rAScalFactor (1.0f / QCS_ASCALE)
#define rBScalFactor (1.0f / QCS_BSCALE)
#define rSScalFactor (1.0f / QCS_SSCALE)

namespace qcs {
namespace {

constexpr int kTPB = 64;  // ROIs (threads) per block

// One ROI's staged photoelectron values: pixel k at p[k * ld].x.
struct PixView {
    const float2 *p;
    int ld;
    __device__ __forceinline__ float operator[](int k) const { return p[k * ld].x; }
};

template <int R, int KIND>
struct SmemLayout {
    enum {
        P = KindTraits<KIND>::P,
        PIX = R * R,
        IMG = 0,                 // float2 (value, log) pairs: 2 floats per element
        W = 2 * PIX * kTPB,
        D = W + (KindTraits<KIND>::WEIGHTED ? PIX * kTPB : 0),
        TOTAL = D + P * P * kTPB,  // floats
    };
};

// Stage the block's ROIs: element k of slot s at smem[k * kTPB + s].
// Each value is stored with its natural log (the data term of the Poisson
// deviance), computed once instead of once per loss evaluation, as one
// float2 so that the loss reads both with a single 64-bit load.
template <int R>
__device__ __forceinline__ void stage_rois(float2 *s_img, const uint16_t *rois, const Queue &q, int base, int cnt,
                                           float Offset, float KAdc) {
    enum { PIX = R * R, WHOLE = R * (R + 1) };
    for (int idx = threadIdx.x; idx < cnt * PIX; idx += kTPB) {
        const int slot = idx / PIX;
        const int k = idx - slot * PIX;
        const int id = queue_at(q, base + slot);
        const uint16_t u = __ldg(rois + (size_t)id * WHOLE + k);
        const float pixval = fmaxf((u - Offset) * KAdc, 1.0f);
        s_img[k * kTPB + slot] = make_float2(pixval, __logf(pixval));
    }
}

__device__ __forceinline__ void store_row(float *loc, int id, const float (&v)[12]) {
    float4 *dst = reinterpret_cast<float4 *>(loc + (size_t)id * 12);
    dst[0] = make_float4(v[0], v[1], v[2], v[3]);
    dst[1] = make_float4(v[4], v[5], v[6], v[7]);
    dst[2] = make_float4(v[8], v[9], v[10], v[11]);
}

__device__ __forceinline__ void zero_row(float *loc, int id) {
    float4 *dst = reinterpret_cast<float4 *>(loc + (size_t)id * 12);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    dst[0] = z;
    dst[1] = z;
    dst[2] = z;
}

template <int R>
__device__ __forceinline__ void edge_means(const PixView &img, float &Mean1, float &Mean2, float &Mean3, float &Mean4) {
    Mean1 = 0;
    Mean2 = 0;
    Mean3 = 0;
    Mean4 = 0;
#pragma unroll
    for (int cnt = 0; cnt < R; cnt++) {
        Mean1 += img[cnt * R + 0];
        Mean2 += img[cnt * R + R - 1];
        Mean3 += img[0 * R + cnt];
        Mean4 += img[(R - 1) * R + cnt];
    }
}

// Start positions of the extra emitters: the brightest (and for three
// emitters also the second brightest) non-central block of a 3 x 3 tiling.
template <int R>
__device__ __forceinline__ void block_starts(const PixView &img, int nstart, float *xs, float *ys) {
    const int ROISize_Half = R / 2;
    const float ROICenter = R / 2.0f;
    const int SumROILen = R / 3 + 1;
    const int SumROILen_Half = SumROILen / 2;
    int StartPos[3];
    StartPos[0] = 0;
    StartPos[1] = ROISize_Half - SumROILen_Half;
    StartPos[2] = R - SumROILen;
    float RegionPos[3];
    RegionPos[0] = ROICenter - SumROILen / 2.0f;
    RegionPos[1] = ROICenter;
    RegionPos[2] = ROICenter + SumROILen / 2.0f;
    float SumData[9];
    for (int cnt = 0; cnt < 9; cnt++) {
        float SumDat_t = 0;
        const int XBias = StartPos[cnt % 3];
        const int YBias = StartPos[cnt / 3];
        for (int r = 0; r < SumROILen; r++)
            for (int c = 0; c < SumROILen; c++) SumDat_t += img[(r + YBias) * R + c + XBias];
        SumData[cnt] = SumDat_t;
    }
    SumData[9 / 2] = 0;
    for (int e = 0; e < nstart; e++) {
        int MaxPos = 0;
        for (int cnt = 0; cnt < 9; cnt++)
            if (SumData[cnt] > SumData[MaxPos]) MaxPos = cnt;
        xs[e] = RegionPos[MaxPos % 3];
        ys[e] = RegionPos[MaxPos / 3];
        SumData[MaxPos] = 0;
    }
}

__device__ __forceinline__ float zpoly(const CorePara &c, float SigmaDif) {
    float CurZPos;
    if (SigmaDif >= 0.0f)
        CurZPos = c.p4_XGY * powf(SigmaDif, 4) + c.p3_XGY * powf(SigmaDif, 3) + c.p2_XGY * powf(SigmaDif, 2) +
                  c.p1_XGY * SigmaDif + c.p0_XGY;
    else
        CurZPos = c.p4_XLY * powf(SigmaDif, 4) + c.p3_XLY * powf(SigmaDif, 3) + c.p2_XLY * powf(SigmaDif, 2) +
                  c.p1_XLY * SigmaDif + c.p0_XLY;
    return CurZPos * c.ZDepthCorrFactor;
}

// ------------------------------------------------------- single emitter ---
// Weighted-MLE mask widths and accept bound of one single-emitter ROI.
struct SinglePrep {
    float WLE_SigmaX, WLE_SigmaY;
    int MoleculeType;
    float Simga_Max_Th;
};

// PreEstimation_GS2D / PreEstimation_AS3D and the WLE mask widths: the start
// point Ininf of the fit from the ROI's edge means and centre pixel.
// PRE = false: the mask widths and bounds only, Ininf untouched (the
// learned-start fit takes its start point from elsewhere).
template <int R, int KIND, bool PRE = true>
__device__ __forceinline__ SinglePrep single_prefit(const PixView &img, const float *pw, const CorePara &c,
                                                    float *Ininf) {
    SinglePrep sp;
    sp.Simga_Max_Th = R / 1.5f / 2.35f;
    if (c.MultiEmitterFitEn) sp.Simga_Max_Th = R / 2.0f / 2.35f;
    if (KIND == kGS2D) {
        float SigmaL = pw[1], SigmaR = pw[2], SigmaU = pw[3], SigmaD = pw[4];
        const int MoleculeType = pw[5];
        SigmaL = fminf(SigmaL, SigmaR);
        SigmaU = fminf(SigmaU, SigmaD);
        float WLE_SigmaX = fminf(SigmaL, SigmaU);
        WLE_SigmaX = fminf(WLE_SigmaX, R / 2.0f / 2.35f);
        // PreEstimation_GS2D
        if constexpr (PRE) {
            const int CenterPos = R / 2;
            float Mean1, Mean2, Mean3, Mean4;
            edge_means<R>(img, Mean1, Mean2, Mean3, Mean4);
            Mean1 = fminf(Mean1, Mean2);
            Mean3 = fminf(Mean3, Mean4);
            const float Bkg = (Mean1 + Mean3) / 2 / R;
            const float Amp = img[CenterPos * R + CenterPos] - Bkg;
            const float SigmaX = WLE_SigmaX;
            const float ParaSigma1 = (1.0f / (2.0f * SigmaX * SigmaX));
            Ininf[0] = Amp * rAScalFactor;
            Ininf[1] = (float)CenterPos + 0.5f;
            Ininf[2] = (float)CenterPos + 0.5f;
            Ininf[3] = ParaSigma1 * rSScalFactor;
            Ininf[4] = Bkg * rBScalFactor;
        }
        if (MoleculeType != QCS_MOLECULE_MLEFIT) {
            WLE_SigmaX = WLE_SigmaX / 1.2f;
            WLE_SigmaX = fminf(WLE_SigmaX, R / 2.0f / 2.35f);
        }
        if (c.WLEEn == 0 && MoleculeType != QCS_MOLECULE_MULTIFIT) WLE_SigmaX = R;
        sp.WLE_SigmaX = WLE_SigmaX;
        sp.WLE_SigmaY = WLE_SigmaX;
        sp.MoleculeType = MoleculeType;
    } else {  // kAS3D
        const float SigmaL = pw[1], SigmaR = pw[2], SigmaU = pw[3], SigmaD = pw[4];
        const int MoleculeType = pw[5];
        float WLE_SigmaX = fminf(SigmaL, SigmaR);
        float WLE_SigmaY = fminf(SigmaU, SigmaD);
        // PreEstimation_AS3D
        if constexpr (PRE) {
            const int CenterPos = R / 2;
            float Mean1, Mean2, Mean3, Mean4;
            edge_means<R>(img, Mean1, Mean2, Mean3, Mean4);
            Mean1 = fminf(Mean1, Mean2);
            Mean3 = fminf(Mean3, Mean4);
            const float Bkg = (Mean1 + Mean3) / 2 / R;
            const float Amp = img[CenterPos * R + CenterPos] - Bkg;
            const float SigmaX = WLE_SigmaX;
            const float SigmaY = WLE_SigmaY;
            const float SigmaX1 = rSScalFactor * (0.5f / (SigmaX * SigmaX));
            const float SigmaY1 = rSScalFactor * (0.5f / (SigmaY * SigmaY));
            Ininf[0] = Amp * rAScalFactor;
            Ininf[1] = (float)CenterPos + 0.5f;
            Ininf[2] = (float)CenterPos + 0.5f;
            Ininf[3] = SigmaX1;
            Ininf[4] = SigmaY1;
            Ininf[5] = Bkg * rBScalFactor;
        }
        if (MoleculeType != QCS_MOLECULE_MLEFIT) {
            WLE_SigmaX = fminf(WLE_SigmaX, R / 1.6f / 2.35f);
            WLE_SigmaY = fminf(WLE_SigmaY, R / 1.6f / 2.35f);
        }
        if (c.WLEEn == 0 && MoleculeType != QCS_MOLECULE_MULTIFIT) {
            WLE_SigmaX = R;
            WLE_SigmaY = R;
        }
        sp.WLE_SigmaX = WLE_SigmaX;
        sp.WLE_SigmaY = WLE_SigmaY;
        sp.MoleculeType = MoleculeType;
    }
    return sp;
}

// Output row and accept decision of a finished single-emitter fit.
template <int R, int KIND>
__device__ __forceinline__ void single_finish(const float *Ininf, const CorePara &c, float Simga_Max_Th, int XOffset,
                                              int YOffset, int CurFrame, float (&row)[12], bool &accepted,
                                              float &CurSNR, int &IsFittingValid) {
    enum { ROISize_Half = R / 2 };
    if (KIND == kGS2D) {
        const float XYLBound = R / 2.0f - 1.5f;
        const float XYUBound = R / 2.0f + 1.5f;
        const float PeakPhoton = Ininf[0] * QCS_ASCALE / c.QE;
        const float Background = Ininf[4] * QCS_BSCALE / c.QE;
        float FittedXPos = Ininf[1];
        float FittedYPos = Ininf[2];
        float SimgaX = Ininf[3] * QCS_SSCALE;
        SimgaX = sqrtf(0.5f / SimgaX);
        FittedXPos = isnan(FittedXPos) ? -1 : FittedXPos;
        FittedYPos = isnan(FittedYPos) ? -1 : FittedYPos;
        SimgaX = isnan(SimgaX) ? -1 : SimgaX;
        CurSNR = sqrtf(c.QE) * PeakPhoton / sqrtf(PeakPhoton + Background);
        const float TotalPhoton = PeakPhoton * 2 * 3.141593f * SimgaX * SimgaX;
        const float XPos = FittedXPos - ROISize_Half + XOffset;
        const float YPos = FittedYPos - ROISize_Half + YOffset;
        IsFittingValid = isnan(Background) ? 0 : 1;
        accepted = IsFittingValid && (CurSNR > 4.0f) && (SimgaX <= Simga_Max_Th) && (SimgaX >= 0.6f) &&
                   (FittedXPos > XYLBound) && (FittedXPos < XYUBound) && (FittedYPos > XYLBound) &&
                   (FittedYPos < XYUBound);
        row[0] = PeakPhoton;
        row[1] = XPos;
        row[2] = YPos;
        row[3] = 0.0f;
        row[4] = SimgaX;
        row[5] = SimgaX;
        row[6] = TotalPhoton;
        row[7] = Background;
        row[8] = CurSNR;
        row[11] = CurFrame;
    } else {  // kAS3D
        const float XYLBound = R / 2.0f - 2.5f;
        const float XYUBound = R / 2.0f + 2.5f;
        const float Simga_Min_Th = 0.8f;
        float PeakPhoton = Ininf[0] * QCS_ASCALE;
        float Background = Ininf[5] * QCS_BSCALE;
        float FittedXPos = Ininf[1];
        float FittedYPos = Ininf[2];
        float SimgaX = Ininf[3] * QCS_SSCALE;
        float SimgaY = Ininf[4] * QCS_SSCALE;
        SimgaX = sqrtf(0.5f / SimgaX);
        SimgaY = sqrtf(0.5f / SimgaY);
        FittedXPos = isnan(FittedXPos) ? -1 : FittedXPos;
        FittedYPos = isnan(FittedYPos) ? -1 : FittedYPos;
        SimgaX = isnan(SimgaX) ? -1 : SimgaX;
        SimgaY = isnan(SimgaY) ? -1 : SimgaY;
        CurSNR = PeakPhoton / sqrtf(PeakPhoton + Background);
        PeakPhoton = PeakPhoton / c.QE;
        Background = Background / c.QE;
        const float TotalPhoton = PeakPhoton * 2 * 3.141593f * SimgaX * SimgaY;
        const float SigmaDif = SimgaX * SimgaX - SimgaY * SimgaY;
        const float CurZPos = zpoly(c, SigmaDif);
        const float XPos = FittedXPos - ROISize_Half + XOffset;
        const float YPos = FittedYPos - ROISize_Half + YOffset;
        const float MeanSigma = (SimgaX + SimgaY) / 2;
        IsFittingValid = isnan(Background) ? 0 : 1;
        accepted = IsFittingValid && (CurSNR > 3.5f) && (MeanSigma > Simga_Min_Th) && (MeanSigma < Simga_Max_Th) &&
                   (FittedXPos > XYLBound) && (FittedXPos < XYUBound) && (FittedYPos > XYLBound) &&
                   (FittedYPos < XYUBound);
        row[0] = PeakPhoton;
        row[1] = XPos;
        row[2] = YPos;
        row[3] = CurZPos;
        row[4] = SimgaX;
        row[5] = SimgaY;
        row[6] = TotalPhoton;
        row[7] = Background;
        row[8] = CurSNR;
        row[11] = CurFrame;
    }
    row[9] = 0.0f;
    row[10] = 0.0f;
}

// Shared memory of fit_single_kernel: per slot (thread) the pixels' (value,
// log) pairs, [pixel][slot], and the mask's unique values, [chunk][slot]
// (MaskShape); the BFGS inverse Hessian lives in registers.  Blocks per SM:
// as many as the shared memory holds (228 KB per SM, 1 KB reserved per
// block), at most 7 (at 7 the register budget is 146 per thread).  S slots
// per block: kTPB, or fewer in the mixed-size kernel (an even count, so the
// mask starts on a 16-byte boundary).
template <int R, bool FULL, int S = kTPB>
struct SingleLayout {
    enum {
        PIX = R * R,
        IMG = 0,                  // float2 per pixel and slot
        WU = 2 * PIX * S,         // floats; a multiple of 4 (16-byte aligned)
        TOTAL = WU + MaskShape<R, FULL>::FLOATS * S,
        BYTES = TOTAL * 4,
        FIT = (228 * 1024) / (BYTES + 1024),
        BLOCKS = FIT < 1 ? 1 : (FIT > 7 ? 7 : FIT),
    };
};

// Stage a block's records: pixel k of slot s at s_img[k * S + s] as
// (max((adu - offset) * gain, 1), its __logf).  WORDS: the records are
// 4-byte aligned and read two pixels per load; element (word, slot) is taken
// slot-fastest so a warp's shared-memory stores fall in distinct banks.
template <int R, bool WORDS, int S = kTPB>
__device__ __forceinline__ void stage_single(float2 *s_img, const uint16_t *rois, const Queue &q, int base, int cnt,
                                             float Offset, float KAdc) {
    enum { PIX = R * R, WHOLE = R * (R + 1), WPR = (PIX + 1) / 2 };
    if (WORDS) {
        for (int idx = threadIdx.x; idx < cnt * WPR; idx += kTPB) {
            const int wd = idx / cnt;
            const int slot = idx - wd * cnt;
            const int id = queue_at(q, base + slot);
            const uint32_t u = __ldg(reinterpret_cast<const uint32_t *>(rois + (size_t)id * WHOLE) + wd);
            const int k = 2 * wd;
            const float v0 = fmaxf(((float)(u & 0xFFFFu) - Offset) * KAdc, 1.0f);
            s_img[k * S + slot] = make_float2(v0, __logf(v0));
            if (k + 1 < PIX) {
                const float v1 = fmaxf(((float)(u >> 16) - Offset) * KAdc, 1.0f);
                s_img[(k + 1) * S + slot] = make_float2(v1, __logf(v1));
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < cnt * PIX; idx += kTPB) {
            const int k = idx / cnt;
            const int slot = idx - k * cnt;
            const int id = queue_at(q, base + slot);
            const uint16_t u = __ldg(rois + (size_t)id * WHOLE + k);
            const float pixval = fmaxf((u - Offset) * KAdc, 1.0f);
            s_img[k * S + slot] = make_float2(pixval, __logf(pixval));
        }
    }
}

// One block's tile of the single-emitter fit: queue entries base .. base+S-1
// (those below n), one thread per ROI, S slots of SingleLayout<R, FULL, S>
// in smem.  Every thread of the block calls it (it synchronises the block
// once, after staging).
template <int R, int KIND, bool WORDS, int DIST, int MASK, bool FULL, int S>
__device__ __forceinline__ void single_tile(float *smem, int base, int n, const uint16_t *__restrict__ rois,
                                            const float *__restrict__ wle, const Queue &q, float *__restrict__ loc,
                                            uint8_t *__restrict__ to2e, const CorePara &c, double *__restrict__ ll) {
    typedef SingleLayout<R, FULL, S> L;
    enum { P = KindTraits<KIND>::P, PIX = R * R, WHOLE = R * (R + 1) };
    if (base >= n) return;
    const int cnt = min(S, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    stage_single<R, WORDS, S>(s_img, rois, q, base, cnt, c.Offset, c.KAdc);
    __syncthreads();
    const int tid = threadIdx.x;
    if (tid >= cnt) return;

    const int CurFluoID = queue_at(q, base + tid);
    const PixView img{s_img + tid, S};
    // the mask: FULL, pixel k at mask[k * S]; else float4 chunk j at ((float4 *)mask)[j * S]
    float *mask = smem + L::WU + (FULL ? tid : 4 * tid);
    const uint16_t *hdr = rois + (size_t)CurFluoID * WHOLE + PIX;
    const int XOffset = hdr[0];
    const int YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const float *pw = wle + (size_t)CurFluoID * QCS_WLE_PARA_NUM;

    float Ininf[P];
    const SinglePrep sp = single_prefit<R, KIND>(img, pw, c, Ininf);
    if constexpr (FULL)
        wle_weights<R, MASK>(mask, S, sp.WLE_SigmaX, sp.WLE_SigmaY, sp.MoleculeType);
    else
        wle_weights_unique<R, MASK>(reinterpret_cast<float4 *>(mask), S, sp.WLE_SigmaX, sp.WLE_SigmaY,
                                    sp.MoleculeType);
    float D[P * P];  // the inverse Hessian, in registers
    bfgs_fit<P, KindTraits<KIND>::IT>(StagedEval<R, KIND, DIST, FULL>{s_img + tid, mask, S}, Ininf, D, 1);
    if (ll) ll[CurFluoID] = model_loglik<R, KIND, DIST, kCompiler>(s_img + tid, S, Ininf, 0, 1);
    float row[12];
    bool accepted;
    float CurSNR;
    int IsFittingValid;
    single_finish<R, KIND>(Ininf, c, sp.Simga_Max_Th, XOffset, YOffset, CurFrame, row, accepted, CurSNR,
                           IsFittingValid);
    if (accepted)
        store_row(loc, CurFluoID, row);
    else
        zero_row(loc, CurFluoID);
    if (to2e) to2e[CurFluoID] = (!accepted && c.MultiEmitterFitEn && IsFittingValid && (CurSNR > 6.0f)) ? 1 : 0;
}

template <int R, int KIND, bool WORDS, int DIST = ArithSpec<KIND, R>::DIST, int MASK = ArithSpec<KIND, R>::MASK,
          bool FULL = MASK == kCompiler>
__global__ void __launch_bounds__(kTPB, (SingleLayout<R, FULL>::BLOCKS)) fit_single_kernel(
    const uint16_t *__restrict__ rois, const float *__restrict__ wle, Queue q, float *__restrict__ loc,
    uint8_t *__restrict__ to2e, CorePara c, double *__restrict__ ll) {
    extern __shared__ __align__(16) float smem[];
    single_tile<R, KIND, WORDS, DIST, MASK, FULL, kTPB>(smem, blockIdx.x * kTPB, queue_len(q), rois, wle, q, loc,
                                                         to2e, c, ll);
}

// ------------------------------------------------ mixed-size single fits ---
// One persistent launch fits the single-emitter queues of several calls of
// different ROI sizes (GS2D / AS3D 7x7, 9x9, 11x11): each block takes the
// next tile of the shared work list with an atomic counter and fits it with
// that size's single_tile, so no block waits on another and the last tiles of
// every size spread over all SMs.  Every block has the same shared memory
// (kMixedBlocks blocks per SM); a tile holds 64 ROIs, else 32 where those fit
// (so no warp runs partly filled), else an even count, one thread each.  The
// tiles of the larger ROIs come first in the list, so the longest fits start
// first.  The arithmetic is fit_single_kernel's: the rows are the per-size
// launches' rows bit for bit.  One launch has one register count: 6 blocks
// per SM allow 168 registers a thread, which the 7x7 (128) and GS2D 9x9 (168)
// fits need, while the per-size GS2D 11x11 and AS3D 9x9 / 11x11 kernels use
// 180 to 254; those fits run slower here than in their own launches.
constexpr int kMixedBlocks = 6;
// floats of dynamic shared memory per block: 228 KB per SM less 1 KB reserved and the kernel's static
// shared memory per block, in 16-byte units
constexpr int kMixedBudget = ((228 * 1024 / kMixedBlocks - 1024 - 64) / 4) & ~3;

template <int R, int KIND>
struct MixedShape {
    enum {
        MASK = ArithSpec<KIND, R>::MASK,
        FULL = MASK == kCompiler,
        PER = 2 * R * R + MaskShape<R, (bool)FULL>::FLOATS,  // floats per ROI
        FIT = kMixedBudget / PER,
        S = FIT >= kTPB ? kTPB : (FIT >= 32 ? 32 : FIT & ~1),
    };
    static_assert(S >= 2, "a mixed-size tile holds at least two ROIs");
};

__host__ __device__ constexpr int mixed_code(int kind, int R) { return kind * 32 + R; }

struct MixedSeg {
    const uint16_t *rois;
    const float *wle;
    Queue q;
    float *loc;
    uint8_t *to2e;
    CorePara c;
    int code;   // mixed_code(kind, R)
    int slots;  // ROIs per tile
};

struct MixedArgs {
    MixedSeg seg[kMixedMax];
    int count;
    int *next;  // zero at launch: the next tile to take
};

template <int R, int KIND>
__device__ __forceinline__ void mixed_tile(float *smem, int base, int n, const MixedSeg &g) {
    typedef MixedShape<R, KIND> M;
    single_tile<R, KIND, true, ArithSpec<KIND, R>::DIST, M::MASK, (bool)M::FULL, M::S>(smem, base, n, g.rois, g.wle,
                                                                                     g.q, g.loc, g.to2e, g.c, nullptr);
}

__global__ void __launch_bounds__(kTPB, kMixedBlocks) fit_mixed_kernel(const __grid_constant__ MixedArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ int s_len[kMixedMax], s_end[kMixedMax], s_tile;
    if (threadIdx.x == 0) {
        int end = 0;
        for (int i = 0; i < a.count; ++i) {
            const int n = queue_len(a.seg[i].q);
            s_len[i] = n;
            end += (n + a.seg[i].slots - 1) / a.seg[i].slots;
            s_end[i] = end;
        }
    }
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(a.next, 1);
        __syncthreads();
        int t = s_tile;
        if (t >= s_end[a.count - 1]) return;  // the same for every thread of the block
        int i = 0;
        while (t >= s_end[i]) ++i;
        if (i > 0) t -= s_end[i - 1];
        const MixedSeg &g = a.seg[i];
        const int base = t * g.slots, n = s_len[i];
        switch (g.code) {
        case mixed_code(kGS2D, 7): mixed_tile<7, kGS2D>(smem, base, n, g); break;
        case mixed_code(kGS2D, 9): mixed_tile<9, kGS2D>(smem, base, n, g); break;
        case mixed_code(kGS2D, 11): mixed_tile<11, kGS2D>(smem, base, n, g); break;
        case mixed_code(kAS3D, 7): mixed_tile<7, kAS3D>(smem, base, n, g); break;
        case mixed_code(kAS3D, 9): mixed_tile<9, kAS3D>(smem, base, n, g); break;
        case mixed_code(kAS3D, 11): mixed_tile<11, kAS3D>(smem, base, n, g); break;
        }
        __syncthreads();  // the tile's shared memory and s_tile are free again
    }
}

// The same fit with G lanes per ROI (GroupEval): bit for bit the rows of
// fit_single_kernel, with about half the latency per ROI and about twice the
// instructions.  For short queues (refits, small calls), where one thread
// per ROI leaves the GPU mostly idle and the launch lasts as long as one
// thread's serial fit.  Each ROI's pixels, weights and loss terms are
// contiguous in shared memory (rows padded to 4 floats); D per lane.
constexpr int kGroupTPB = 128;
// Lanes per ROI of the multi-emitter group kernel: one central-difference
// point per lane (2E: 16 points; 3E, AS3D-2E: 22 points).
__host__ __device__ constexpr int multi_lanes(int kind) { return kind == k2E ? 16 : 32; }

// Multi-emitter kinds and sizes whose roundings (pixel distance and the first
// two emitters' model sum) are fixed in the source: there the group kernel's
// rows equal the thread kernel's bit for bit.
__host__ __device__ constexpr bool multi_group_supported(int kind, int R) {
    return ((kind == k2E || kind == k3E) && (R == 7 || R == 11)) || (kind == kAS3D2E && R == 7);
}

template <int R, int KIND>
struct GroupLayout {
    enum {
        P = KindTraits<KIND>::P,
        PIX = R * R,
        PIXP = (PIX + 3) / 4 * 4,
    };
    template <int G>
    struct At {
        enum {
            SLOTS = kGroupTPB / G,
            IMG = 0,                       // float2 per pixel
            W = IMG + 2 * PIXP * SLOTS,    // floats
            PART = W + PIXP * SLOTS,
            D = PART + PIXP * SLOTS,
            TOTAL = D + P * P * kGroupTPB,
        };
    };
};

template <int R, int KIND, int G, int DIST = ArithSpec<KIND, R>::DIST, int MASK = ArithSpec<KIND, R>::MASK>
__global__ void __launch_bounds__(kGroupTPB) fit_single_group_kernel(const uint16_t *__restrict__ rois,
                                                                     const float *__restrict__ wle, Queue q,
                                                                     float *__restrict__ loc,
                                                                     uint8_t *__restrict__ to2e, CorePara c) {
    typedef GroupLayout<R, KIND> GL;
    typedef typename GL::template At<G> L;
    enum { P = KindTraits<KIND>::P, PIX = R * R, PIXP = GL::PIXP, WHOLE = R * (R + 1), SLOTS = L::SLOTS };
    static_assert(G == 4 || G == 8 || G == 16, "lanes per ROI");
    static_assert(DIST != kCompiler, "the group sums equal the thread kernel's only for a fixed distance rounding");
    extern __shared__ __align__(16) float smem[];
    const int n = queue_len(q);
    const int base = blockIdx.x * SLOTS;
    if (base >= n) return;
    const int cnt = min(SLOTS, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    for (int idx = threadIdx.x; idx < cnt * PIX; idx += kGroupTPB) {
        const int slot = idx / PIX;
        const int k = idx - slot * PIX;
        const int id = queue_at(q, base + slot);
        const uint16_t u = __ldg(rois + (size_t)id * WHOLE + k);
        const float pixval = fmaxf((u - c.Offset) * c.KAdc, 1.0f);
        s_img[slot * PIXP + k] = make_float2(pixval, __logf(pixval));
    }
    __syncthreads();
    const int slot = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    if (slot >= cnt) return;
    const unsigned mask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));

    const int CurFluoID = queue_at(q, base + slot);
    const float2 *img2 = s_img + slot * PIXP;
    float *w = smem + L::W + slot * PIXP;
    float *part = smem + L::PART + slot * PIXP;
    float *D = smem + L::D + threadIdx.x;
    const uint16_t *hdr = rois + (size_t)CurFluoID * WHOLE + PIX;
    const int XOffset = hdr[0];
    const int YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const float *pw = wle + (size_t)CurFluoID * QCS_WLE_PARA_NUM;

    float Ininf[P];
    const SinglePrep sp = single_prefit<R, KIND>(PixView{img2, 1}, pw, c, Ininf);
    if (lane == 0) wle_weights<R, MASK>(w, 1, sp.WLE_SigmaX, sp.WLE_SigmaY, sp.MoleculeType);
    __syncwarp(mask);
    bfgs_fit<P, KindTraits<KIND>::IT>(GroupEval<R, KIND, DIST, G>{img2, w, part, lane, mask}, Ininf, D, kGroupTPB);
    float row[12];
    bool accepted;
    float CurSNR;
    int IsFittingValid;
    single_finish<R, KIND>(Ininf, c, sp.Simga_Max_Th, XOffset, YOffset, CurFrame, row, accepted, CurSNR,
                           IsFittingValid);
    if (lane != 0) return;
    if (accepted)
        store_row(loc, CurFluoID, row);
    else
        zero_row(loc, CurFluoID);
    if (to2e) to2e[CurFluoID] = (!accepted && c.MultiEmitterFitEn && IsFittingValid && (CurSNR > 6.0f)) ? 1 : 0;
}

// ------------------------------------------- learned-start single fits ---
// The single-emitter fit of fit_single_kernel (GS2D or AS3D) started from a
// given point (GS2D: peak e-, x, y in ROI pixels, sigma, background e-; AS3D:
// peak e-, x, y, sigma_x, sigma_y, background e-) instead of the centre /
// edge-mean pre-estimate, with ITERS BFGS iterations of NB line-search steps
// instead of the reference's schedule, and the analytic gradient
// (AnalyticEvalGS2D / AnalyticEvalAS3D) instead of the central difference.
// The same weighted loss, WLE mask, accept rules (the narrower sigma bound
// with multi-emitter fitting on) and output row, over the records of a queue.
// refit[id] = 1 when the fit is not accepted or when its unweighted Poisson
// deviance 2 sum(mu - n - n ln(mu / n)) exceeds dev_th: those ROIs are
// refitted by the plain kernel, which also decides whether a rejected one
// goes on to the two-emitter fit (to2e).
// Layout of fit_single_kernel: the pixels' (value, log) pairs and the mask's
// unique values (the full mask where its rounding is nvcc's per pixel) in
// shared memory, the inverse Hessian in registers.
template <int KIND, int R, int ITERS, int NB, int DIST = ArithSpec<KIND, R>::DIST,
          int MASK = ArithSpec<KIND, R>::MASK, bool FULL = (ArithSpec<KIND, R>::MASK == kCompiler)>
__global__ void __launch_bounds__(kTPB, (SingleLayout<R, FULL>::BLOCKS))
    fit_learned_kernel(const uint16_t *__restrict__ rois, const float *__restrict__ wle,
                       const float *__restrict__ start, Queue q, float *__restrict__ loc,
                       uint8_t *__restrict__ refit, uint8_t *__restrict__ to2e, CorePara c, float dev_th,
                       int direct2e) {
    typedef SingleLayout<R, FULL> L;
    enum { P = KindTraits<KIND>::P, PIX = R * R, WHOLE = R * (R + 1) };
    typedef StagedAnalyticEval<R, KIND, DIST, FULL> Eval;
    extern __shared__ __align__(16) float smem[];
    const int n = queue_len(q);
    const int base = blockIdx.x * kTPB;
    if (base >= n) return;
    const int cnt = min(kTPB, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    stage_rois<R>(s_img, rois, q, base, cnt, c.Offset, c.KAdc);
    __syncthreads();
    const int tid = threadIdx.x;
    if (tid >= cnt) return;
    const int id = queue_at(q, base + tid);
    // the mask: FULL, pixel k at mask[k * kTPB]; else float4 chunk j at ((float4 *)mask)[j * kTPB]
    float *mask = smem + L::WU + (FULL ? tid : 4 * tid);
    const uint16_t *hdr = rois + (size_t)id * WHOLE + PIX;
    const int XOffset = hdr[0], YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const float *pw = wle + (size_t)id * QCS_WLE_PARA_NUM;
    const PixView img{s_img + tid, kTPB};

    float Ininf[P];
    const SinglePrep sp = single_prefit<R, KIND, false>(img, pw, c, Ininf);  // mask widths only
    if constexpr (FULL)
        wle_weights<R, MASK>(mask, kTPB, sp.WLE_SigmaX, sp.WLE_SigmaY, sp.MoleculeType);
    else
        wle_weights_unique<R, MASK>(reinterpret_cast<float4 *>(mask), kTPB, sp.WLE_SigmaX, sp.WLE_SigmaY,
                                    sp.MoleculeType);
    const float *st = start + (size_t)id * P;
    Ininf[0] = st[0] * rAScalFactor;
    Ininf[1] = st[1];
    Ininf[2] = st[2];
    Ininf[3] = (0.5f / (st[3] * st[3])) * rSScalFactor;
    if (KIND == kGS2D) {
        Ininf[4] = st[4] * rBScalFactor;
    } else {
        Ininf[4] = (0.5f / (st[4] * st[4])) * rSScalFactor;
        Ininf[P - 1] = st[5] * rBScalFactor;
    }
    float D[P * P];  // the inverse Hessian, in registers
    bfgs_fit<P, ITERS, Eval, NB>(Eval{{s_img + tid, mask, kTPB}}, Ininf, D, 1);

    float row[12];
    bool accepted;
    float CurSNR;
    int IsFittingValid;
    single_finish<R, KIND>(Ininf, c, sp.Simga_Max_Th, XOffset, YOffset, CurFrame, row, accepted, CurSNR,
                           IsFittingValid);
    // goodness of fit at the final point (unweighted Poisson deviance)
    float dev = 0.0f;
#pragma unroll 1
    for (int r = 0; r < R; r++)
        for (int col = 0; col < R; col++) {
            const float2 pl = s_img[tid + (r * R + col) * kTPB];
            const float e = single_expo<KIND, DIST>(col + 0.5f, r + 0.5f, Ininf);
            dev += single_term<KIND>(e, Ininf, pl.x, pl.y);
        }
    dev *= 2.0f;
    const bool poor = !accepted || !(dev <= dev_th);
    if (direct2e && to2e && poor && IsFittingValid && CurSNR > 6.0f) {
        // a bright ROI the single model does not fit: on to the two-emitter fit
        refit[id] = 0;
        to2e[id] = 1;
        zero_row(loc, id);
        return;
    }
    refit[id] = poor ? 1 : 0;
    if (to2e) to2e[id] = 0;  // a kept fit is final; a refit sets the flag again
    if (accepted)
        store_row(loc, id, row);
    else
        zero_row(loc, id);
}

template <int KIND, int R, int ITERS, int NB>
cudaError_t launch_learned(const FitLaunch &a, const float *start, float dev_th, uint8_t *refit) {
    const size_t smem = SingleLayout<R, ArithSpec<KIND, R>::MASK == kCompiler>::BYTES;
    auto k = fit_learned_kernel<KIND, R, ITERS, NB>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + kTPB - 1) / kTPB;
    if (grid == 0) return cudaSuccess;
    k<<<grid, kTPB, smem, a.stream>>>(a.rois, a.wle, start, a.q, a.loc, refit, a.to2e, a.para, dev_th, a.direct2e);
    return cudaGetLastError();
}

// Ids of the records with a nonzero flag (in no particular order: every
// record is fitted on its own, so the order changes no result) and their
// count; *count must be zero on entry.
__global__ void flag_queue_kernel(const uint8_t *__restrict__ flags, int n, int *__restrict__ ids,
                                  int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int f = (i < n) ? (flags[i] != 0) : 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, f);
    int base = 0;
    if (lane == 0 && ballot) base = atomicAdd(count, __popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (f) ids[base + __popc(ballot & ((1u << lane) - 1u))] = i;
}

// -------------------------------------------------------- multi emitter ---
// Emitter selection, accept rules and output of the multi-emitter fits
// (2Emitter_core.h:245-333, 3Emitter_core.h:247-347, AS3D_2Emitter_core.h:
// 307-406) at the fitted parameters Ininf (fit units): the first emitter's row
// into loc[CurFluoID] (or a zero row), the second's into mo.extra[slot] and the
// stage result (0: none kept, 1: one, 2: both) into mo.result[slot].
template <int R, int KIND>
__device__ __forceinline__ void multi_finish(float *Ininf, const CorePara &c, int XOffset, int YOffset, int CurFrame,
                                             float NearNeighborDistance, float *__restrict__ loc, int CurFluoID,
                                             MultiOut mo, int slot) {
    enum { P = KindTraits<KIND>::P, ROISize_Half = R / 2 };
    const float ROICenter = R / 2.0f;
    const float QE = c.QE;
    // emitter selection (2Emitter_core.h:245-271, 3Emitter_core.h:247-280)
    enum { NE = (KIND == k3E) ? 3 : 2, STRIDE = (KIND == kAS3D2E) ? 5 : 3 };
    float row0[12], row1[12];
    int result = 0;
    if (KIND == kAS3D2E) {
        Ininf[0] = Ininf[0] * QCS_ASCALE / QE;
        Ininf[5] = Ininf[5] * QCS_ASCALE / QE;
        Ininf[3] = sqrtf(0.5f / (Ininf[3] * QCS_SSCALE));
        Ininf[4] = sqrtf(0.5f / (Ininf[4] * QCS_SSCALE));
        Ininf[8] = sqrtf(0.5f / (Ininf[8] * QCS_SSCALE));
        Ininf[9] = sqrtf(0.5f / (Ininf[9] * QCS_SSCALE));
    } else if (KIND == k2E) {
        Ininf[0] = Ininf[0] * QCS_ASCALE / QE;
        Ininf[3] = Ininf[3] * QCS_ASCALE / QE;
    } else {
        Ininf[0] = Ininf[0] * QCS_ASCALE / QE;
        Ininf[3] = Ininf[3] * QCS_ASCALE / QE;
        Ininf[6] = Ininf[6] * QCS_ASCALE / QE;
    }
    const float Background = Ininf[P - 1] * QCS_BSCALE / QE;
    const int IsFittingValid = isnan(Background) ? 0 : 1;
    float Distance[NE];
#pragma unroll
    for (int e = 0; e < NE; e++) {
        const float curPeak = Ininf[STRIDE * e + 0];
        float curx = Ininf[STRIDE * e + 1];
        float cury = Ininf[STRIDE * e + 2];
        if (fabsf(curx - ROICenter) >= ROISize_Half) curx = -100;
        if (fabsf(cury - ROICenter) >= ROISize_Half) cury = -100;
        Distance[e] = sqrtf((curx - ROICenter) * (curx - ROICenter) + (cury - ROICenter) * (cury - ROICenter));
        Distance[e] = curPeak * (R - Distance[e]);
    }
    int MoleculeSel0 = 0, MoleculeSel1 = 0;
#pragma unroll
    for (int e = 0; e < NE; e++)
        if (Distance[e] > Distance[MoleculeSel0]) MoleculeSel0 = e;
    if (NE == 2) {
        MoleculeSel1 = 1 - MoleculeSel0;
    } else {
#pragma unroll
        for (int e = 0; e < NE; e++)
            if (e == MoleculeSel0) Distance[e] = -100;
#pragma unroll
        for (int e = 0; e < NE; e++)
            if (Distance[e] > Distance[MoleculeSel1]) MoleculeSel1 = e;
    }
    // dynamic-index reads through a small switch keep Ininf in registers
    auto get = [&](int i) {
        float v = Ininf[0];
#pragma unroll
        for (int k = 1; k < P; k++)
            if (k == i) v = Ininf[k];
        return v;
    };
    const float PeakPhoton0 = get(STRIDE * MoleculeSel0 + 0);
    const float XPos0_0 = get(STRIDE * MoleculeSel0 + 1);
    const float YPos0_0 = get(STRIDE * MoleculeSel0 + 2);
    const float PeakPhoton1 = get(STRIDE * MoleculeSel1 + 0);
    const float XPos1_0 = get(STRIDE * MoleculeSel1 + 1);
    const float YPos1_0 = get(STRIDE * MoleculeSel1 + 2);
    const float Dist01 = sqrtf((XPos0_0 - XPos1_0) * (XPos0_0 - XPos1_0) + (YPos0_0 - YPos1_0) * (YPos0_0 - YPos1_0));

    if (KIND == kAS3D2E) {
        const float Simga_Max_Th = R / 1.9f / 2.35f;
        const float Simga_Min_Th = 0.8f;
        const float SimgaX0 = get(STRIDE * MoleculeSel0 + 3), SimgaY0 = get(STRIDE * MoleculeSel0 + 4);
        const float SimgaX1 = get(STRIDE * MoleculeSel1 + 3), SimgaY1 = get(STRIDE * MoleculeSel1 + 4);
        const float TotalPhoton0 = PeakPhoton0 * 2 * 3.141593f * SimgaX0 * SimgaY0;
        const float CurSNR0 = sqrtf(QE) * PeakPhoton0 / sqrtf(PeakPhoton0 + Background);
        const float CurZPos0 = zpoly(c, SimgaX0 * SimgaX0 - SimgaY0 * SimgaY0);
        const float MeanSigma0 = (SimgaX0 + SimgaY0) / 2;
        const float TotalPhoton1 = PeakPhoton1 * 2 * 3.141593f * SimgaX1 * SimgaY1;
        const float CurSNR1 = sqrtf(QE) * PeakPhoton1 / sqrtf(PeakPhoton1 + Background);
        const float CurZPos1 = zpoly(c, SimgaX1 * SimgaX1 - SimgaY1 * SimgaY1);
        const float MeanSigma1 = (SimgaX1 + SimgaY1) / 2;
        if (IsFittingValid && (CurSNR0 > 5.5f) && (MeanSigma0 > 0.6f) && (MeanSigma0 > Simga_Min_Th) &&
            (MeanSigma0 <= Simga_Max_Th)) {
            result = 1;
            row0[0] = PeakPhoton0; row0[1] = XPos0_0 - ROISize_Half + XOffset; row0[2] = YPos0_0 - ROISize_Half + YOffset;
            row0[3] = CurZPos0; row0[4] = SimgaX0; row0[5] = SimgaY0; row0[6] = TotalPhoton0; row0[7] = Background;
            row0[8] = CurSNR0; row0[9] = 0.0f; row0[10] = 0.0f; row0[11] = CurFrame;
            if ((Dist01 > 1.5f) && (CurSNR1 > 5.2f) && (NearNeighborDistance > ROICenter) && (MeanSigma1 > 0.6f) &&
                (MeanSigma1 > Simga_Min_Th) && (MeanSigma1 <= Simga_Max_Th) && (PeakPhoton1 > PeakPhoton0 / 3.0f) &&
                (XPos1_0 > 1) && (YPos1_0 > 1) && (XPos1_0 < R - 1) && (YPos1_0 < R - 1)) {
                result = 2;
                row1[0] = PeakPhoton1; row1[1] = XPos1_0 - ROISize_Half + XOffset; row1[2] = YPos1_0 - ROISize_Half + YOffset;
                row1[3] = CurZPos1; row1[4] = SimgaX1; row1[5] = SimgaY1; row1[6] = TotalPhoton1; row1[7] = Background;
                row1[8] = CurSNR1; row1[9] = 0.0f; row1[10] = 0.0f; row1[11] = CurFrame;
            }
        }
    } else {
        const float Simga_Max_Th = R / 2.0f / 2.35f;
        const float SimgaX = sqrtf(0.5f / (Ininf[P - 2] * QCS_SSCALE));
        const float TotalPhoton0 = PeakPhoton0 * 2 * 3.141593f * SimgaX * SimgaX;
        const float CurSNR0 = sqrtf(QE) * PeakPhoton0 / sqrtf(PeakPhoton0 + Background);
        const float TotalPhoton1 = PeakPhoton1 * 2 * 3.141593f * SimgaX * SimgaX;
        const float CurSNR1 = sqrtf(QE) * PeakPhoton1 / sqrtf(PeakPhoton1 + Background);
        if (IsFittingValid && (CurSNR0 > 5.5f) && (SimgaX > 0.6f) && (SimgaX <= Simga_Max_Th)) {
            result = 1;
            row0[0] = PeakPhoton0; row0[1] = XPos0_0 - ROISize_Half + XOffset; row0[2] = YPos0_0 - ROISize_Half + YOffset;
            row0[3] = 0.0f; row0[4] = SimgaX; row0[5] = SimgaX; row0[6] = TotalPhoton0; row0[7] = Background;
            row0[8] = CurSNR0; row0[9] = 0.0f; row0[10] = 0.0f; row0[11] = CurFrame;
            const bool nn_ok = (KIND == k3E) ? (NearNeighborDistance > ROICenter) : (NearNeighborDistance >= ROICenter);
            if ((Dist01 > 1.5f) && (CurSNR1 > 5.2f) && nn_ok && (PeakPhoton1 > PeakPhoton0 / 2.0f) && (XPos1_0 > 1) &&
                (YPos1_0 > 1) && (XPos1_0 < R - 1) && (YPos1_0 < R - 1)) {
                result = 2;
                row1[0] = PeakPhoton1; row1[1] = XPos1_0 - ROISize_Half + XOffset; row1[2] = YPos1_0 - ROISize_Half + YOffset;
                row1[3] = 0.0f; row1[4] = SimgaX; row1[5] = SimgaX; row1[6] = TotalPhoton1; row1[7] = Background;
                row1[8] = CurSNR1; row1[9] = 0.0f; row1[10] = 0.0f; row1[11] = CurFrame;
            }
        }
    }
    if (result >= 1)
        store_row(loc, CurFluoID, row0);
    else
        zero_row(loc, CurFluoID);
    if (result == 2) store_row(mo.extra, slot, row1);
    mo.result[slot] = (int8_t)result;
}

// Start point of a multi-emitter fit (PreEstimation_GS2D_2E, _3E and
// PreEstimation_AS3D_2E: 2Emitter_core.h:596-698, 3Emitter_core.h:593-710,
// AS3D_2Emitter_core.h:648-750) from the ROI's pixels, and the weighted-MLE
// mask width of the 2E fit (a fixed R / 1.8 / 2.35, or R without WLE; the
// other kinds are unweighted).
template <int R, int KIND>
__device__ __forceinline__ void multi_prefit(const PixView &img, const CorePara &c, float *Ininf, float &WLE_SigmaX) {
    enum { ROISize_Half = R / 2 };
    const float ROICenter = R / 2.0f;
    WLE_SigmaX = R;
    if (KIND == k2E) {
        WLE_SigmaX = R / 1.8f / 2.35f;
        float Mean1, Mean2, Mean3, Mean4;
        edge_means<R>(img, Mean1, Mean2, Mean3, Mean4);
        Mean1 = fminf(Mean1, Mean2);
        Mean3 = fminf(Mean3, Mean4);
        Mean1 = fminf(Mean1, Mean3);
        const float Bkg = Mean1 / R;
        const float Amp = img[ROISize_Half * R + ROISize_Half] - Bkg;
        const float SigmaX = R / 2.2f / 2.35f;
        const float SigmaX1 = (1.0f / (2.0f * SigmaX * SigmaX));
        float xs[1], ys[1];
        block_starts<R>(img, 1, xs, ys);
        Ininf[0] = 0.8f * Amp * rAScalFactor;
        Ininf[1] = ROICenter;
        Ininf[2] = ROICenter;
        Ininf[3] = 0.8f * Amp * rAScalFactor;
        Ininf[4] = xs[0];
        Ininf[5] = ys[0];
        Ininf[6] = SigmaX1 * rSScalFactor;
        Ininf[7] = 0.8f * Bkg * rBScalFactor;
        if (c.WLEEn == 0) WLE_SigmaX = R;
    } else if (KIND == k3E) {
        float Mean1, Mean2, Mean3, Mean4;
        edge_means<R>(img, Mean1, Mean2, Mean3, Mean4);
        Mean1 = fminf(Mean1, Mean2);
        Mean3 = fminf(Mean3, Mean4);
        const float Bkg = (Mean1 + Mean3) / 2 / R;
        const float Amp = img[ROISize_Half * R + ROISize_Half] - Bkg;
        const float SigmaX = R / 2.2f / 2.35f;
        const float SigmaX1 = (1.0f / (2.0f * SigmaX * SigmaX));
        float xs[2], ys[2];
        block_starts<R>(img, 2, xs, ys);
        Ininf[0] = 0.7f * Amp * rAScalFactor;
        Ininf[1] = ROICenter;
        Ininf[2] = ROICenter;
        Ininf[3] = 0.7f * Amp * rAScalFactor;
        Ininf[4] = xs[0];
        Ininf[5] = ys[0];
        Ininf[6] = 0.3f * Amp * rAScalFactor;
        Ininf[7] = xs[1];
        Ininf[8] = ys[1];
        Ininf[9] = SigmaX1 * rSScalFactor;
        Ininf[10] = 0.8f * Bkg * rBScalFactor;
    } else {  // kAS3D2E
        float Mean1, Mean2, Mean3, Mean4;
        edge_means<R>(img, Mean1, Mean2, Mean3, Mean4);
        Mean1 = fminf(Mean1, Mean2);
        Mean3 = fminf(Mean3, Mean4);
        const float Bkg = (Mean1 + Mean3) / 2 / R;
        const float Amp = img[ROISize_Half * R + ROISize_Half] - Bkg;
        const float SigmaX = R / 2.2f / 2.35f;
        const float SigmaY = R / 2.2f / 2.35f;
        const float SigmaX1 = rSScalFactor * (0.5f / (SigmaX * SigmaX));
        const float SigmaY1 = rSScalFactor * (0.5f / (SigmaY * SigmaY));
        float xs[1], ys[1];
        block_starts<R>(img, 1, xs, ys);
        Ininf[0] = 0.7f * Amp * rAScalFactor;
        Ininf[1] = ROICenter;
        Ininf[2] = ROICenter;
        Ininf[3] = SigmaX1;
        Ininf[4] = SigmaY1;
        Ininf[5] = 0.7f * Amp * rAScalFactor;
        Ininf[6] = xs[0];
        Ininf[7] = ys[0];
        Ininf[8] = SigmaX1;
        Ininf[9] = SigmaY1;
        Ininf[10] = 0.8f * Bkg * rBScalFactor;
    }
}

template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST, int MASK = ArithSpec<KIND, R>::MASK,
          int SUM2 = ArithSpec<KIND, R>::SUM2>
__global__ void __launch_bounds__(kTPB) fit_multi_kernel(const uint16_t *__restrict__ rois,
                                                         const float *__restrict__ wle, Queue q,
                                                         float *__restrict__ loc, MultiOut mo, CorePara c,
                                                         double *__restrict__ ll, int min_n) {
    typedef SmemLayout<R, KIND> L;
    enum { P = KindTraits<KIND>::P, PIX = R * R, WHOLE = R * (R + 1) };
    extern __shared__ float smem[];
    const int n = queue_len(q);
    if (n <= min_n) return;  // a queue this short is the lane-group kernel's
    const int base = blockIdx.x * kTPB;
    if (base >= n) return;
    const int cnt = min(kTPB, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    stage_rois<R>(s_img, rois, q, base, cnt, c.Offset, c.KAdc);
    __syncthreads();
    const int tid = threadIdx.x;
    if (tid >= cnt) return;

    const int slot = base + tid;
    const int CurFluoID = queue_at(q, slot);
    const PixView img{s_img + tid, kTPB};
    float *w = smem + L::W + tid;
    float *D = smem + L::D + tid;
    const uint16_t *hdr = rois + (size_t)CurFluoID * WHOLE + PIX;
    const int XOffset = hdr[0];
    const int YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];

    float Ininf[P];
    const RoiRef roi{s_img + tid, w, kTPB};
    // the 2E fit's selection reads the nearest-neighbour distance of the WLE pre-pass
    const float NearNeighborDistance = KIND == k2E ? wle[(size_t)CurFluoID * QCS_WLE_PARA_NUM + 0] : 1000.0f;
    float WLE_SigmaX;
    multi_prefit<R, KIND>(img, c, Ininf, WLE_SigmaX);
    if (KIND == k2E) wle_weights<R, MASK>(w, kTPB, WLE_SigmaX, WLE_SigmaX, QCS_MOLECULE_MULTIFIT);
    mle_fit<R, KIND, DIST, SUM2>(roi, Ininf, D, kTPB);
    if (ll) ll[CurFluoID] = model_loglik<R, KIND, DIST, SUM2>(s_img + tid, kTPB, Ininf, 0, 1);
    if (KIND == k3E && mo.params) {
#pragma unroll
        for (int k = 0; k < P; k++) mo.params[(size_t)slot * P + k] = Ininf[k];
    }

    multi_finish<R, KIND>(Ininf, c, XOffset, YOffset, CurFrame, NearNeighborDistance, loc, CurFluoID, mo, slot);
}

// The multi-emitter fit of fit_multi_kernel with G lanes per ROI
// (MultiGroupEval): bit for bit the same rows, stage results and second
// emitters.  The thread kernel runs a stage's queue with one thread per ROI at
// ~255 registers (two warps per SM), so a queue shorter than a wave (the
// usual 2E / 3E queue) takes as long as one thread's whole fit; here a ROI's
// pixel terms and gradient points are spread over G lanes.  Per slot: the
// ROI's (value, log) pairs, its mask and loss terms contiguous (rows padded to
// 4 floats), and one inverse Hessian with its update scratch and the search
// direction, which the group's first lane alone updates (bfgs_fit_shared).
template <int R, int KIND>
struct MultiGroupLayout {
    enum {
        P = KindTraits<KIND>::P,
        PIX = R * R,
        PIXP = (PIX + 3) / 4 * 4,
        HP = (2 * P * P + P + 3) / 4 * 4,  // D, T and the direction per slot
        SLOTS = kGroupTPB / multi_lanes(KIND),
        IMG = 0,                       // float2 per pixel
        W = IMG + 2 * PIXP * SLOTS,    // floats
        PART = W + PIXP * SLOTS,
        H = PART + PIXP * SLOTS,
        TOTAL = H + HP * SLOTS,
    };
};

// The shared inverse Hessian's last update: nvcc fuses the separately
// computed s s'/(y's) product of bfgs_update into the final sum (found by
// building both forms against the reference's multi-emitter cascades: only
// the fused one gives their rows bit for bit).
constexpr bool kSkskFused = true;

template <int R, int KIND, int DIST = ArithSpec<KIND, R>::DIST, int MASK = ArithSpec<KIND, R>::MASK,
          int SUM2 = ArithSpec<KIND, R>::SUM2>
__global__ void __launch_bounds__(kGroupTPB, 4) fit_multi_group_kernel(const uint16_t *__restrict__ rois,
                                                                    const float *__restrict__ wle, Queue q,
                                                                    float *__restrict__ loc, MultiOut mo,
                                                                    CorePara c, double *__restrict__ ll, int max_n) {
    typedef MultiGroupLayout<R, KIND> L;
    enum { G = multi_lanes(KIND), P = KindTraits<KIND>::P, PIX = R * R, PIXP = L::PIXP, WHOLE = R * (R + 1),
           SLOTS = L::SLOTS };
    static_assert(DIST != kCompiler && SUM2 != kCompiler, "the group sums equal the thread kernel's only for "
                                                          "roundings fixed in the source");
    extern __shared__ __align__(16) float smem[];
    const int n = queue_len(q);
    if (n > max_n) return;  // a longer queue is the one-thread-per-ROI kernel's
    const int base = blockIdx.x * SLOTS;
    if (base >= n) return;
    const int cnt = min(SLOTS, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    for (int idx = threadIdx.x; idx < cnt * PIX; idx += kGroupTPB) {
        const int sl = idx / PIX;
        const int k = idx - sl * PIX;
        const int id = queue_at(q, base + sl);
        const uint16_t u = __ldg(rois + (size_t)id * WHOLE + k);
        const float pixval = fmaxf((u - c.Offset) * c.KAdc, 1.0f);
        s_img[sl * PIXP + k] = make_float2(pixval, __logf(pixval));
    }
    __syncthreads();
    const int sl = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    if (sl >= cnt) return;
    const unsigned mask = G == 32 ? 0xffffffffu : ((1u << (G % 32)) - 1u) << ((threadIdx.x & 31) & ~(G - 1));

    const int slot = base + sl;
    const int CurFluoID = queue_at(q, slot);
    const float2 *img2 = s_img + sl * PIXP;
    float *w = smem + L::W + sl * PIXP;
    float *part = smem + L::PART + sl * PIXP;
    float *hess = smem + L::H + sl * L::HP;  // D (P x P), T (P x P), direction (P)
    const uint16_t *hdr = rois + (size_t)CurFluoID * WHOLE + PIX;
    const int XOffset = hdr[0];
    const int YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const float NearNeighborDistance = KIND == k2E ? wle[(size_t)CurFluoID * QCS_WLE_PARA_NUM + 0] : 1000.0f;

    float Ininf[P];
    float WLE_SigmaX;
    multi_prefit<R, KIND>(PixView{img2, 1}, c, Ininf, WLE_SigmaX);
    if (KIND == k2E && lane == 0) wle_weights<R, MASK>(w, 1, WLE_SigmaX, WLE_SigmaX, QCS_MOLECULE_MULTIFIT);
    __syncwarp(mask);
    bfgs_fit_shared<P, KindTraits<KIND>::IT, MultiGroupEval<R, KIND, DIST, SUM2, G>, kSkskFused>(
        MultiGroupEval<R, KIND, DIST, SUM2, G>{img2, w, part, lane, mask}, Ininf, hess, hess + P * P,
        hess + 2 * P * P, lane, mask);
    if (ll) {  // the lanes' pixel sums, combined in a fixed order
        double s = model_loglik<R, KIND, DIST, SUM2>(img2, 1, Ininf, lane, G);
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(mask, s, o, G);
        if (lane == 0) ll[CurFluoID] = s;
    }
    if (KIND == k3E && mo.params && lane == 0) {
#pragma unroll
        for (int k = 0; k < P; k++) mo.params[(size_t)slot * P + k] = Ininf[k];
    }
    if (lane == 0)
        multi_finish<R, KIND>(Ininf, c, XOffset, YOffset, CurFrame, NearNeighborDistance, loc, CurFluoID, mo, slot);
}

// -------------------------------------- learned-start two-emitter fits ---
// The GS2D two-emitter fit of fit_multi_kernel<R, k2E> over the records of
// its queue, started from a given point (start[8 id ..]: peak e- of emitter
// 0, its x, y in ROI pixels, peak e- of emitter 1, its x, y, the shared sigma,
// background e-) instead of the centre / 3x3-block pre-estimate, with ITERS
// BFGS iterations of NB line-search steps and the analytic gradient
// (AnalyticEval2E); the same weighted loss (fixed-width WLE mask), selection,
// accept rules and output (multi_finish). A fit is judged poor when no
// emitter is kept or when the unweighted Poisson deviance of the two-emitter
// model exceeds dev_th; with to3e = 0, refit[slot] = 1 marks it for the plain
// two-emitter fit, with to3e = 1 its rows are dropped and its stage result set
// to 0, so the cascade hands it to the three-emitter fit as it hands on the
// reference fit's rejects.
template <int R, int ITERS, int NB, int DIST = ArithSpec<k2E, R>::DIST, int MASK = ArithSpec<k2E, R>::MASK>
__global__ void __launch_bounds__(kTPB) fit_learned_2e_kernel(const uint16_t *__restrict__ rois,
                                                              const float *__restrict__ wle,
                                                              const float *__restrict__ start, Queue q,
                                                              float *__restrict__ loc, MultiOut mo,
                                                              uint8_t *__restrict__ refit, CorePara c, float dev_th,
                                                              int to3e) {
    typedef SmemLayout<R, k2E> L;
    enum { P = 8, PIX = R * R, WHOLE = R * (R + 1) };
    extern __shared__ float smem[];
    const int n = queue_len(q);
    const int base = blockIdx.x * kTPB;
    if (base >= n) return;
    const int cnt = min(kTPB, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    stage_rois<R>(s_img, rois, q, base, cnt, c.Offset, c.KAdc);
    __syncthreads();
    const int tid = threadIdx.x;
    if (tid >= cnt) return;
    const int slot = base + tid;
    const int id = queue_at(q, slot);
    float *w = smem + L::W + tid;
    float *D = smem + L::D + tid;
    const uint16_t *hdr = rois + (size_t)id * WHOLE + PIX;
    const int XOffset = hdr[0], YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const RoiRef roi{s_img + tid, w, kTPB};
    const float NearNeighborDistance = wle[(size_t)id * QCS_WLE_PARA_NUM + 0];
    float WLE_SigmaX = R / 1.8f / 2.35f;
    if (c.WLEEn == 0) WLE_SigmaX = R;
    wle_weights<R, MASK>(w, kTPB, WLE_SigmaX, WLE_SigmaX, QCS_MOLECULE_MULTIFIT);
    const float *st = start + (size_t)id * P;
    float Ininf[P];
    Ininf[0] = st[0] * rAScalFactor;
    Ininf[1] = st[1];
    Ininf[2] = st[2];
    Ininf[3] = st[3] * rAScalFactor;
    Ininf[4] = st[4];
    Ininf[5] = st[5];
    Ininf[6] = (0.5f / (st[6] * st[6])) * rSScalFactor;
    Ininf[7] = st[7] * rBScalFactor;
    bfgs_fit<P, ITERS, AnalyticEval2E<R, DIST>, NB>(AnalyticEval2E<R, DIST>{roi}, Ininf, D, kTPB);
    // goodness of fit at the final point (unweighted Poisson deviance of the two-emitter model)
    float dev = 0.0f;
    {
        float v[P];
#pragma unroll
        for (int k = 0; k < P; k++) v[k] = Ininf[k] < 0.0f ? 0.0f : Ininf[k];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE, S01 = v[6] * QCS_SSCALE, B64 = v[7] * QCS_BSCALE;
#pragma unroll 1
        for (int r = 0; r < R; r++)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(r * R + col) * roi.ld];
                const float dx0 = col + 0.5f - v[1], dy0 = r + 0.5f - v[2];
                const float dx1 = col + 0.5f - v[4], dy1 = r + 0.5f - v[5];
                const float mu = A0 * __expf(-(dx0 * dx0 + dy0 * dy0) * S01) +
                                 A1 * __expf(-(dx1 * dx1 + dy1 * dy1) * S01) + B64;
                dev += mu - pl.x - pl.x * (__logf(mu) - pl.y);
            }
        dev *= 2.0f;
    }
    multi_finish<R, k2E>(Ininf, c, XOffset, YOffset, CurFrame, NearNeighborDistance, loc, id, mo, slot);
    const bool poor = mo.result[slot] == 0 || !(dev <= dev_th);
    if (to3e) {
        if (poor && mo.result[slot] != 0) {
            zero_row(loc, id);
            mo.result[slot] = 0;
        }
        refit[slot] = 0;
    } else {
        refit[slot] = poor ? 1 : 0;
    }
}

// ------------------------------------ learned-start three-emitter fits ---
// The GS2D three-emitter fit of fit_multi_kernel<R, k3E> over the records of
// its queue, started from a given point (start[11 id ..]: peak e-, x, y in
// ROI pixels of emitters 0, 1, 2, the shared sigma, background e-) instead of
// the reference's pre-estimate (bfgsMLE_GS2D_3Emitter_core.h:593-710), with
// ITERS BFGS iterations of NB line-search steps and the analytic gradient
// (AnalyticEval3E); the same loss, selection of the two kept emitters, accept
// rules and output (multi_finish). A fit is judged poor when no emitter is
// kept or when its unweighted Poisson deviance exceeds dev_th: refit[slot] = 1
// marks it for the plain three-emitter fit.
template <int R, int ITERS, int NB, int DIST = ArithSpec<k3E, R>::DIST>
__global__ void __launch_bounds__(kTPB) fit_learned_3e_kernel(const uint16_t *__restrict__ rois,
                                                              const float *__restrict__ start, Queue q,
                                                              float *__restrict__ loc, MultiOut mo,
                                                              uint8_t *__restrict__ refit, CorePara c, float dev_th,
                                                              int min_n) {
    typedef SmemLayout<R, k3E> L;
    enum { P = 11, PIX = R * R, WHOLE = R * (R + 1) };
    extern __shared__ float smem[];
    const int n = queue_len(q);
    if (n <= min_n) return;  // a queue this short is the one-warp-per-ROI kernel's
    const int base = blockIdx.x * kTPB;
    if (base >= n) return;
    const int cnt = min(kTPB, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    stage_rois<R>(s_img, rois, q, base, cnt, c.Offset, c.KAdc);
    __syncthreads();
    const int tid = threadIdx.x;
    if (tid >= cnt) return;
    const int slot = base + tid;
    const int id = queue_at(q, slot);
    float *D = smem + L::D + tid;
    const uint16_t *hdr = rois + (size_t)id * WHOLE + PIX;
    const int XOffset = hdr[0], YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const RoiRef roi{s_img + tid, nullptr, kTPB};  // the three-emitter loss is unweighted
    const float *st = start + (size_t)id * P;
    float Ininf[P];
#pragma unroll
    for (int e = 0; e < 3; e++) {
        Ininf[3 * e] = st[3 * e] * rAScalFactor;
        Ininf[3 * e + 1] = st[3 * e + 1];
        Ininf[3 * e + 2] = st[3 * e + 2];
    }
    Ininf[9] = (0.5f / (st[9] * st[9])) * rSScalFactor;
    Ininf[10] = st[10] * rBScalFactor;
    bfgs_fit<P, ITERS, AnalyticEval3E<R, DIST>, NB>(AnalyticEval3E<R, DIST>{roi}, Ininf, D, kTPB);
    // goodness of fit at the final point (unweighted Poisson deviance of the three-emitter model)
    float dev = 0.0f;
    {
        float v[P];
#pragma unroll
        for (int k = 0; k < P; k++) v[k] = Ininf[k] < 0.0f ? 0.0f : Ininf[k];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE, A2 = v[6] * QCS_ASCALE;
        const float S = v[9] * QCS_SSCALE, B64 = v[10] * QCS_BSCALE;
#pragma unroll 1
        for (int r = 0; r < R; r++)
            for (int col = 0; col < R; col++) {
                const float2 pl = roi.img[(r * R + col) * roi.ld];
                const float dx0 = col + 0.5f - v[1], dy0 = r + 0.5f - v[2];
                const float dx1 = col + 0.5f - v[4], dy1 = r + 0.5f - v[5];
                const float dx2 = col + 0.5f - v[7], dy2 = r + 0.5f - v[8];
                const float mu = A0 * __expf(-(dx0 * dx0 + dy0 * dy0) * S) + A1 * __expf(-(dx1 * dx1 + dy1 * dy1) * S) +
                                 A2 * __expf(-(dx2 * dx2 + dy2 * dy2) * S) + B64;
                dev += mu - pl.x - pl.x * (__logf(mu) - pl.y);
            }
        dev *= 2.0f;
    }
    multi_finish<R, k3E>(Ininf, c, XOffset, YOffset, CurFrame, 1000.0f, loc, id, mo, slot);
    refit[slot] = (mo.result[slot] == 0 || !(dev <= dev_th)) ? 1 : 0;
}

// The same fit with one warp per ROI (AnalyticWarpEval3E: the pixels spread
// over the lanes, one shared inverse Hessian per ROI updated by lane 0,
// bfgs_fit_shared) for queues of at most max_n records, where one ROI's
// latency, not throughput, sets the stage's time.
template <int R, int ITERS, int NB>
__global__ void __launch_bounds__(kGroupTPB) fit_learned_3e_warp_kernel(const uint16_t *__restrict__ rois,
                                                                       const float *__restrict__ start, Queue q,
                                                                       float *__restrict__ loc, MultiOut mo,
                                                                       uint8_t *__restrict__ refit, CorePara c,
                                                                       float dev_th, int max_n) {
    typedef MultiGroupLayout<R, k3E> L;
    enum { P = 11, PIX = R * R, PIXP = L::PIXP, WHOLE = R * (R + 1), SLOTS = kGroupTPB / 32 };
    static_assert(L::SLOTS == SLOTS, "one warp per slot");
    extern __shared__ __align__(16) float smem[];
    const int n = queue_len(q);
    if (n > max_n) return;  // a longer queue is the one-thread-per-ROI kernel's
    const int base = blockIdx.x * SLOTS;
    if (base >= n) return;
    const int cnt = min((int)SLOTS, n - base);
    float2 *s_img = reinterpret_cast<float2 *>(smem + L::IMG);
    for (int idx = threadIdx.x; idx < cnt * PIX; idx += kGroupTPB) {
        const int sl = idx / PIX;
        const int k = idx - sl * PIX;
        const int id = queue_at(q, base + sl);
        const uint16_t u = __ldg(rois + (size_t)id * WHOLE + k);
        const float pixval = fmaxf((u - c.Offset) * c.KAdc, 1.0f);
        s_img[sl * PIXP + k] = make_float2(pixval, __logf(pixval));
    }
    __syncthreads();
    const int sl = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (sl >= cnt) return;
    const unsigned mask = 0xffffffffu;
    const int slot = base + sl;
    const int id = queue_at(q, slot);
    const float2 *img2 = s_img + sl * PIXP;
    float *hess = smem + L::H + sl * L::HP;  // D (P x P), T (P x P), direction (P)
    const uint16_t *hdr = rois + (size_t)id * WHOLE + PIX;
    const int XOffset = hdr[0], YOffset = hdr[1];
    const int CurFrame = hdr[2] + 65536 * hdr[3];
    const float *st = start + (size_t)id * P;
    float Ininf[P];
#pragma unroll
    for (int e = 0; e < 3; e++) {
        Ininf[3 * e] = st[3 * e] * rAScalFactor;
        Ininf[3 * e + 1] = st[3 * e + 1];
        Ininf[3 * e + 2] = st[3 * e + 2];
    }
    Ininf[9] = (0.5f / (st[9] * st[9])) * rSScalFactor;
    Ininf[10] = st[10] * rBScalFactor;
    const AnalyticWarpEval3E<R> ev{img2, lane, mask};
    bfgs_fit_shared<P, ITERS, AnalyticWarpEval3E<R>, kSkskFused, NB>(ev, Ininf, hess, hess + P * P, hess + 2 * P * P,
                                                                     lane, mask);
    // goodness of fit at the final point (unweighted Poisson deviance of the three-emitter model)
    float dev;
    {
        float v[P];
#pragma unroll
        for (int k = 0; k < P; k++) v[k] = Ininf[k] < 0.0f ? 0.0f : Ininf[k];
        const float A0 = v[0] * QCS_ASCALE, A1 = v[3] * QCS_ASCALE, A2 = v[6] * QCS_ASCALE;
        const float S = v[9] * QCS_SSCALE, B64 = v[10] * QCS_BSCALE;
        float part = 0.0f;
        for (int k = lane; k < PIX; k += 32) {
            const int r = k / R, col = k - r * R;
            const float2 pl = img2[k];
            const float dx0 = col + 0.5f - v[1], dy0 = r + 0.5f - v[2];
            const float dx1 = col + 0.5f - v[4], dy1 = r + 0.5f - v[5];
            const float dx2 = col + 0.5f - v[7], dy2 = r + 0.5f - v[8];
            const float mu = A0 * __expf(-(dx0 * dx0 + dy0 * dy0) * S) + A1 * __expf(-(dx1 * dx1 + dy1 * dy1) * S) +
                             A2 * __expf(-(dx2 * dx2 + dy2 * dy2) * S) + B64;
            part += mu - pl.x - pl.x * (__logf(mu) - pl.y);
        }
        dev = 2.0f * ev.uniform_sum(part);
    }
    if (lane == 0) {
        multi_finish<R, k3E>(Ininf, c, XOffset, YOffset, CurFrame, 1000.0f, loc, id, mo, slot);
        refit[slot] = (mo.result[slot] == 0 || !(dev <= dev_th)) ? 1 : 0;
    }
}

// slots[] / ids[]: the queue slots i < *n_dev with flags[i] != 0 and their
// record ids q[i] (any order); *count = their number (zero on entry).
__global__ void flag_slots_kernel(const uint8_t *__restrict__ flags, const int *__restrict__ n_dev, int max_n,
                                  const int *__restrict__ q, int *__restrict__ slots, int *__restrict__ ids,
                                  int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = min(*n_dev, max_n);
    const bool f = i < n && flags[i] != 0;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    int b = 0;
    if ((threadIdx.x & 31) == 0 && m) b = atomicAdd(count, __popc(m));
    b = __shfl_sync(0xffffffffu, b, 0);
    if (f) {
        const int k = b + __popc(m & ((1u << (threadIdx.x & 31)) - 1u));
        slots[k] = i;
        ids[k] = q[i];
    }
}

// The plain refits' stage results and second-emitter rows (indexed by refit
// position k) back into the slots they were taken from.
__global__ void merge_refit_kernel(const int *__restrict__ slots, const int *__restrict__ count, int max_n,
                                   const int8_t *__restrict__ res_k, const float *__restrict__ extra_k,
                                   int8_t *__restrict__ res, float *__restrict__ extra) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= min(*count, max_n)) return;
    const int slot = slots[k];
    res[slot] = res_k[k];
    if (res_k[k] == 2) {
#pragma unroll
        for (int j = 0; j < 12; j++) extra[(size_t)slot * 12 + j] = extra_k[(size_t)k * 12 + j];
    }
}

template <int R, int IT, int NB>
cudaError_t launch_learned_2e(const FitLaunch &a, const float *start, float dev_th, uint8_t *refit, int to3e) {
    const size_t smem = SmemLayout<R, k2E>::TOTAL * sizeof(float);
    auto k = fit_learned_2e_kernel<R, IT, NB>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + kTPB - 1) / kTPB;
    if (grid == 0) return cudaSuccess;
    k<<<grid, kTPB, smem, a.stream>>>(a.rois, a.wle, start, a.q, a.loc, a.mo, refit, a.para, dev_th, to3e);
    return cudaGetLastError();
}

// Learned-start three-emitter queues up to this length run one warp per ROI.
constexpr int kLearned3EWarpLimit = 4096;

// Both kernels are launched; each reads the stage's queue length on the
// device and only one of them fits it.
template <int R, int IT, int NB>
cudaError_t launch_learned_3e(const FitLaunch &a, const float *start, float dev_th, uint8_t *refit) {
    if (a.max_count <= 0) return cudaSuccess;
    {
        typedef MultiGroupLayout<R, k3E> L;
        const size_t smem = L::TOTAL * sizeof(float);
        auto k = fit_learned_3e_warp_kernel<R, IT, NB>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int m = a.max_count < kLearned3EWarpLimit ? a.max_count : kLearned3EWarpLimit;
        k<<<(m + L::SLOTS - 1) / L::SLOTS, kGroupTPB, smem, a.stream>>>(a.rois, start, a.q, a.loc, a.mo, refit,
                                                                        a.para, dev_th, kLearned3EWarpLimit);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (a.max_count <= kLearned3EWarpLimit) return cudaSuccess;
    const size_t smem = SmemLayout<R, k3E>::TOTAL * sizeof(float);
    auto k = fit_learned_3e_kernel<R, IT, NB>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + kTPB - 1) / kTPB;
    k<<<grid, kTPB, smem, a.stream>>>(a.rois, start, a.q, a.loc, a.mo, refit, a.para, dev_th, kLearned3EWarpLimit);
    return cudaGetLastError();
}

template <int R, int KIND>
cudaError_t launch_single(const FitLaunch &a) {
    const size_t smem = SingleLayout<R, ArithSpec<KIND, R>::MASK == kCompiler>::BYTES;
    // two pixels per load when every record starts on a 4-byte boundary
    auto k = (reinterpret_cast<uintptr_t>(a.rois) & 3) == 0 ? fit_single_kernel<R, KIND, true>
                                                             : fit_single_kernel<R, KIND, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + kTPB - 1) / kTPB;
    if (grid == 0) return cudaSuccess;
    k<<<grid, kTPB, smem, a.stream>>>(a.rois, a.wle, a.q, a.loc, a.to2e, a.para, a.ll);
    return cudaGetLastError();
}

template <int R, int KIND, int G>
cudaError_t launch_single_group(const FitLaunch &a) {
    typedef typename GroupLayout<R, KIND>::template At<G> L;
    const size_t smem = L::TOTAL * sizeof(float);
    auto k = fit_single_group_kernel<R, KIND, G>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + L::SLOTS - 1) / L::SLOTS;
    if (grid == 0) return cudaSuccess;
    k<<<grid, kGroupTPB, smem, a.stream>>>(a.rois, a.wle, a.q, a.loc, a.to2e, a.para);
    return cudaGetLastError();
}

// Queue lengths up to which the lane-group kernel fits a multi-emitter stage:
// about three waves of the ROIs it holds at once.  Beyond that the lanes'
// repeated pixel sums cost more than the latency they save, and the
// one-thread-per-ROI kernel (whose single wave holds far more ROIs) is faster.
template <int R, int KIND>
int group_queue_limit() {
    static int limit = -2;
    if (limit == -2) {
        typedef MultiGroupLayout<R, KIND> L;
        int dev = 0, sms = 0, blocks = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(fit_multi_group_kernel<R, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(L::TOTAL * sizeof(float)));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fit_multi_group_kernel<R, KIND>, kGroupTPB,
                                                      L::TOTAL * sizeof(float));
        limit = 3 * sms * (blocks > 0 ? blocks : 1) * L::SLOTS;
    }
    return limit;
}

}  // namespace

int multi_group_default_limit(int kind, int R) {
    if (kind == k2E && R == 7) return group_queue_limit<7, k2E>();
    if (kind == k2E && R == 11) return group_queue_limit<11, k2E>();
    if (kind == k3E && R == 7) return group_queue_limit<7, k3E>();
    if (kind == k3E && R == 11) return group_queue_limit<11, k3E>();
    if (kind == kAS3D2E && R == 7) return group_queue_limit<7, kAS3D2E>();
    return 0;
}

bool multi_group_available(int kind, int R) { return multi_group_supported(kind, R); }

namespace {

// Both kernels are launched; each reads the stage's queue length on the
// device and only one of them fits it (no host synchronisation).
template <int R, int KIND>
cudaError_t launch_multi(const FitLaunch &a) {
    int min_n = -1;
    if constexpr (multi_group_supported(KIND, R)) {
        if (!a.thread_per_roi) {
            typedef MultiGroupLayout<R, KIND> L;
            const size_t smem = L::TOTAL * sizeof(float);
            auto k = fit_multi_group_kernel<R, KIND>;
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            // group_limit > 0: tuned; < 0: one thread per ROI always; 0: the default
            min_n = a.group_limit > 0 ? a.group_limit : (a.group_limit < 0 ? -1 : group_queue_limit<R, KIND>());
            const int grid = (min(a.max_count, min_n) + L::SLOTS - 1) / L::SLOTS;
            if (grid > 0) {
                k<<<grid, kGroupTPB, smem, a.stream>>>(a.rois, a.wle, a.q, a.loc, a.mo, a.para, a.ll, min_n);
                if ((e = cudaGetLastError()) != cudaSuccess) return e;
            }
            if (a.max_count <= min_n) return cudaSuccess;  // the queue cannot outgrow the group kernel
        }
    }
    const size_t smem = SmemLayout<R, KIND>::TOTAL * sizeof(float);
    auto k = fit_multi_kernel<R, KIND>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.max_count + kTPB - 1) / kTPB;
    if (grid == 0) return cudaSuccess;
    k<<<grid, kTPB, smem, a.stream>>>(a.rois, a.wle, a.q, a.loc, a.mo, a.para, a.ll, min_n);
    return cudaGetLastError();
}

}  // namespace

// Schedules compiled per shape: every shape 2..4 iterations of 6 steps and
// 3 of 11; GS2D 7x7 (the bench's shape) also 2..5 or 8 iterations of 11
// steps and 2 or 3 of 4 or 8.
bool learned_schedule_supported(int kind, int R, int iters, int bisections) {
    if (kind == kGS2D && R == 7)
        return (bisections == kBisections && ((iters >= 2 && iters <= 5) || iters == 8)) ||
               ((iters == 2 || iters == 3) && (bisections == 4 || bisections == 8)) ||
               (bisections == 6 && iters >= 2 && iters <= 4);
    if ((kind == kGS2D || kind == kAS3D) && (R == 7 || R == 9 || R == 11))
        return (bisections == 6 && iters >= 2 && iters <= 4) || (bisections == kBisections && iters == 3);
    return false;
}

template <int KIND, int R>
cudaError_t launch_learned_shape(int iters, int bisections, const FitLaunch &a, const float *start, float dev_th,
                                 uint8_t *refit) {
#define QCS_LEARNED(IT, NB) \
    if (iters == IT && bisections == NB) return launch_learned<KIND, R, IT, NB>(a, start, dev_th, refit);
    QCS_LEARNED(2, 6)
    QCS_LEARNED(3, 6)
    QCS_LEARNED(4, 6)
    QCS_LEARNED(3, kBisections)
    if constexpr (KIND == kGS2D && R == 7) {
        QCS_LEARNED(2, kBisections)
        QCS_LEARNED(4, kBisections)
        QCS_LEARNED(5, kBisections)
        QCS_LEARNED(8, kBisections)
        QCS_LEARNED(2, 4)
        QCS_LEARNED(2, 8)
        QCS_LEARNED(3, 4)
        QCS_LEARNED(3, 8)
    }
#undef QCS_LEARNED
    return cudaErrorInvalidValue;
}

cudaError_t launch_fit_learned(int kind, int R, int iters, int bisections, const FitLaunch &a, const float *start,
                               float dev_th, uint8_t *refit) {
    if (!learned_schedule_supported(kind, R, iters, bisections)) return cudaErrorInvalidValue;
    if (kind == kGS2D) {
        switch (R) {
        case 7: return launch_learned_shape<kGS2D, 7>(iters, bisections, a, start, dev_th, refit);
        case 9: return launch_learned_shape<kGS2D, 9>(iters, bisections, a, start, dev_th, refit);
        case 11: return launch_learned_shape<kGS2D, 11>(iters, bisections, a, start, dev_th, refit);
        }
    } else if (kind == kAS3D) {
        switch (R) {
        case 7: return launch_learned_shape<kAS3D, 7>(iters, bisections, a, start, dev_th, refit);
        case 9: return launch_learned_shape<kAS3D, 9>(iters, bisections, a, start, dev_th, refit);
        case 11: return launch_learned_shape<kAS3D, 11>(iters, bisections, a, start, dev_th, refit);
        }
    }
    return cudaErrorInvalidValue;
}

// Learned-start two-emitter schedules: 3 or 4 iterations of 6 steps, and the
// reference's 13 of 11; ROI sizes 7, 9, 11.
bool learned_2e_supported(int R, int iters, int bisections) {
    return (R == 7 || R == 9 || R == 11) &&
           ((bisections == 6 && (iters == 3 || iters == 4)) || (bisections == kBisections && iters == 13));
}

cudaError_t launch_fit_learned_2e(int R, int iters, int bisections, const FitLaunch &a, const float *start,
                                  float dev_th, uint8_t *refit, int to3e) {
    if (!learned_2e_supported(R, iters, bisections)) return cudaErrorInvalidValue;
#define QCS_L2E(RR)                                                                                   \
    if (R == RR) {                                                                                  \
        if (iters == 3 && bisections == 6) return launch_learned_2e<RR, 3, 6>(a, start, dev_th, refit, to3e); \
        if (iters == 4 && bisections == 6) return launch_learned_2e<RR, 4, 6>(a, start, dev_th, refit, to3e); \
        return launch_learned_2e<RR, 13, kBisections>(a, start, dev_th, refit, to3e);                       \
    }
    QCS_L2E(7)
    QCS_L2E(9)
    QCS_L2E(11)
#undef QCS_L2E
    return cudaErrorInvalidValue;
}

bool learned_3e_supported(int R, int iters, int bisections) {
    return (R == 7 || R == 9 || R == 11) &&
           ((bisections == 6 && (iters == 4 || iters == 6)) || (bisections == kBisections && iters == 16));
}

cudaError_t launch_fit_learned_3e(int R, int iters, int bisections, const FitLaunch &a, const float *start,
                                  float dev_th, uint8_t *refit) {
    if (!learned_3e_supported(R, iters, bisections)) return cudaErrorInvalidValue;
#define QCS_L3E(RR)                                                                          \
    if (R == RR) {                                                                         \
        if (iters == 4 && bisections == 6) return launch_learned_3e<RR, 4, 6>(a, start, dev_th, refit); \
        if (iters == 6 && bisections == 6) return launch_learned_3e<RR, 6, 6>(a, start, dev_th, refit); \
        return launch_learned_3e<RR, 16, kBisections>(a, start, dev_th, refit);                        \
    }
    QCS_L3E(7)
    QCS_L3E(9)
    QCS_L3E(11)
#undef QCS_L3E
    return cudaErrorInvalidValue;
}

cudaError_t launch_flag_slots(const uint8_t *flags, const int *n_dev, int max_n, const int *q, int *slots, int *ids,
                              int *count, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), s);
    if (e != cudaSuccess || max_n <= 0) return e;
    flag_slots_kernel<<<(max_n + 255) / 256, 256, 0, s>>>(flags, n_dev, max_n, q, slots, ids, count);
    return cudaGetLastError();
}

cudaError_t launch_merge_refit(const int *slots, const int *count, int max_n, const int8_t *res_k,
                               const float *extra_k, int8_t *res, float *extra, cudaStream_t s) {
    if (max_n <= 0) return cudaSuccess;
    merge_refit_kernel<<<(max_n + 255) / 256, 256, 0, s>>>(slots, count, max_n, res_k, extra_k, res, extra);
    return cudaGetLastError();
}

cudaError_t launch_flag_queue(const uint8_t *flags, int n, int *ids, int *count, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), s);
    if (e != cudaSuccess || n <= 0) return e;
    flag_queue_kernel<<<(n + 255) / 256, 256, 0, s>>>(flags, n, ids, count);
    return cudaGetLastError();
}

// Sizes whose pixel distance is written with an explicit contraction
// (ArithSpec DIST != kCompiler): there the group kernel's per-pixel terms are
// the thread kernel's bit for bit.  Where nvcc chooses the contraction from
// the surrounding code (GS2D / AS3D 5x5, 15x15, 17x17, AS3D 13x13) the two
// kernels' choices differ, so those sizes are not offered.
bool group_fit_supported(int kind, int R) {
    if (kind == kGS2D) return R == 7 || R == 9 || R == 11 || R == 13;
    if (kind == kAS3D) return R == 7 || R == 9 || R == 11;
    return false;
}

cudaError_t launch_fit_group(int kind, int R, int lanes, const FitLaunch &a) {
    if (!group_fit_supported(kind, R)) return cudaErrorInvalidValue;
    const bool gs = kind == kGS2D;
    if (lanes == 4 || lanes == 16) {
        if (!gs || R != 7) return cudaErrorInvalidValue;
        return lanes == 4 ? launch_single_group<7, kGS2D, 4>(a) : launch_single_group<7, kGS2D, 16>(a);
    }
    if (lanes != 8) return cudaErrorInvalidValue;
    switch (R) {
    case 7: return gs ? launch_single_group<7, kGS2D, 8>(a) : launch_single_group<7, kAS3D, 8>(a);
    case 9: return gs ? launch_single_group<9, kGS2D, 8>(a) : launch_single_group<9, kAS3D, 8>(a);
    case 11: return gs ? launch_single_group<11, kGS2D, 8>(a) : launch_single_group<11, kAS3D, 8>(a);
    case 13: return launch_single_group<13, kGS2D, 8>(a);
    }
    return cudaErrorInvalidValue;
}

bool mixed_fit_supported(int kind, int R) { return (kind == kGS2D || kind == kAS3D) && (R == 7 || R == 9 || R == 11); }

namespace {
int mixed_slots(int kind, int R) {
    switch (mixed_code(kind, R)) {
    case mixed_code(kGS2D, 7): return MixedShape<7, kGS2D>::S;
    case mixed_code(kGS2D, 9): return MixedShape<9, kGS2D>::S;
    case mixed_code(kGS2D, 11): return MixedShape<11, kGS2D>::S;
    case mixed_code(kAS3D, 7): return MixedShape<7, kAS3D>::S;
    case mixed_code(kAS3D, 9): return MixedShape<9, kAS3D>::S;
    case mixed_code(kAS3D, 11): return MixedShape<11, kAS3D>::S;
    }
    return 0;
}
}  // namespace

cudaError_t launch_fit_mixed(const FitLaunch *f, const int *kind, const int *R, int count, int *d_next,
                             cudaStream_t s) {
    if (count < 1 || count > kMixedMax || !d_next) return cudaErrorInvalidValue;
    MixedArgs a{};
    a.count = count;
    a.next = d_next;
    // larger ROIs first (their fits take longest); ties keep the caller's order
    int order[kMixedMax];
    for (int i = 0; i < count; ++i) order[i] = i;
    for (int i = 1; i < count; ++i)
        for (int j = i; j > 0 && R[order[j]] > R[order[j - 1]]; --j) std::swap(order[j], order[j - 1]);
    long long tiles = 0;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        if (!mixed_fit_supported(kind[i], R[i]) || f[i].ll || (reinterpret_cast<uintptr_t>(f[i].rois) & 3) != 0)
            return cudaErrorInvalidValue;
        MixedSeg &g = a.seg[k];
        g.rois = f[i].rois;
        g.wle = f[i].wle;
        g.q = f[i].q;
        g.loc = f[i].loc;
        g.to2e = f[i].to2e;
        g.c = f[i].para;
        g.code = mixed_code(kind[i], R[i]);
        g.slots = mixed_slots(kind[i], R[i]);
        tiles += (f[i].max_count + g.slots - 1) / g.slots;
    }
    cudaError_t e = cudaMemsetAsync(d_next, 0, sizeof(int), s);
    if (e != cudaSuccess || tiles == 0) return e;
    const size_t smem = kMixedBudget * sizeof(float);
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_mixed_kernel, kTPB, smem)) != cudaSuccess)
        return e;
    const long long resident = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(tiles < resident ? tiles : resident);
    fit_mixed_kernel<<<grid, kTPB, smem, s>>>(a);
    return cudaGetLastError();
}

// ROI sizes: odd 5..17 for single emitter, 5..13 for multi emitter (the
// reference's shared-memory limit, bfgsMLE_Multi_Emitter_Fit.cu:62-70).
cudaError_t launch_fit(int kind, int R, const FitLaunch &a) {
#define QCS_SINGLE(RR)                                              \
    case RR:                                                        \
        return kind == kGS2D ? launch_single<RR, kGS2D>(a) : launch_single<RR, kAS3D>(a);
#define QCS_MULTI(RR)                                                                        \
    case RR:                                                                                 \
        return kind == k2E ? launch_multi<RR, k2E>(a)                                        \
                           : (kind == k3E ? launch_multi<RR, k3E>(a) : launch_multi<RR, kAS3D2E>(a));
    if (kind == kGS2D || kind == kAS3D) {
        switch (R) {
            QCS_SINGLE(5)
            QCS_SINGLE(7)
            QCS_SINGLE(9)
            QCS_SINGLE(11)
            QCS_SINGLE(13)
            QCS_SINGLE(15)
            QCS_SINGLE(17)
        }
    } else {
        switch (R) {
            QCS_MULTI(5)
            QCS_MULTI(7)
            QCS_MULTI(9)
            QCS_MULTI(11)
            QCS_MULTI(13)
        }
    }
#undef QCS_SINGLE
#undef QCS_MULTI
    return cudaErrorInvalidValue;
}

}  // namespace qcs
