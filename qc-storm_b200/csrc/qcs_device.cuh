// Device-side shared definitions of the qcstorm_b200 kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"

namespace qcs {

// Fitting parameters copied to the device by value in every launch; the
// fields and their meaning are those of the reference's CoreFittingPara
// (bfgsMLE_Loc_LD/bfgs_base.h:113-141).
struct CorePara {
    int MultiEmitterFitEn;
    int WLEEn;
    float Offset;
    float KAdc;
    float QE;
    float ReadNoise_e;
    float ZDepthCorrFactor;
    float p4_XGY, p3_XGY, p2_XGY, p1_XGY, p0_XGY;
    float p4_XLY, p3_XLY, p2_XLY, p1_XLY, p0_XLY;
};

inline CorePara core_para(const qcs_loc_para &p) {
    CorePara c;
    c.MultiEmitterFitEn = p.MultiEmitterFitEn;
    c.WLEEn = p.WLEEn;
    c.Offset = p.Offset;
    c.KAdc = p.KAdc;
    c.QE = p.QE;
    c.ReadNoise_e = p.ReadNoise_e;
    c.ZDepthCorrFactor = p.ZDepthCorrFactor;
    c.p4_XGY = p.p4_XGY; c.p3_XGY = p.p3_XGY; c.p2_XGY = p.p2_XGY; c.p1_XGY = p.p1_XGY; c.p0_XGY = p.p0_XGY;
    c.p4_XLY = p.p4_XLY; c.p3_XLY = p.p3_XLY; c.p2_XLY = p.p2_XLY; c.p1_XLY = p.p1_XLY; c.p0_XLY = p.p0_XLY;
    return c;
}

// A list of ROI indices processed by one fit launch.  Either an identity range
// [0, n) or `ids[0..count)`; the count can live in device memory (written by
// an earlier kernel of the same stream), so no host round trip is needed.
struct Queue {
    const int *ids;        // nullptr: identity
    const int *count_dev;  // nullptr: use count
    int count;
};

__device__ __forceinline__ int queue_len(const Queue &q) { return q.count_dev ? *q.count_dev : q.count; }
__device__ __forceinline__ int queue_at(const Queue &q, int i) { return q.ids ? q.ids[i] : i; }

// Per-slot result of a multi-emitter fit: 0 rejected, 1 first emitter only,
// 2 first and second emitter (the second one's row is in `extra`).
struct MultiOut {
    int8_t *result;
    float *extra;  // 12 floats per queue slot
    // three-emitter kind only, when set: each slot's final fitted parameters
    // (11 floats, fit units: peak / 128, x, y per emitter, 1/(2 sigma^2) / 0.1,
    // background / 64), written before the emitter selection
    float *params = nullptr;
};

}  // namespace qcs
