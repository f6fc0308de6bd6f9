// Constants of the learned start-point network (qcs_learned.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"

namespace qcs {
namespace learned {

constexpr int kR = 7;                   // ROI size the network is built for
constexpr int kPix = kR * kR;           // 49 pixels
constexpr int kWhole = kR * (kR + 1);   // record length in uint16
constexpr int kHalf = kR / 2;
constexpr float kCentre = kR / 2.0f;    // ROI centre in the fit's pixel coordinates
constexpr float kSigma0 = 1.3f;         // sigma offset of the sigma output
constexpr int kIn = 64;                 // 49 pixels + 2 scale features + zero padding
constexpr int kHidden = 128;
constexpr int kOut = 8;                 // 5 start-point outputs, 3 emitter-count logits
constexpr int kOutUsed = 5;             // dx, dy, sigma - 1.3, log(peak / range), (bkg - min) / range
constexpr int kCount0 = 5;              // logits of the emitter-count classes 0, 1, 2 (outputs 5..7)
constexpr int kClasses = 3;             // one emitter / two-emitter stage / three-emitter stage
constexpr int kStart = 5;               // start point: peak e-, x, y, sigma, background e-
constexpr int kParams = kIn * kHidden + kHidden + kHidden * kHidden + kHidden + kHidden * kOut + kOut;

// loss weight of each output (positions matter most) and of the emitter-count
// cross-entropy
__constant__ const float kTargetWeight[kOutUsed] = {4.0f, 4.0f, 1.0f, 1.0f, 1.0f};
constexpr float kCountWeight = 0.5f;

// Emitter-count class from the three logits: 2 when p(class 2) >= th, else 1
// when p(class 1) + p(class 2) >= th, else 0 (softmax probabilities).
__host__ __device__ inline int count_class(float l0, float l1, float l2, float th) {
    const float m = fmaxf(l0, fmaxf(l1, l2));
    const float e0 = expf(l0 - m), e1 = expf(l1 - m), e2 = expf(l2 - m);
    const float sum = e0 + e1 + e2;
    if (e2 >= th * sum) return 2;
    if (e1 + e2 >= th * sum) return 1;
    return 0;
}

// Start points (peak e-, x, y, sigma, background e- per record) of n device
// records into out (n x 5 floats); with cls set, also each record's
// emitter-count class at the network's count threshold.  With n_dev set the
// fused kernel reads the record count there (at most n); the layer-by-layer
// path computes all n.
cudaError_t start_points(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n, float *out,
                         cudaStream_t s, uint8_t *cls = nullptr, const int *n_dev = nullptr);

}  // namespace learned
}  // namespace qcs
