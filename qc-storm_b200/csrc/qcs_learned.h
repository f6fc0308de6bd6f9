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
constexpr int kOut = 8;                 // 5 used, padded for the tensor-core tiles
constexpr int kOutUsed = 5;             // dx, dy, sigma - 1.3, log(peak / range), (bkg - min) / range
constexpr int kStart = 5;               // start point: peak e-, x, y, sigma, background e-
constexpr int kParams = kIn * kHidden + kHidden + kHidden * kHidden + kHidden + kHidden * kOut + kOut;

// loss weight of each output (positions matter most)
__constant__ const float kTargetWeight[kOutUsed] = {4.0f, 4.0f, 1.0f, 1.0f, 1.0f};

// Start points (peak e-, x, y, sigma, background e- per record) of n device
// records into out (n x 5 floats).
cudaError_t start_points(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n, float *out,
                         cudaStream_t s);

}  // namespace learned
}  // namespace qcs
