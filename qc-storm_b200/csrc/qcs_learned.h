// Constants of the learned start-point network (qcs_learned.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qcstorm_b200.h"

namespace qcs {
namespace learned {

constexpr float kSigma0 = 1.3f;         // sigma offset of the sigma outputs
constexpr int kHidden = 128;
constexpr int kOut = 8;                 // start-point outputs, then (GS2D) three emitter-count logits
constexpr int kOutMax = 16;             // outputs of the widest kind (three-emitter GS2D: 11 used)
constexpr int kUsedMax = 11;            // start-point outputs of the widest kind (three-emitter GS2D)
constexpr int kTwo = QCS_LEARNED_GS2D_2E;    // network kind of the two-emitter start points
constexpr int kThree = QCS_LEARNED_GS2D_3E;  // network kind of the three-emitter start points
constexpr int kCount0 = 5;              // GS2D: logits of the emitter-count classes 0, 1, 2 (outputs 5..7)
constexpr int kClasses = 3;             // one emitter / two-emitter stage / three-emitter stage

// Network shapes: one per localization type (GS2D, AS3D) and ROI size (7, 9, 11).
// Input: the R*R photoelectron pixels scaled to [0, 1] by the ROI's range,
// log(range) / 8, log(min) / 8, zero padding to 64 (7x7) or 128 (9x9, 11x11).
__host__ __device__ constexpr int in_width(int R) { return R * R + 2 <= 64 ? 64 : 128; }
// Outputs fitted to the targets: GS2D dx, dy, sigma - 1.3, log(peak / range),
// (background - min) / range; AS3D the same with sigma_x and then sigma_y - 1.3;
// two-emitter GS2D dx0, dy0, dx1, dy1, log(peak0 / range), log(peak1 / range),
// sigma - 1.3, (background - min) / range; three-emitter GS2D dx0, dy0, dx1,
// dy1, dx2, dy2, log(peak0..2 / range), sigma - 1.3, (background - min) / range.
__host__ __device__ constexpr int used_outputs(int loc_type) {
    return loc_type == kThree ? 11 : (loc_type == kTwo ? 8 : (loc_type == QCS_LOCTYPE_AS3D ? 6 : 5));
}
// Network outputs per record: 8, or 16 for the three-emitter kind.
__host__ __device__ constexpr int out_width(int loc_type) { return loc_type == kThree ? kOutMax : kOut; }
// Start point per record: GS2D peak e-, x, y, sigma, background e-; AS3D
// peak e-, x, y, sigma_x, sigma_y, background e-; two- and three-emitter
// GS2D peak e-, x, y of each emitter, then sigma, background e- (each fit's
// parameter order).
__host__ __device__ constexpr int start_width(int loc_type) {
    return loc_type == kThree ? 11 : (loc_type == kTwo ? 8 : (loc_type == QCS_LOCTYPE_AS3D ? 6 : 5));
}
constexpr int param_count(int kin, int nout = kOut) {
    return kin * kHidden + kHidden + kHidden * kHidden + kHidden + kHidden * nout + nout;
}
inline bool shape_supported(int loc_type, int R) {
    return (loc_type == QCS_LOCTYPE_GS2D || loc_type == QCS_LOCTYPE_AS3D || loc_type == kTwo || loc_type == kThree) &&
           (R == 7 || R == 9 || R == 11);
}

// loss weight of each start-point output (positions matter most) and of the
// emitter-count cross-entropy
// (row 0: single-emitter kinds, row 1: two-emitter GS2D, row 2: three-emitter GS2D)
__constant__ const float kTargetWeight[3][kUsedMax] = {
    {4.0f, 4.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {4.0f, 4.0f, 4.0f, 4.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f},
    {4.0f, 4.0f, 4.0f, 4.0f, 4.0f, 4.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f}};
__host__ __device__ constexpr int weight_row(int loc_type) { return loc_type == kThree ? 2 : (loc_type == kTwo ? 1 : 0); }
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

// Network outputs y (bias included) -> the fit's start point st
// (start_width(LT) floats: peak e-, x, y, sigma(s), background e-), with
// positions held inside the kind's accept window and widths in range.
template <int R, int LT>
__device__ __forceinline__ void start_from_outputs(const float *y, float lo, float rng, float *st) {
    const float centre = R / 2.0f;
    if (LT == kThree) {
        // emitters anywhere up to a pixel inside the ROI's edge
        const float w2 = R / 2.0f - 1.0f;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            st[3 * e] = rng * expf(fminf(fmaxf(y[6 + e], -6.0f), 3.0f));
            st[3 * e + 1] = centre + fminf(fmaxf(y[2 * e], -w2), w2);
            st[3 * e + 2] = centre + fminf(fmaxf(y[2 * e + 1], -w2), w2);
        }
        st[9] = fminf(fmaxf(kSigma0 + y[9], 0.6f), 3.0f);
        st[10] = fmaxf(lo + rng * y[10], 1.0f);
        return;
    }
    if (LT == kTwo) {
        // emitters anywhere up to a pixel inside the ROI's edge
        const float w2 = R / 2.0f - 1.0f;
        st[0] = rng * expf(fminf(fmaxf(y[4], -6.0f), 3.0f));
        st[1] = centre + fminf(fmaxf(y[0], -w2), w2);
        st[2] = centre + fminf(fmaxf(y[1], -w2), w2);
        st[3] = rng * expf(fminf(fmaxf(y[5], -6.0f), 3.0f));
        st[4] = centre + fminf(fmaxf(y[2], -w2), w2);
        st[5] = centre + fminf(fmaxf(y[3], -w2), w2);
        st[6] = fminf(fmaxf(kSigma0 + y[6], 0.6f), 3.0f);
        st[7] = fmaxf(lo + rng * y[7], 1.0f);
        return;
    }
    const float win = LT == QCS_LOCTYPE_AS3D ? 2.5f : 1.5f;
    const float smax = LT == QCS_LOCTYPE_AS3D ? 4.0f : 3.0f;
    st[0] = rng * expf(fminf(fmaxf(y[3], -6.0f), 3.0f));
    st[1] = centre + fminf(fmaxf(y[0], -win), win);
    st[2] = centre + fminf(fmaxf(y[1], -win), win);
    st[3] = fminf(fmaxf(kSigma0 + y[2], 0.6f), smax);
    if (LT == QCS_LOCTYPE_AS3D) {
        st[4] = fminf(fmaxf(kSigma0 + y[5], 0.6f), smax);
        st[5] = fmaxf(lo + rng * y[4], 1.0f);
    } else {
        st[4] = fmaxf(lo + rng * y[4], 1.0f);
    }
}

// C = beta C + A B on the tensor cores (tcgen05, BF16 operands rounded from
// the FP32 ones, FP32 accumulation): M x N x K, A(m, k) = A[m sam + k sak],
// B(k, n) = B[k sbk + n sbn], C row-major with ldc.  ws (ws_floats floats,
// may be null): split-K partial sums, reduced in a fixed order.  err: set
// when an MMA wait gave up.
cudaError_t gemm(int M, int N, int K, const float *A, long long sam, long long sak, const float *B, long long sbk,
                 long long sbn, float *C, int ldc, float beta, cudaStream_t s, float *ws, size_t ws_floats, int *err);

// g[c] = sum over rows r of d[r * cols + c], FP32, in a fixed order (two
// passes: up to kColsumSplits row splits into part, then their sum); part
// holds kColsumSplits * cols floats.
constexpr int kColsumSplits = 128;
cudaError_t column_sums(const float *d, long long rows, int cols, float *g, float *part, cudaStream_t s);

// Start points (start_width floats per record) of n device records into out;
// with cls set (GS2D networks), also each record's emitter-count class at the
// network's count threshold.  With n_dev set the fused kernel reads the
// record count there (at most n); the layer-by-layer path computes all n.
cudaError_t start_points(qcs_learned_net *net, const qcs_loc_para *p, const uint16_t *d_rois, int n, float *out,
                         cudaStream_t s, uint8_t *cls = nullptr, const int *n_dev = nullptr);

// The convolutional network (qcs_convnet.cu): parameter count, training
// activations and inference buffers (State), forward / backward of one
// batch of feature rows, and the start points of n records through its two
// tcgen05 kernels (weight images rebuilt when `version` changes).
namespace conv {
struct State;
int param_count(int R);
cudaError_t create(int R, int batch, State **out);
void destroy(State *st);
void init_params(float *h, int R, unsigned long long seed);
cudaError_t forward(State *st, const float *par, const float *feat, int rows, int kin, float *y, cudaStream_t s,
                    float *ws, size_t wsf, int *err);
cudaError_t backward(State *st, const float *par, float *grad, const float *feat, int rows, int kin, const float *dy,
                     cudaStream_t s, float *ws, size_t wsf, int *err);
cudaError_t start_points(State *st, const float *par, unsigned version, int loc_type, const qcs_loc_para *p,
                         const uint16_t *rois, int n, const int *n_dev, float *out, uint8_t *cls, float th,
                         cudaStream_t s, int *err);
}  // namespace conv

// The two-emitter network attached to a GS2D network (qcs_learned_set_two_emitter),
// its schedule and fallback (to3e: poor fits go on to the three-emitter fit), or null.
qcs_learned_net *two_emitter(const qcs_learned_net *net, int *iters, int *bisections, float *dev_th, int *to3e);
// The three-emitter network attached to a GS2D network (qcs_learned_set_three_emitter)
// and its schedule, or null.
qcs_learned_net *three_emitter(const qcs_learned_net *net, int *iters, int *bisections, float *dev_th);
// qcs_learned_set_single_refits's setting
bool single_refits(const qcs_learned_net *net);
// qcs_learned_set_direct_two_emitter's setting
bool direct_two_emitter(const qcs_learned_net *net);
}  // namespace learned
}  // namespace qcs
