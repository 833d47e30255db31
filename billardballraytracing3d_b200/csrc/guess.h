// Shapes, parameter layout and entry points of the learned-guess MLP
// (guess_mlp.cu), shared with the host code that trains and uses it.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dscene.h"

namespace bbrt {

// 41 inputs (9 geometric + 32 embedding) padded to 64; 3 hidden layers of
// 128; 4 outputs (u, v, s, confidence logit) padded to 16.
constexpr int kIn = 64, kH = 128, kOut = 16, kEmb = 32, kGeo = 9;

// FP32 master parameters, flat: W0 [128][64], b0, W1 [128][128], b1,
// W2 [128][128], b2, W3 [16][128], b3 [16], then E [patches][32].
constexpr int oW0 = 0, oB0 = oW0 + kH * kIn, oW1 = oB0 + kH, oB1 = oW1 + kH * kH, oW2 = oB1 + kH,
              oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kOut * kH, oE = oB3 + kOut;

// BF16 weight image: core-blocked W0 (128 x 64), W1, W2 (128 x 128), W3 (16 x 128).
constexpr int iW0 = 0, iW1 = iW0 + kH * kIn * 2, iW2 = iW1 + kH * kH * 2, iW3 = iW2 + kH * kH * 2,
              kImageBytes = iW3 + kOut * kH * 2;

// Shared-memory maps (bytes) of the training and inference kernels.
constexpr int kTrainX = kImageBytes, kTrainH1 = kTrainX + 128 * kIn * 2, kTrainH2 = kTrainH1 + 128 * kH * 2,
              kTrainH3 = kTrainH2 + 128 * kH * 2, kTrainG4 = kTrainH3 + 128 * kH * 2,
              kTrainBias = kTrainG4 + 128 * kOut * 2, kTrainSmem = kTrainBias + (3 * kH + kOut) * 4;
constexpr int kInferX = kImageBytes, kInferH = kInferX + 128 * kIn * 2, kInferBias = kInferH + 128 * kH * 2,
              kInferSmem = kInferBias + (3 * kH + kOut) * 4;

// Default bound of a tensor-core completion wait (SM cycles, about 2 s).
constexpr long long kMbarDefault = 4000000000LL;

constexpr float kGeluC = 0.7978845608028654f;   // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;

// Per-patch frame, 16 doubles: centre (3), tangent t1 (3), tangent t2 (3),
// normal (3), size L (half the box diagonal), box half-extents / L (3).
constexpr int kFrame = 16;

// The 9 geometric inputs of a ray against a patch frame: closest-approach
// point to the centre in the frame (/ L), direction in the frame, box
// extents; t0 = ray parameter of the closest approach (d of unit length).
__host__ __device__ inline void ray_features(const double* f, double ox, double oy, double oz, double dx, double dy,
                                             double dz, float* geo, double& t0) {
    t0 = (f[0] - ox) * dx + (f[1] - oy) * dy + (f[2] - oz) * dz;
    const double px = ox + t0 * dx - f[0], py = oy + t0 * dy - f[1], pz = oz + t0 * dz - f[2];
    const double il = 1.0 / f[12];
    geo[0] = static_cast<float>((px * f[3] + py * f[4] + pz * f[5]) * il);
    geo[1] = static_cast<float>((px * f[6] + py * f[7] + pz * f[8]) * il);
    geo[2] = static_cast<float>((px * f[9] + py * f[10] + pz * f[11]) * il);
    geo[3] = static_cast<float>(dx * f[3] + dy * f[4] + dz * f[5]);
    geo[4] = static_cast<float>(dx * f[6] + dy * f[7] + dz * f[8]);
    geo[5] = static_cast<float>(dx * f[9] + dy * f[10] + dz * f[11]);
    geo[6] = static_cast<float>(f[13]);
    geo[7] = static_cast<float>(f[14]);
    geo[8] = static_cast<float>(f[15]);
}

// Index of parameter p's gradient in the gradient buffer (W0..W2 are stored
// transposed there, [i][o], so that the kernels' adds are coalesced).
__host__ __device__ inline long long grad_index(long long p) {
    if (p < oB0) return oW0 + (p - oW0) % kIn * kH + (p - oW0) / kIn;
    if (p >= oW1 && p < oB1) return oW1 + (p - oW1) % kH * kH + (p - oW1) / kH;
    if (p >= oW2 && p < oB2) return oW2 + (p - oW2) % kH * kH + (p - oW2) / kH;
    return p;
}

// One training sample recorded by the trace: a (ray, patch) pair and, for a
// positive, the converged Newton solution.
struct GuessSample {
    double o[3], d[3];
    double u, v, t;
    int patch;
    int label;   // 1: Newton converged inside the patch, 0: stage 1 found no triangle
};

struct MlpBatch {
    const float* feat;   // [N][9]
    const int* pid;      // [N] patch of each row
    const float* tgt;    // [N][3] u, v, s
    const float* lbl;    // [N] 1 / 0
    const int* idx;      // [B] sample rows of this batch, or nullptr for 0..B-1
    int B;
    float inv_b;
};

struct MlpNet {
    const uint8_t* image;   // BF16 weight image
    float* P;               // FP32 master parameters
    float* G;               // gradients (W0..W2 transposed: [i][o])
    float* loss;            // loss accumulator
    float* out;             // optional [B][4] forward outputs of a training batch
    int* err;               // set when an MMA completion wait timed out
    long long mbar_limit = kMbarDefault;   // SM cycles a completion wait may take before it gives up
};

cudaError_t mlp_pack(const float* P, uint8_t* image, cudaStream_t st);
cudaError_t mlp_train_batch(const MlpBatch& Bt, const MlpNet& M, cudaStream_t st);
cudaError_t mlp_adam(const MlpNet& M, float* m1, float* m2, long long n, float lr, int step, cudaStream_t st);
cudaError_t mlp_infer_features(const float* feat, const int* pid, long long n, const MlpNet& M, double* out,
                               cudaStream_t st);
// n_dev (graph launch): the request count is read on the device; n sizes the grid.
cudaError_t mlp_infer_requests(const NewtonRequest* req, long long n, const double* o, const double* d,
                               const int* obj_sub, const double* frame, const MlpNet& M, double* out,
                               cudaStream_t st, const unsigned int* n_dev = nullptr);
cudaError_t mlp_make_rows(const GuessSample* S, long long n, const double* frame, float* feat, int* pid, float* tgt,
                          float* lbl, cudaStream_t st);

}  // namespace bbrt
