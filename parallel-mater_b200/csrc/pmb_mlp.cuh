// SPDX-License-Identifier: MIT
// Learned warm start: an 8 -> 64 -> 64 -> 2 MLP over per-contact features,
// predicting the normal row's converged (lambda, penalty). BF16 operands on
// the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM), FP32
// accumulation, FP32 master weights and Adam moments.
//
// Biases are folded into the weight matrices through constant-one columns:
// feature 8 of X is 1 (so W1[:, 8] = b1), column 64 of both hidden
// activations is 1 (W2[:, 64] = b2, W3[:, 64] = b3). Padding columns are zero,
// so their gradients are exactly zero and no mask is needed.
#pragma once
#include <cstdint>

namespace pmb {

constexpr uint32_t kMlpFeatures = 8;   // real inputs
constexpr uint32_t kMlpIn = 16;        // X columns: 8 features, 1, zeros
constexpr uint32_t kMlpHidden = 64;
constexpr uint32_t kMlpHiddenK = 80;   // hidden + constant-one column + zeros (K multiple of 16)
constexpr uint32_t kMlpOut = 2;
constexpr uint32_t kMlpOutN = 16;      // padded output rows of W3
constexpr uint32_t kMlpTile = 128;     // contacts per tile (the MMA's M)

// Master parameter vector: W1 [64][16], W2 [64][80], W3 [16][80], row-major.
constexpr uint32_t kMlpW1 = 0;
constexpr uint32_t kMlpW2 = kMlpW1 + kMlpHidden * kMlpIn;
constexpr uint32_t kMlpW3 = kMlpW2 + kMlpHidden * kMlpHiddenK;
constexpr uint32_t kMlpParams = kMlpW3 + kMlpOutN * kMlpHiddenK;  // 7424
// A CTA's partial vector: the gradient, the weighted squared error and the
// weighted squared error of a zero prediction (the plain warm start).
constexpr uint32_t kMlpPartial = kMlpParams + 2;
// Output scaling: o0 = kLamOut * correction of log1p(lambda / scale),
// o1 = kPenOut * correction of log10(penalty).
constexpr float kLamOut = 4.0f;
constexpr float kPenOut = 100.0f;
// Largest applied correction in those log spaces (1 = a decade of penalty).
constexpr float kMaxCorrection = 1.0f;

// BF16 weight images in the tensor cores' shared-memory layout (no swizzle,
// K-major core matrices of 8 rows x 16 bytes), copied into shared memory
// with one bulk copy each.
constexpr uint32_t kImgW1 = 0;                                   // 2048 B
constexpr uint32_t kImgW2 = kImgW1 + kMlpHidden * kMlpIn * 2;    // 10240 B
constexpr uint32_t kImgW3 = kImgW2 + kMlpHidden * kMlpHiddenK * 2;  // 2560 B
constexpr uint32_t kImgBytes = kImgW3 + kMlpOutN * kMlpHiddenK * 2;

// Byte offset of element (row n, column k) of an N-row weight matrix image.
__host__ __device__ constexpr uint32_t img_offset(uint32_t n, uint32_t k, uint32_t rows) {
    return (k / 8) * (rows / 8) * 128 + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
}
// Byte offset of element (row r, column j) of a 128-row activation tile:
// column blocks of 8 are 2048 B apart, row groups of 8 are 128 B apart.
__host__ __device__ constexpr uint32_t tile_offset(uint32_t r, uint32_t j) {
    return (j / 8) * 2048 + (r / 8) * 128 + (r % 8) * 16 + (j % 8) * 2;
}

// Per-contact row metadata beside X: target lambda and penalty (normalised),
// loss weight, lambda scale.
struct MlpMeta {
    float y0, y1, weight, scale;
};

}  // namespace pmb
