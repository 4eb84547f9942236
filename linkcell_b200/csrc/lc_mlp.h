// The shell-proposal MLP: sizes, scratch layout and launch wrappers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lc_kernels.h"

namespace lc {

constexpr int kMlpIn = 126;      // 125 log(1 + occupancy) features + k / 64
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 8;       // settled shell 1..7, and "8 or more"
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden +
                           kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;

// Activation scratch of a batch of B rows (caller-provided device memory).
struct MlpScratch {
  float *z1, *h1, *z2, *h2, *z3, *dz3, *dz2, *dz1;
  static size_t floats(int B) {
    return size_t(B) * (4 * kMlpHidden + 2 * kMlpOut + 2 * kMlpHidden);
  }
  static MlpScratch carve(float *base, int B) {
    MlpScratch t;
    float *q = base;
    t.z1 = q; q += size_t(B) * kMlpHidden;
    t.h1 = q; q += size_t(B) * kMlpHidden;
    t.z2 = q; q += size_t(B) * kMlpHidden;
    t.h2 = q; q += size_t(B) * kMlpHidden;
    t.z3 = q; q += size_t(B) * kMlpOut;
    t.dz3 = q; q += size_t(B) * kMlpOut;
    t.dz2 = q; q += size_t(B) * kMlpHidden;
    t.dz1 = q;
    return t;
  }
};

cudaError_t mlp_cell_features(const FrameDesc *frames, const uint32_t *off,
                              const int *frame_of_row, const uint32_t *cell_of_row, long long rows,
                              float *X, cudaStream_t s);
cudaError_t mlp_forward(const float *params, const float *X, int B, MlpScratch &t, float *probs,
                        cudaStream_t s);
cudaError_t mlp_grad(const float *params, const float *X, const int *y, int B, MlpScratch &t,
                     float *grad, float *loss, cudaStream_t s);
cudaError_t mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr,
                     cudaStream_t s);
// Proposed shell per cell (tcgen05 inference over 16 x 8-cell tiles of 128
// cells, the first layer as a 5x5x5 convolution of the
// occupancy grid), then per sorted source.
cudaError_t mlp_propose(const void *image, const BatchBuffers &b, int8_t *cell_prop,
                        int8_t *source_prop, float tau, cudaStream_t s);
// The inference kernel's operand image of a parameter vector (mlp_image_bytes
// of device memory, 16-byte aligned), written once per model.
size_t mlp_image_bytes();
cudaError_t mlp_pack(const float *params, void *image, cudaStream_t s);
// Training rows from a logged search: features of the cell of every
// stride-th sorted source and its settled shell class (min(R*, 8) - 1).
cudaError_t mlp_training_rows(const BatchBuffers &b, const int8_t *stop_log, long long stride,
                              long long first, float *X, int *y, long long cap, cudaStream_t s);

}  // namespace lc
