// mvr_prune.cuh -- training of the learned candidate pruner's MLP (33 -> 256
// -> 256 -> 1, GELU over per-candidate features) on CUDA cores
// (mvr_prune.cu); its tensor-core inference kernel is in mvr_tc.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mvr {

// Features of one (query, shortlisted doc) pair: for each of up to 32 query
// tokens the best centroid score among the doc's tokens' centroids (the
// token's top centroid score over the doc; 0 for tokens past the query's
// last), then log(doc length).
constexpr int kFeat = 33;
constexpr int kFeatTok = 32;
constexpr int kHid = 256;

// Parameter vector (float): W1 [256][33], b1 [256], W2 [256][256], b2 [256],
// w3 [256], b3 [1]; weights are applied rounded to BF16, accumulation is FP32.
constexpr uint32_t kOffW1 = 0;
constexpr uint32_t kOffB1 = kOffW1 + kHid * kFeat;
constexpr uint32_t kOffW2 = kOffB1 + kHid;
constexpr uint32_t kOffB2 = kOffW2 + kHid * kHid;
constexpr uint32_t kOffW3 = kOffB2 + kHid;
constexpr uint32_t kOffB3 = kOffW3 + kHid;
constexpr uint32_t kNumParams = kOffB3 + 1;  // 74,753

// floats of training workspace for minibatches of n rows
inline size_t mlp_work_floats(uint32_t n) {
  return (size_t)n * (6 * kHid + 2) + 2 * (size_t)kNumParams + 64;
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the mean squared error
// 0.5 * mean((mlp(x) - y)^2) of a minibatch: x [n][33], y [n] (device);
// params / adam_m / adam_v [kNumParams] (device, updated in place); work
// [mlp_work_floats(n)]; loss_out (nullable, device float) receives the
// minibatch loss before the step.  step counts from 1.
cudaError_t mlp_train_step(const float *x, const float *y, uint32_t n, float *params,
                           float *adam_m, float *adam_v, float *work, float lr, uint32_t step,
                           float *loss_out, cudaStream_t st);

// Reference forward pass on CUDA cores (FP32 accumulation, BF16-rounded
// weights): out [n] (device).
cudaError_t mlp_forward_ref(const float *x, uint32_t n, const float *params, float *work,
                            float *out, cudaStream_t st);

}  // namespace mvr
