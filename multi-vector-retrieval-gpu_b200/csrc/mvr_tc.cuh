// mvr_tc.cuh -- launchers of the tensor-core (tcgen05) kernels (mvr_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include "mvr_common.cuh"

namespace mvr {

cudaError_t configure_tc_kernels();
cudaError_t make_bf16(const float *in, size_t n, void *out, cudaStream_t st);
cudaError_t launch_rerank_tc(const DevIndex &ix, const void *cen_bf16, const void *lut_bf16,
                             const float *q, const uint64_t *q_off, uint32_t n_query,
                             const uint32_t *short_id, const uint32_t *n_short,
                             uint32_t probe_topk, int semantics, float *approx, unsigned *err,
                             cudaStream_t st, int *n_launch);

}  // namespace mvr
