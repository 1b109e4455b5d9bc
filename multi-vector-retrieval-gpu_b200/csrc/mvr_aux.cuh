// mvr_aux.cuh -- launchers of the index-side kernels (mvr_aux.cu).
#pragma once
#include <cuda_runtime.h>
#include "mvr_common.cuh"

namespace mvr {

struct Cutoffs { float v[255]; };  // up to 2^8 - 1 bucket cutoffs, by value

cudaError_t launch_transpose_centroid(const float *cen, uint32_t n_cent, uint32_t n_cent_pad,
                                      float *ct, cudaStream_t st);
cudaError_t launch_decompress(const DevIndex &ix, const uint64_t *vec_id, uint64_t n, float *out,
                              cudaStream_t st);
cudaError_t launch_unpack(const DevIndex &ix, const uint64_t *vec_id, uint64_t n, uint8_t *out,
                          cudaStream_t st);
cudaError_t launch_pack_residual(const float *vec, uint64_t n_vec, const float *cen,
                                 const uint32_t *code, const Cutoffs &cut, uint32_t n_bit,
                                 uint8_t *out, cudaStream_t st);
cudaError_t launch_kmeans_accumulate(const float *vec, uint64_t n_vec, const uint32_t *code,
                                     double *sum, uint64_t *count, cudaStream_t st);
// out[r] = the rank[r]-th smallest (0-based) residual error vec - centroid[code]
// over all n_vec * 128 values (synchronises st)
cudaError_t residual_select(const float *vec, uint64_t n_vec, const float *cen,
                            const uint32_t *code, const uint64_t *rank, uint32_t n_rank,
                            float *out, cudaStream_t st);

}  // namespace mvr
