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
                             uint32_t probe_topk, int semantics, uint32_t nq_max, float *approx,
                             unsigned *err, cudaStream_t st, int *n_launch);

// bucket-weight tables of the tensor-memory MaxSim kernels (make_tm_weights):
//  BF16 (1-, 2-bit): w[0] / w[1] = low / high bytes of the BF16 weights;
//  FP8 2-bit: w[0] = the 4 E4M3 weights;
//  FP8 4-bit: w[0..1] = |E4M3| of weights 0..7, w[2..3] of weights 8..15,
//             w[4..5] byte j: bit 6 = sign of weight j, bit 7 = of weight 8 + j
struct TmWeights {
  uint32_t w[6];
};
TmWeights make_tm_weights(uint32_t n_bit, const float *weight, bool fp8);

// BF16 MaxSim with the decoded doc tokens in tensor memory (1- and 2-bit
// codes); cen_perm: [C][64] bf16x2 centroid rows in the kernel's K order
// (make_centroid_perm); x_bound: upper bound on the norm of every decoded
// doc token
bool tmem_rerank_supported(uint32_t n_bit);
// largest L2 norm of the centroid rows (d_tmp: one device word of scratch)
cudaError_t max_centroid_norm(const float *cen, uint32_t n_cent, unsigned *d_tmp, float *out,
                              cudaStream_t st);
cudaError_t make_centroid_perm(const float *cen, uint32_t n_cent, uint32_t n_bit, void *out,
                               cudaStream_t st);
cudaError_t launch_rerank_tmem(const DevIndex &ix, const void *cen_perm, const TmWeights &tw,
                               const float *q, const uint64_t *q_off, uint32_t n_query,
                               const uint32_t *short_id, const uint32_t *n_short,
                               uint32_t probe_topk, int semantics, uint32_t nq_max, float x_bound,
                               float *approx, unsigned *err, cudaStream_t st, int *n_launch,
                               bool fp8);
// FP8 (E4M3) MaxSim for 2- and 4-bit codes: cen8 [C][128] E4M3 centroid
// rows in the FP8 kernel's K order for n_bit (make_centroid_fp8); pass it as
// cen_perm with fp8 = true
bool fp8_rerank_supported(uint32_t n_bit);
cudaError_t make_centroid_fp8(const float *cen, uint32_t n_cent, uint32_t n_bit, void *out,
                              cudaStream_t st);

// The same FP8 MaxSim, warp-specialised (producer / decoders / MMA / epilogue
// over a shared-memory ring fed by bulk copies): cen8 as above with one zero
// row appended (row n_centroid); the vq code array must be readable 16 bytes
// past its last code.  wait_ns bounds every pipeline wait of the kernel (on
// expiry it stops and sets bit 4 of *err); docs: shortlisted docs per CTA.
cudaError_t launch_rerank_ws(const DevIndex &ix, const void *cen8, const TmWeights &tw,
                             const float *q, const uint64_t *q_off, uint32_t n_query,
                             const uint32_t *short_id, const uint32_t *n_short,
                             uint32_t probe_topk, int semantics, uint32_t nq_max, float x_bound,
                             float *approx, unsigned *err, cudaStream_t st, int *n_launch,
                             uint64_t wait_ns, uint32_t docs);
// shortlisted docs per CTA the FP8 kernel is built for (32, 64, 128, 256)
bool ws_docs_supported(uint32_t docs);

// Learned-pruner features of every shortlisted doc with the FP8 kernel's
// centroid part only: feat [n_query][probe_topk][33] = per query token the
// best E4M3 centroid score q.c over the doc's tokens, then log(doc length).
// Queries of up to 32 tokens.
cudaError_t launch_prune_features(const DevIndex &ix, const void *cen8, const float *q,
                                  const uint64_t *q_off, uint32_t n_query,
                                  const uint32_t *short_id, const uint32_t *n_short,
                                  uint32_t probe_topk, float x_bound, float *feat, unsigned *err,
                                  cudaStream_t st, int *n_launch, uint64_t wait_ns);
// The docs the rerank takes after the pruner (see mvr_tc.cu).
cudaError_t launch_prune_choose(const DevIndex &ix, const uint32_t *short_id,
                                const uint32_t *n_short, const uint32_t *kept_id,
                                const float *kept_s, uint32_t n_query, uint32_t probe_topk,
                                uint32_t keep, uint32_t R, float margin, uint32_t *fin_id,
                                uint32_t *n_fin, uint32_t *qstat,
                                unsigned long long *n_fallback, cudaStream_t st, int *n_launch);
// The learned pruner's MLP on the tensor cores: pred [n_query][probe_topk]
// from the features of the rows d < n_short[query]; wts / vecs: the weights
// prepared by prune_prepare (prune_weight_bytes() bytes / 769 floats).
size_t prune_weight_bytes();
cudaError_t prune_prepare(const float *params, uint8_t *wts, float *vecs, cudaStream_t st);
cudaError_t launch_prune_mlp(const float *feat, const uint32_t *n_short, uint32_t n_query,
                             uint32_t probe_topk, const uint8_t *wts, const float *vecs,
                             float *pred, unsigned *err, int n_sm, cudaStream_t st,
                             int *n_launch);

// tensor-core centroid scoring: candidates per token = splits * 16; the
// centroid tiles hold 64 centroids each (n_tiles = C_pad / 64)
uint32_t probe_tc_cand_per_token(uint32_t n_tok, uint32_t n_cent, int n_sm, uint32_t *splits);
cudaError_t make_centroid_tiles(const float *cen, uint32_t n_cent, uint32_t n_tiles, void *out,
                                cudaStream_t st);
cudaError_t launch_probe_tc(const float *q, uint32_t n_tok, const void *cen_sw, const float *cen,
                            uint32_t n_cent, uint32_t nprobe, uint32_t splits, uint32_t *cand,
                            uint32_t *out_id, float *out_s, unsigned *err, cudaStream_t st,
                            int *n_launch);

}  // namespace mvr
