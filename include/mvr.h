/*
 * mvr.h -- C ABI of libmvr, the B200-native (sm_100a) GPU multi-vector
 * (ColBERT-style) search engine: centroid scoring -> IVF probe -> candidate
 * filter -> residual decompression -> exact MaxSim rerank -> top-k.
 *
 * Plain pointers and sizes only.  Every entry point returns an mvr_status
 * (MVR_OK == 0); on failure mvr_last_error() describes the error of the
 * calling thread.  No entry point calls exit().  One index handle is used
 * from one host thread at a time.  Index-resident arrays live in the HBM of
 * the device named at load; search workspaces are owned by the handle and
 * reused across calls (the reference re-allocates and frees them per call).
 *
 * The product path never falls back to the CPU: without a usable CUDA device
 * the entry points fail with MVR_ERR_CUDA.
 */
#ifndef MVR_H
#define MVR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MVR_OK = 0,
  MVR_ERR_INVALID_ARG = 1, /* bad size / shape / parameter */
  MVR_ERR_IO = 2,          /* file missing, unreadable or malformed */
  MVR_ERR_CUDA = 3,        /* CUDA runtime or kernel error, no device */
  MVR_ERR_OOM = 4,         /* device or host allocation failed */
  MVR_ERR_UNSUPPORTED = 5  /* valid for the reference, not supported here */
} mvr_status;

/* search flags */
#define MVR_SEM_PP 0u    /* rerank over each doc's true token count
                            (RerankPP.hpp:115-161) */
#define MVR_SEM_BASIC 1u /* rerank over docs zero-padded to the longest doc,
                            i.e. max(0, .) per query token for shorter docs
                            (Rerank.hpp:166-179,287-306) */
#define MVR_PREC_BF16 2u /* mixed precision: the shortlist is scored by the
                            BF16 tensor-core (tcgen05) MaxSim kernel with FP32
                            accumulation, and its best R docs are re-scored by
                            the exact FP32 kernel (R: mvr_index_set_rescore).
                            Returned scores are always exact FP32 MaxSim. */
#define MVR_PREC_FP8 4u  /* as MVR_PREC_BF16 with the shortlist scored in FP8
                            (E4M3) on the tensor cores: query tokens with
                            per-token power-of-two scales, centroid rows and
                            bucket weights as E4M3, FP32 accumulation; the
                            best R docs are re-scored exactly in FP32.
                            2- and 4-bit indexes; other code widths run the
                            BF16 kernel.  May be combined with MVR_SEM_BASIC. */

#define MVR_CAND_IMPUTE 8u /* candidate filter: a query token that visits no
                            probed list holding the doc adds its lowest probed
                            centroid score to the doc's approximate score
                            (the reference adds 0).  Ranks the shortlist
                            closer to the exact MaxSim; not a reference
                            option, so candidate scores then differ from the
                            reference's. */

#define MVR_PRUNE 16u /* learned candidate pruner (no counterpart in the
                          reference; needs a 2- or 4-bit index, queries of
                          up to 32 tokens and weights set by
                          mvr_index_set_pruner; alone, or with
                          MVR_PREC_FP8): after the shortlist, the pruner's
                          MLP predicts each shortlisted doc's MaxSim from its
                          features, and only the `keep` docs with the best
                          predictions are decompressed and scored -- by the
                          exact FP32 MaxSim (no precision flag) or by the FP8
                          MaxSim then the exact FP32 re-score (MVR_PREC_FP8)
                          -- unless the query's R-th best prediction (R = the
                          re-score count, 4 k by default) leads its keep-th
                          best by less than `margin` (low confidence), when
                          the whole shortlist is scored.  Returned scores are
                          always exact FP32 MaxSim. */

typedef struct mvr_index mvr_index;

typedef struct {
  uint32_t n_item, n_centroid, dim, n_bit;
  uint64_t n_vec, n_ele_ivf;
  uint32_t max_item_n_vec, max_ivf_list;
  uint64_t device_bytes; /* HBM held by the index arrays */
  int device;
} mvr_index_info;

typedef struct {
  double wall_s;          /* host wall time of the whole call */
  double device_ms;       /* CUDA-event time of the device pipeline */
  double batch_ms_max;    /* slowest batch (device time) */
  uint32_t n_batch;       /* query batches processed */
  uint32_t gpu_launches;  /* kernels launched by the call */
  uint64_t h2d_bytes, d2h_bytes;
  uint64_t n_cand_total;  /* sum over queries of candidate-set sizes */
  uint64_t n_rerank_tok;  /* sum over queries of reranked doc tokens */
  uint64_t n_list_ent;    /* sum over queries of probed IVF entries read */
  double stage_ms[6];     /* CUDA-event time summed over batches: query
                             copy, scoring + probe, filter, rerank (FP32 or
                             BF16 tensor-core), FP32 re-score + top-k,
                             result copy */
  uint64_t n_prune_fallback; /* MVR_PRUNE: queries whose whole shortlist was
                                scored (low-confidence predictions) */
} mvr_stats;

/* Per-query stage trace (parity tests).  Caller-owned host buffers. */
typedef struct {
  uint32_t *probe_id;    /* [nq*nprobe] per token, by (score desc, id asc) */
  float *probe_score;    /* [nq*nprobe] S = q.c + 1 */
  uint32_t cand_cap;     /* capacity of cand_id / cand_score */
  uint32_t n_cand;       /* out: candidate-set size */
  uint32_t *cand_id;     /* [cand_cap] candidate doc ids, ascending */
  float *cand_score;     /* [cand_cap] approximate score of cand_id[i] */
  uint32_t n_short;      /* out: shortlist size = min(probe_topk, n_cand) */
  uint32_t *short_id;    /* [probe_topk] shortlist, ascending doc id */
  float *short_approx;   /* [probe_topk] approximate score */
  float *short_exact;    /* [probe_topk] exact MaxSim */
  float *topk_score;     /* [topk] final result */
  uint32_t *topk_id;     /* [topk] */
  float *short_feat;     /* nullable [probe_topk][33]: learned-pruner features
                            of short_id[i] (FP8 index, <= 32 query tokens) */
  float *short_pred;     /* nullable [probe_topk]: the pruner's prediction
                            for short_id[i] (a pruner must be set) */
} mvr_trace;

/* Error text of the last failing call on this thread ("" if none). */
const char *mvr_last_error(void);

/* Number of visible CUDA devices (0 when none). */
int mvr_device_count(void);

/* Load the reference's on-disk index from `index_dir`:
 *   item_n_vec_l.npy  uint32 [n_item]          doc lengths
 *   centroid_l.npy    float32 [C, dim]
 *   vq_code_l.npy     int32/uint32 [n_vec]     token -> centroid
 *   weight_l.npy      float32 [2^n_bit]        bucket weights
 *   residual_code_l.npy uint8 [n_vec*dim*n_bit/8] MSB-first packed buckets
 *   ivf.index         binary CSR (IVFIndex.hpp:168-183)
 * Replaces IGPGPUPP(item_n_vec_l_fname, n_cpu_thread) + buildIndex(...)
 * (src/impl/IGPGPUPP.hpp:67-92,120-251) and the IGPGPUBasic equivalents
 * (src/impl/IGPGPUBasic.hpp:71-94,122-188).  n_centroid / n_bit must match
 * the files (the reference asserts the same).  dim must be 128. */
int mvr_index_load(const char *index_dir, uint32_t n_centroid, uint32_t n_bit,
                   int device, mvr_index **out);

/* Same, from the individual files (IGPGPUPP::buildIndex's argument list,
 * src/impl/IGPGPUPP.hpp:120-124, plus the item_n_vec_l file its constructor
 * takes). */
int mvr_index_load_files(const char *item_n_vec_l_fname,
                         const char *centroid_l_fname,
                         const char *vq_code_l_fname,
                         const char *ivf_index_fname,
                         const char *weight_l_fname,
                         const char *residual_code_l_fname,
                         uint32_t n_centroid, uint32_t n_bit, int device,
                         mvr_index **out);

/* Same index from host arrays (the contents of the files above; ivf as the
 * CSR triple offsets/sizes/ids).  Arrays are copied; the caller keeps them. */
int mvr_index_from_arrays(const uint32_t *item_n_vec_l, uint32_t n_item,
                          const float *centroid_l, uint32_t n_centroid,
                          uint32_t dim, const uint32_t *vq_code_l,
                          uint64_t n_vec, const uint64_t *ivf_offset_l,
                          const uint32_t *ivf_size_l, const uint32_t *ivf,
                          uint64_t n_ele_ivf, const float *weight_l,
                          uint32_t n_bit, const uint8_t *residual_code_l,
                          int device, mvr_index **out);

/* Same, from arrays already resident on `device` (device pointers; copied
 * device-to-device), e.g. an index built on the GPU. */
int mvr_index_from_device_arrays(const uint32_t *item_n_vec_l, uint32_t n_item,
                                 const float *centroid_l, uint32_t n_centroid,
                                 uint32_t dim, const uint32_t *vq_code_l,
                                 uint64_t n_vec, const uint64_t *ivf_offset_l,
                                 const uint32_t *ivf_size_l, const uint32_t *ivf,
                                 uint64_t n_ele_ivf, const float *weight_l,
                                 uint32_t n_bit,
                                 const uint8_t *residual_code_l, int device,
                                 mvr_index **out);

int mvr_index_free(mvr_index *h);
int mvr_index_get_info(const mvr_index *h, mvr_index_info *info);

/* Queries per device batch (default chosen from the index size). */
int mvr_index_set_batch(mvr_index *h, uint32_t max_batch_queries);

/* Docs per query that the MVR_PREC_BF16 path re-scores exactly in FP32
 * (0 = default 4 * topk; clamped to [topk, probe_topk]). */
int mvr_index_set_rescore(mvr_index *h, uint32_t n_rescore);

/* CUDA graphs for repeated device-buffer searches (no counterpart in the
 * reference, whose search loop launches every stage from the host per
 * query; enable = 0 by default).  With graphs on, mvr_search_device records
 * the whole call -- every batch's probe, filter, rerank, re-score and top-k
 * kernels, on the handle's own stream, ordered after the caller's stream --
 * as one CUDA graph the first time, and replays it while the call repeats
 * (same query / result pointers, query count and token offsets, topk,
 * nprobe, probe_topk, flags, re-score width and batch size); any change
 * records a new graph.  The host buffers of mvr_search are not captured. */
int mvr_index_set_graphs(mvr_index *h, int enable);

/* Batched search with HOST buffers (queries in, results out; copies inside).
 * query_l: float32 tokens, query i = rows [tok_off[i], tok_off[i+1]) of a
 * [*, dim] matrix; tok_off == NULL means every query has query_n_vec tokens
 * (the reference's uniform layout, IGPGPUPP::search src/impl/IGPGPUPP.hpp:
 * 253-331).  1 <= tokens per query <= 64, 1 <= nprobe <= min(32, C),
 * topk <= probe_topk <= 8192, topk <= 1024 (probe_topk >= topk is the
 * reference's own check, IGPGPUPP.hpp:256-259).  Results per query are
 * sorted by (score desc, doc id asc); when fewer than topk docs qualify the
 * tail holds id 0xffffffff and score -inf.  query_time_s (nullable) receives
 * each query's batch latency in seconds. */
int mvr_search(mvr_index *h, const float *query_l, const uint64_t *tok_off,
               uint32_t n_query, uint32_t query_n_vec, uint32_t topk,
               uint32_t nprobe, uint32_t probe_topk, uint32_t flags,
               float *result_score_l, uint32_t *result_id_l,
               double *query_time_s, mvr_stats *stats);

/* mvr_search plus per-query stage times (seconds, of the query's batch):
 * stage_time_s[i*6 + k], k = 0 query copy, 1 centroid scoring + probe,
 * 2 candidate filter + shortlist, 3 rerank, 4 re-score + top-k, 5 result
 * copy -- the stage columns of the reference's performance TSV
 * (IGPGPUBasic.cpp:183-204). */
int mvr_search_staged(mvr_index *h, const float *query_l,
                      const uint64_t *tok_off, uint32_t n_query,
                      uint32_t query_n_vec, uint32_t topk, uint32_t nprobe,
                      uint32_t probe_topk, uint32_t flags,
                      float *result_score_l, uint32_t *result_id_l,
                      double *query_time_s, double *stage_time_s,
                      mvr_stats *stats);

/* Same search with DEVICE buffers already resident on the index's device;
 * tok_off stays a host array.  Runs on `cuda_stream` (NULL: the legacy
 * default stream) and returns after the results are written (the stream is
 * synchronised). */
int mvr_search_device(mvr_index *h, const float *d_query_l,
                      const uint64_t *tok_off, uint32_t n_query,
                      uint32_t query_n_vec, uint32_t topk, uint32_t nprobe,
                      uint32_t probe_topk, uint32_t flags,
                      float *d_result_score_l, uint32_t *d_result_id_l,
                      void *cuda_stream, mvr_stats *stats);

/* One query through the same kernels with every stage's output copied back
 * (parity tests).  query: host float32 [nq, dim]. */
int mvr_search_trace(mvr_index *h, const float *query, uint32_t nq,
                     uint32_t topk, uint32_t nprobe, uint32_t probe_topk,
                     uint32_t flags, mvr_trace *trace);

/* ---- learned candidate pruner (no counterpart in the reference) ----
 * An MLP 33 -> 256 -> 256 -> 1 with GELU (tanh form) over per-candidate
 * features -- per query token (up to 32) the best centroid score among the
 * doc's tokens' centroids, then log(doc length) -- predicting each
 * shortlisted doc's exact MaxSim.  Parameters: one float vector of
 * MVR_MLP_NUM_PARAMS values, W1 [256][33], b1 [256], W2 [256][256],
 * b2 [256], w3 [256], b3; weights are applied rounded to BF16 with FP32
 * accumulation. */
#define MVR_MLP_NUM_PARAMS 74753u
#define MVR_MLP_FEAT 33u

/* Training workspace, in floats, for minibatches of n rows. */
size_t mvr_mlp_work_floats(uint32_t n);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8, learning rate lr; step counts
 * from 1) on the loss 0.5 * mean((mlp(x) - y)^2) of a minibatch, with the
 * library's hand-written kernels.  Device buffers: d_x [n][33], d_y [n],
 * d_params / d_adam_m / d_adam_v [MVR_MLP_NUM_PARAMS] (updated in place),
 * d_work [mvr_mlp_work_floats(n)], d_loss (nullable, one float: the
 * minibatch loss before the step).  Synchronises cuda_stream. */
int mvr_mlp_train_step(const float *d_x, const float *d_y, uint32_t n,
                       float *d_params, float *d_adam_m, float *d_adam_v,
                       float *d_work, float lr, uint32_t step, float *d_loss,
                       void *cuda_stream);

/* The MLP's forward pass on CUDA cores (the training kernels' arithmetic):
 * d_out [n] from d_x [n][33]; d_work as for training. */
int mvr_mlp_forward(const float *d_x, uint32_t n, const float *d_params,
                    float *d_work, float *d_out, void *cuda_stream);

/* Sets the learned pruner of a handle (MVR_PRUNE): params = host float
 * [MVR_MLP_NUM_PARAMS] (NULL removes it), keep = docs scored per query when
 * the predictions are confident (1..probe_topk of the searches), margin =
 * the confidence threshold (prediction units). */
int mvr_index_set_pruner(mvr_index *h, const float *params, uint32_t keep,
                         float margin);

/* Tile shape of the FP8 MaxSim kernel (MVR_PREC_FP8): shortlisted docs per
 * CTA, 32, 64, 128 or 256 (0: the default, 256; queries of more than 32
 * tokens use at most 128); chosen by the library's tuner
 * (mvr.tune.tune_tile).  No counterpart in the reference. */
int mvr_index_set_rerank_tile(mvr_index *h, uint32_t docs_per_cta);

/* Failure detection (test hook; no counterpart in the reference, whose
 * kernels have no bounded waits): the time bound of every pipeline wait of
 * the FP8 MaxSim kernel and of the exact FP32 MaxSim kernel, in ns (0
 * restores the default, 1 s).  A wait that runs out stops the kernel, which
 * still lets its own copies and MMAs finish and frees its tensor memory; the
 * search then fails with MVR_ERR_CUDA and the handle stays usable.  Tests set
 * a tiny bound to make a wait run out. */
int mvr_index_set_wait_limit(mvr_index *h, uint64_t wait_ns);

/* Candidate filter for ONE query with no device allocation in the call: the
 * probe lists -> candidate set -> approximate scores -> top-probe_topk
 * shortlist stage of mvr_search, its scratch held in a fixed array compiled
 * into libmvr (about 11 MB on every GPU that loads the library, kept until
 * the process exits).  No counterpart in the reference: it is for callers
 * that cannot allocate device memory while serving (a plugin inside a host
 * whose GPU memory is all reserved by the host's own pool allocator, or a
 * latency-critical caller that cannot afford cudaMalloc's implicit device
 * synchronisation).  Inputs and outputs are the caller's DEVICE buffers:
 * d_probe_id / d_probe_score [nq*nprobe], the token-major probe lists sorted
 * best-first as mvr_search_trace returns them; d_short_id /
 * d_short_approx [probe_topk] (unordered) and d_n_short [1].  Limits:
 * index of at most 262,144 docs, 1..32 query tokens; larger sizes fail with
 * MVR_ERR_INVALID_ARG.  Runs asynchronously on cuda_stream.  All calls on a
 * device share the array: calls whose GPU work overlaps race -- serialise
 * them.  The first call on a device does the one-time set-up (looks up the
 * array's device address); make it before any stream capture.  The address
 * is cached for the life of the process: after a cudaDeviceReset on that
 * device it no longer points at the array, so do not call this entry point
 * again in a process that has reset the device. */
int mvr_filter_noalloc(mvr_index *h, const uint32_t *d_probe_id,
                       const float *d_probe_score, uint32_t nq,
                       uint32_t nprobe, uint32_t probe_topk,
                       uint32_t *d_short_id, float *d_short_approx,
                       uint32_t *d_n_short, void *cuda_stream);

/* Decompressed token vectors x = centroid[code] + W[bucket] for the given
 * global token ids (host in/out, out: float32 [n, dim]); the decoder of
 * decompressAndAddResidual (RerankPP.hpp:65-113). */
int mvr_decompress(mvr_index *h, const uint64_t *vec_id, uint64_t n,
                   float *out);

/* Bucket index of every dimension of the given tokens (host out: uint8
 * [n, dim]), unpacked on the device by the rerank decoder's bit layout. */
int mvr_unpack_buckets(mvr_index *h, const uint64_t *vec_id, uint64_t n,
                       uint8_t *out);

/* ---- index build (device pointers; GPU counterpart of the reference's
 *      build pipeline, vq_sq_pack.py:30-109 and
 *      ResidualScalarQuantizationPackGPU.hpp:30-80) ---- */

/* code[i] = argmax_c dot(vec_i, centroid_c), lowest id on ties; score[i]
 * (nullable) = that max + 1.  FP32, canonical dot order. */
int mvr_assign_device(const float *d_vec, uint64_t n_vec,
                      const float *d_centroid, uint32_t n_centroid,
                      uint32_t dim, uint32_t *d_code, float *d_score,
                      void *cuda_stream);

/* mvr_assign_device on the tensor cores, for large builds: BF16 tcgen05
 * scoring keeps each vector's 16 best centroids per centroid split, which are
 * re-scored with the canonical FP32 dot; code[i] is the best of those (equal
 * to mvr_assign_device's unless the true best missed the BF16 candidates),
 * score[i] (nullable) its FP32 score + 1. */
int mvr_assign_tc_device(const float *d_vec, uint64_t n_vec,
                         const float *d_centroid, uint32_t n_centroid,
                         uint32_t dim, uint32_t *d_code, float *d_score,
                         void *cuda_stream);

/* Packed residual bytes (MSB-first, bucket = #cutoffs <= vec - centroid):
 * out [n_vec * dim*n_bit/8]. */
int mvr_pack_residual_device(const float *d_vec, uint64_t n_vec,
                             const float *d_centroid, uint32_t dim,
                             const uint32_t *d_code, const float *cutoff_l,
                             uint32_t n_bit, uint8_t *d_out,
                             void *cuda_stream);

/* Bucket cutoffs and weights of the residual quantizer (GPU counterpart of
 * ComputeQuantizedScalarPack, ResidualScalarQuantizationPack.hpp:17-100):
 * over all n_vec * 128 residual errors e = vec - centroid[code] (one rounded
 * FP32 subtraction), cutoff_out[c] (host, 2^n_bit - 1 values) = the
 * floor((c + 1) / 2^n_bit * N)-th smallest, weight_out[w] (host, 2^n_bit
 * values) = the floor((w + 0.5) / 2^n_bit * N)-th smallest (0-based ranks,
 * the reference's nth_element positions), selected exactly by two
 * histogram passes over order keys. */
int mvr_residual_quantiles_device(const float *d_vec, uint64_t n_vec,
                                  const float *d_centroid, uint32_t dim,
                                  const uint32_t *d_code, uint32_t n_bit,
                                  float *cutoff_out, float *weight_out,
                                  void *cuda_stream);

/* FP64 k-means update: sum[c][d] += vec[i][d] and count[c] += 1 over
 * code[i] == c (double accumulation; caller zeroes sum/count). */
int mvr_kmeans_accumulate_device(const float *d_vec, uint64_t n_vec,
                                 uint32_t dim, const uint32_t *d_code,
                                 double *d_sum, uint64_t *d_count,
                                 void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* MVR_H */
