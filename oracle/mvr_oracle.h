/*
 * mvr_oracle.h -- CPU restatement of the reference's GPU multi-vector search
 * path, used ONLY as test infrastructure: the checker in tests/, the smoke()
 * cross-check and the cpu_baseline / reference leg of bench.py.  Nothing in
 * the product (libmvr) links or calls this code.
 *
 * Parity status:
 *   - codec (decode table, bucket unpack, quantile cutoffs/weights, residual
 *     packing) and the IVF build / ivf.index byte layout are PINNED against the
 *     reference's own C++ (ResidualScalarQuantizationPack.hpp, IVFIndex.hpp)
 *     compiled from its sources into oracle/_ref and frozen as golden fixtures
 *     under tests/golden/.
 *   - the search stages (probe, candidate filter, shortlist, rerank, top-k)
 *     restate src/include/alg/igp_gpu_pp/{GenerateVQScoreCandidatePP,FilterPP,
 *     RerankPP,IGPGPURetrievalPP}.hpp, whose GPU code needs RAFT 25.04 (absent)
 *     and so cannot run here: those stages are "parity unpinned" against the
 *     reference binary; the reference ships no golden vectors for them.
 *
 * Canonical arithmetic (the contract the CUDA path reproduces bit-for-bit):
 *   dot(a,b)   = sequential fmaf over d = 0..D-1 starting from 0.0f
 *   S[q][c]    = dot(q, c) + 1.0f                       (single FP32 add)
 *   probe      = top-nprobe per query token by (S desc, centroid id asc)
 *   approx[c]  = sum over q of the score of the highest-ranked probe of
 *                token q whose IVF list holds doc c, summed exactly in 2^-32
 *                fixed point (int64) and rounded once to FP32
 *   shortlist  = top-probe_topk candidates by (approx desc, doc id asc)
 *   x[t][d]    = centroid[code_t][d] + W[bucket(t,d)]   (single FP32 add)
 *   maxsim     = sum over q (in order, FP32, from 0.0f) of max_t dot(q, x_t)
 *   top-k      = by (score desc, doc id asc)
 */
#ifndef MVR_ORACLE_H
#define MVR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* rerank semantics: PP uses the true doc length (RerankPP.hpp:141-157);
 * BASIC pads every doc to max_item_n_vec with zero rows (Rerank.hpp:166-179,
 * 293-306), i.e. max(0, .) for docs shorter than the longest doc. */
enum { ORC_SEM_PP = 0, ORC_SEM_BASIC = 1 };
/* search flag (OR-ed into semantics; not a reference option): approximate
 * scores impute an unmatched query token with its lowest probed score */
enum { ORC_CAND_IMPUTE = 8 };

typedef struct {
  uint32_t n_item, n_centroid, dim, n_bit;
  uint64_t n_vec, n_ele_ivf;
  const uint32_t *item_n_vec;   /* [n_item] */
  const uint64_t *item_off;     /* [n_item] prefix sums of item_n_vec */
  const float *centroid;        /* [n_centroid][dim] */
  const uint32_t *vq_code;      /* [n_vec] */
  const uint8_t *residual;      /* [n_vec][dim*n_bit/8] */
  const float *weight;          /* [2^n_bit] */
  const uint64_t *ivf_off;      /* [n_centroid] */
  const uint32_t *ivf_size;     /* [n_centroid] */
  const uint32_t *ivf_ids;      /* [n_ele_ivf] */
  uint32_t max_item_n_vec;
} orc_index;

typedef struct {
  /* filled by orc_search_one when non-NULL */
  uint32_t *probe_id;     /* [nq*nprobe] */
  float *probe_score;     /* [nq*nprobe] */
  uint32_t cand_cap;
  uint32_t n_cand;        /* out */
  uint32_t *cand_id;      /* [cand_cap] ascending doc id */
  float *cand_score;      /* [cand_cap] approximate score */
  uint32_t n_short;       /* out */
  uint32_t *short_id;     /* [probe_topk] by (approx desc, id asc) */
  float *short_approx;    /* [probe_topk] */
  float *short_exact;     /* [probe_topk] exact MaxSim of short_id */
} orc_trace;

/* ---- codec ---------------------------------------------------------- */
void orc_decode_table(uint32_t n_bit, const float *weight, float *out);
void orc_unpack_buckets(const uint8_t *residual, uint64_t n_vec, uint32_t dim,
                        uint32_t n_bit, uint8_t *out);
void orc_decompress(const orc_index *ix, const uint64_t *vec_id, uint64_t n,
                    float *out);
void orc_decompress_item(const orc_index *ix, uint32_t item, float *out);
int orc_quantize(const float *vec, uint64_t n_vec, uint32_t dim,
                 const float *centroid, const uint32_t *code, uint32_t n_bit,
                 float *cutoff_out, float *weight_out);
void orc_pack_residual(const float *vec, uint64_t n_vec, uint32_t dim,
                       const float *centroid, const uint32_t *code,
                       const float *cutoff, uint32_t n_bit, uint8_t *out);
uint64_t orc_ivf_build(const uint32_t *code, const uint32_t *item_n_vec,
                       uint32_t n_item, uint32_t n_centroid, uint64_t *off,
                       uint32_t *size, uint32_t *ids);

/* ---- search stages -------------------------------------------------- */
int64_t orc_fixed(float v);
float orc_unfixed(int64_t acc);
void orc_centroid_scores(const float *q, uint32_t nq, const float *centroid,
                         uint32_t n_centroid, uint32_t dim, float *S);
void orc_assign(const float *vec, uint64_t n_vec, const float *centroid,
                uint32_t n_centroid, uint32_t dim, int n_threads,
                uint32_t *code);
void orc_probe(const float *S, uint32_t nq, uint32_t n_centroid,
               uint32_t nprobe, uint32_t *id, float *score);
float orc_maxsim_item(const orc_index *ix, const float *q, uint32_t nq,
                      uint32_t item, int semantics);
double orc_maxsim_f64(const float *q, uint32_t nq, const float *tok,
                      uint32_t n_tok, uint32_t dim);
int orc_search_one(const orc_index *ix, const float *q, uint32_t nq,
                   uint32_t topk, uint32_t nprobe, uint32_t probe_topk,
                   int semantics, orc_trace *tr, float *out_score,
                   uint32_t *out_id);
int orc_search(const orc_index *ix, const float *q, const uint64_t *q_tok_off,
               uint32_t n_query, uint32_t topk, uint32_t nprobe,
               uint32_t probe_topk, int semantics, int n_threads,
               float *out_score, uint32_t *out_id);
/* exhaustive FP64 MaxSim over raw token embeddings (GPUComputeScore.hpp:
 * 209-264 semantics) returning top-k by (score desc, id asc) */
int orc_exhaustive_f64(const float *q, const uint64_t *q_tok_off,
                       uint32_t n_query, const float *tok,
                       const uint32_t *item_n_vec, const uint64_t *item_off,
                       uint32_t n_item, uint32_t dim, uint32_t topk,
                       int n_threads, double *out_score, uint32_t *out_id);

#ifdef __cplusplus
}
#endif
#endif
