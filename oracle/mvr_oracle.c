/*
 * mvr_oracle.c -- CPU restatement (test infrastructure only) of the
 * reference's GPU multi-vector search path and its residual codec.  See
 * mvr_oracle.h for the parity status of each part and for the canonical
 * arithmetic that the CUDA path reproduces bit-for-bit.
 *
 * Build: oracle/Makefile  (gcc -O3 -mavx2 -mfma -ffp-contract=off -fopenmp)
 * -ffp-contract=off matters: every multiply-add on the canonical path is an
 * explicit fmaf, every other add/multiply is rounded on its own.
 */
#include "mvr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FMA(a, b, c) __builtin_fmaf((a), (b), (c))

/* ------------------------------------------------------------------ */
/* codec                                                              */
/* ------------------------------------------------------------------ */

/* Byte -> per-value weight table, MSB-first:
 * value i of a packed byte is (byte >> (8 - b*(i+1))) & (2^b - 1).
 * Restates SQInfoPP ctor + decompressSQPackedCode (DataStructPP.hpp:150-187)
 * and ResidualCodePack ctor (ResidualScalarQuantizationPack.hpp:296-328). */
void orc_decode_table(uint32_t n_bit, const float *weight, float *out) {
  const uint32_t vpb = 8u / n_bit;
  const uint32_t mask = (1u << n_bit) - 1u;
  for (uint32_t code = 0; code < 256; code++)
    for (uint32_t i = 0; i < vpb; i++)
      out[code * vpb + i] = weight[(code >> (8u - n_bit * (i + 1u))) & mask];
}

void orc_unpack_buckets(const uint8_t *residual, uint64_t n_vec, uint32_t dim,
                        uint32_t n_bit, uint8_t *out) {
  const uint32_t vpb = 8u / n_bit;
  const uint32_t bpv = (dim + vpb - 1u) / vpb;
  const uint32_t mask = (1u << n_bit) - 1u;
  for (uint64_t v = 0; v < n_vec; v++)
    for (uint32_t d = 0; d < dim; d++) {
      const uint8_t byte = residual[v * bpv + d / vpb];
      const uint32_t i = d % vpb;
      out[v * dim + d] = (uint8_t)((byte >> (8u - n_bit * (i + 1u))) & mask);
    }
}

/* x[d] = centroid[code][d] + W[bucket(d)]  (decompressAndAddResidual,
 * RerankPP.hpp:65-113; ResidualCodePack::Decode,
 * ResidualScalarQuantizationPack.hpp:351-378) */
static void decompress_vec(const orc_index *ix, const float *table,
                           uint64_t v, float *out) {
  const uint32_t dim = ix->dim, vpb = 8u / ix->n_bit;
  const uint32_t bpv = (dim + vpb - 1u) / vpb;
  const float *c = ix->centroid + (uint64_t)ix->vq_code[v] * dim;
  const uint8_t *r = ix->residual + v * bpv;
  for (uint32_t d = 0; d < dim; d++) {
    const float w = table[(uint32_t)r[d / vpb] * vpb + d % vpb];
    out[d] = c[d] + w;
  }
}

void orc_decompress(const orc_index *ix, const uint64_t *vec_id, uint64_t n,
                    float *out) {
  float table[256 * 8];
  orc_decode_table(ix->n_bit, ix->weight, table);
  for (uint64_t i = 0; i < n; i++)
    decompress_vec(ix, table, vec_id[i], out + i * ix->dim);
}

void orc_decompress_item(const orc_index *ix, uint32_t item, float *out) {
  float table[256 * 8];
  orc_decode_table(ix->n_bit, ix->weight, table);
  const uint64_t off = ix->item_off[item];
  for (uint32_t t = 0; t < ix->item_n_vec[item]; t++)
    decompress_vec(ix, table, off + t, out + (uint64_t)t * ix->dim);
}

static int cmp_float(const void *a, const void *b) {
  const float x = *(const float *)a, y = *(const float *)b;
  return (x > y) - (x < y);
}

/* Quantile cutoffs / weights from order statistics of all residual
 * coordinates (ComputeQuantizedScalarPack, ResidualScalarQuantizationPack.hpp:
 * 17-99): cutoff_i = e_(floor(i/2^b * N)), i = 1..2^b-1;
 * weight_i = e_(floor((i/2^b + 0.5/2^b) * N)), i = 0..2^b-1, where e_(k) is
 * the k-th smallest (0-based) residual error vec[d] - centroid[d] (FP32). */
int orc_quantize(const float *vec, uint64_t n_vec, uint32_t dim,
                 const float *centroid, const uint32_t *code, uint32_t n_bit,
                 float *cutoff_out, float *weight_out) {
  const uint64_t n = n_vec * dim;
  float *err = (float *)malloc(n * sizeof(float));
  if (!err) return -1;
  for (uint64_t v = 0; v < n_vec; v++) {
    const float *c = centroid + (uint64_t)code[v] * dim;
    for (uint32_t d = 0; d < dim; d++) err[v * dim + d] = vec[v * dim + d] - c[d];
  }
  qsort(err, n, sizeof(float), cmp_float);
  const uint32_t nq = 1u << n_bit;
  for (uint32_t i = 0; i + 1 < nq; i++) {
    const double quantile = 1.0 * (i + 1) / nq;
    const uint64_t idx = (uint64_t)floor(quantile * (double)n);
    cutoff_out[i] = err[idx];
  }
  for (uint32_t i = 0; i < nq; i++) {
    const double quantile = 1.0 * i / nq + 0.5 / nq;
    const uint64_t idx = (uint64_t)floor(quantile * (double)n);
    weight_out[i] = err[idx];
  }
  free(err);
  return 0;
}

/* bucket = number of cutoffs <= error (first cutoff > error), packed
 * MSB-first (CompressResidualCode::compute_residual_code / compress,
 * ResidualScalarQuantizationPack.hpp:154-236; compressSQCode,
 * ResidualScalarQuantizationPackGPU.hpp:30-80). */
void orc_pack_residual(const float *vec, uint64_t n_vec, uint32_t dim,
                       const float *centroid, const uint32_t *code,
                       const float *cutoff, uint32_t n_bit, uint8_t *out) {
  const uint32_t vpb = 8u / n_bit;
  const uint32_t bpv = (dim + vpb - 1u) / vpb;
  const uint32_t n_cut = (1u << n_bit) - 1u;
  const uint32_t mask = (1u << n_bit) - 1u;
  for (uint64_t v = 0; v < n_vec; v++) {
    const float *c = centroid + (uint64_t)code[v] * dim;
    for (uint32_t p = 0; p < bpv; p++) {
      uint32_t byte = 0;
      for (uint32_t i = 0; i < vpb; i++) {
        const uint32_t d = p * vpb + i;
        uint32_t b = 0;
        if (d < dim) {
          const float e = vec[v * dim + d] - c[d];
          b = n_cut;
          for (uint32_t k = 0; k < n_cut; k++)
            if (cutoff[k] > e) { b = k; break; }
        }
        byte = (byte << n_bit) | (b & mask);
      }
      out[v * bpv + p] = (uint8_t)byte;
    }
  }
}

/* doc -> unique centroid inverted lists, ascending doc ids per list
 * (IVFIndex::build, IVFIndex.hpp:92-166).  Returns n_ele; off/size/ids may be
 * NULL to size the output. */
uint64_t orc_ivf_build(const uint32_t *code, const uint32_t *item_n_vec,
                       uint32_t n_item, uint32_t n_centroid, uint64_t *off,
                       uint32_t *size, uint32_t *ids) {
  uint32_t *cnt = (uint32_t *)calloc(n_centroid, sizeof(uint32_t));
  uint32_t *stamp = (uint32_t *)malloc(n_centroid * sizeof(uint32_t));
  memset(stamp, 0xff, n_centroid * sizeof(uint32_t));
  uint64_t pos = 0;
  for (uint32_t it = 0; it < n_item; it++) {
    for (uint32_t t = 0; t < item_n_vec[it]; t++) {
      const uint32_t c = code[pos + t];
      if (stamp[c] != it) { stamp[c] = it; cnt[c]++; }
    }
    pos += item_n_vec[it];
  }
  uint64_t n_ele = 0;
  for (uint32_t c = 0; c < n_centroid; c++) n_ele += cnt[c];
  if (off && size && ids) {
    uint64_t acc = 0;
    for (uint32_t c = 0; c < n_centroid; c++) { off[c] = acc; size[c] = cnt[c]; acc += cnt[c]; }
    uint64_t *fill = (uint64_t *)malloc(n_centroid * sizeof(uint64_t));
    for (uint32_t c = 0; c < n_centroid; c++) fill[c] = off[c];
    memset(stamp, 0xff, n_centroid * sizeof(uint32_t));
    pos = 0;
    for (uint32_t it = 0; it < n_item; it++) {
      for (uint32_t t = 0; t < item_n_vec[it]; t++) {
        const uint32_t c = code[pos + t];
        if (stamp[c] != it) { stamp[c] = it; ids[fill[c]++] = it; }
      }
      pos += item_n_vec[it];
    }
    free(fill);
  }
  free(cnt);
  free(stamp);
  return n_ele;
}

/* ------------------------------------------------------------------ */
/* search stages                                                      */
/* ------------------------------------------------------------------ */

/* centroid block transposed to [dim][16] so that the 16 sequential fmaf
 * chains vectorise across centroids without changing any rounding. */
#define CB 16
static void score_token(const float *q, const float *centroid,
                        uint32_t n_centroid, uint32_t dim, float *S) {
  float blk[256 * CB];
  for (uint32_t c0 = 0; c0 < n_centroid; c0 += CB) {
    const uint32_t nc = (n_centroid - c0 < CB) ? n_centroid - c0 : CB;
    for (uint32_t j = 0; j < CB; j++)
      for (uint32_t d = 0; d < dim; d++)
        blk[d * CB + j] = (j < nc) ? centroid[(uint64_t)(c0 + j) * dim + d] : 0.0f;
    float acc[CB];
    for (uint32_t j = 0; j < CB; j++) acc[j] = 0.0f;
    for (uint32_t d = 0; d < dim; d++) {
      const float qd = q[d];
#pragma omp simd
      for (uint32_t j = 0; j < CB; j++) acc[j] = FMA(qd, blk[d * CB + j], acc[j]);
    }
    for (uint32_t j = 0; j < nc; j++) S[c0 + j] = acc[j] + 1.0f;
  }
}

/* S = Q.C^T + 1 (MatrixMultiply + thrust +1, GenerateVQScoreCandidatePP.hpp:
 * 137-144) with the canonical sequential-fmaf dot product. */
void orc_centroid_scores(const float *q, uint32_t nq, const float *centroid,
                         uint32_t n_centroid, uint32_t dim, float *S) {
  for (uint32_t t = 0; t < nq; t++)
    score_token(q + (uint64_t)t * dim, centroid, n_centroid, dim,
                S + (uint64_t)t * n_centroid);
}

/* arg max_c dot(vec, c), lowest id on ties (vq_sq_pack.py compute_assignment
 * argmax semantics). */
void orc_assign(const float *vec, uint64_t n_vec, const float *centroid,
                uint32_t n_centroid, uint32_t dim, int n_threads,
                uint32_t *code) {
#pragma omp parallel num_threads(n_threads > 0 ? n_threads : 1)
  {
    float *S = (float *)malloc(n_centroid * sizeof(float));
#pragma omp for schedule(dynamic, 64)
    for (int64_t v = 0; v < (int64_t)n_vec; v++) {
      score_token(vec + (uint64_t)v * dim, centroid, n_centroid, dim, S);
      uint32_t best = 0;
      for (uint32_t c = 1; c < n_centroid; c++)
        if (S[c] > S[best]) best = c;
      code[v] = best;
    }
    free(S);
  }
}

static int better(float s1, uint32_t i1, float s2, uint32_t i2) {
  return s1 > s2 || (s1 == s2 && i1 < i2);
}

/* top-nprobe per token, sorted by (score desc, id asc) -- the order RAFT's
 * select_k (GenerateVQScoreCandidatePP.hpp:166-174) leaves unspecified. */
void orc_probe(const float *S, uint32_t nq, uint32_t n_centroid,
               uint32_t nprobe, uint32_t *id, float *score) {
  for (uint32_t t = 0; t < nq; t++) {
    const float *row = S + (uint64_t)t * n_centroid;
    uint32_t *pid = id + t * nprobe;
    float *ps = score + t * nprobe;
    uint32_t n = 0;
    for (uint32_t c = 0; c < n_centroid; c++) {
      const float s = row[c];
      if (n == nprobe && !better(s, c, ps[n - 1], pid[n - 1])) continue;
      uint32_t k = (n < nprobe) ? n++ : nprobe - 1;
      while (k > 0 && better(s, c, ps[k - 1], pid[k - 1])) {
        ps[k] = ps[k - 1];
        pid[k] = pid[k - 1];
        k--;
      }
      ps[k] = s;
      pid[k] = c;
    }
  }
}

/* exact MaxSim of one query against one item's decompressed tokens
 * (RerankPP::RerankFunc, RerankPP.hpp:368-475; BASIC: Rerank.hpp:236-339). */
static float maxsim_tokens(const float *qt /*[dim][nq]*/, uint32_t nq,
                           const float *x, uint32_t n_tok, uint32_t dim,
                           int clamp_zero, float *m /*[nq]*/) {
  float acc[64];
  for (uint32_t q = 0; q < nq; q++) m[q] = -INFINITY;
  for (uint32_t t = 0; t < n_tok; t++) {
    const float *xt = x + (uint64_t)t * dim;
    for (uint32_t q = 0; q < nq; q++) acc[q] = 0.0f;
    for (uint32_t d = 0; d < dim; d++) {
      const float xd = xt[d];
#pragma omp simd
      for (uint32_t q = 0; q < 64; q++) acc[q] = FMA(qt[d * 64 + q], xd, acc[q]);
    }
    for (uint32_t q = 0; q < nq; q++) m[q] = fmaxf(m[q], acc[q]);
  }
  float s = 0.0f;
  for (uint32_t q = 0; q < nq; q++) {
    const float mq = clamp_zero ? fmaxf(m[q], 0.0f) : m[q];
    s = s + mq;
  }
  return s;
}

static void transpose_query(const float *q, uint32_t nq, uint32_t dim,
                            float *qt) {
  for (uint32_t d = 0; d < dim; d++)
    for (uint32_t k = 0; k < 64; k++)
      qt[d * 64 + k] = (k < nq) ? q[(uint64_t)k * dim + d] : 0.0f;
}

float orc_maxsim_item(const orc_index *ix, const float *q, uint32_t nq,
                      uint32_t item, int semantics) {
  const uint32_t L = ix->item_n_vec[item];
  float *qt = (float *)malloc((size_t)ix->dim * 64 * sizeof(float));
  float *x = (float *)malloc((size_t)(L ? L : 1) * ix->dim * sizeof(float));
  float m[64];
  transpose_query(q, nq, ix->dim, qt);
  orc_decompress_item(ix, item, x);
  const int clamp = semantics == ORC_SEM_BASIC && L < ix->max_item_n_vec;
  const float s = maxsim_tokens(qt, nq, x, L, ix->dim, clamp, m);
  free(qt);
  free(x);
  return s;
}

double orc_maxsim_f64(const float *q, uint32_t nq, const float *tok,
                      uint32_t n_tok, uint32_t dim) {
  double s = 0.0;
  for (uint32_t a = 0; a < nq; a++) {
    double m = -INFINITY;
    for (uint32_t t = 0; t < n_tok; t++) {
      double ip = 0.0;
      for (uint32_t d = 0; d < dim; d++)
        ip += (double)q[(uint64_t)a * dim + d] * (double)tok[(uint64_t)t * dim + d];
      if (ip > m) m = ip;
    }
    s += m;
  }
  return s;
}

typedef struct { float s; uint32_t id; } scored;

/* Fixed-point approximate-score terms: v * 2^32 rounded to nearest-even
 * (exact for |v| >= 2^-9 since FP32 has a 24-bit significand), clamped to
 * +-2^30 * 2^32 so that 64 terms cannot overflow; the sum converts back by
 * one round-to-nearest int64 -> float conversion and an exact 2^-32 scale. */
int64_t orc_fixed(float v) {
  double x = (double)v * 4294967296.0;
  const double lim = 4611686018427387904.0; /* 2^62 */
  if (x > lim) x = lim;
  if (x < -lim) x = -lim;
  return (int64_t)llrint(x);
}
float orc_unfixed(int64_t acc) { return (float)acc * (1.0f / 4294967296.0f); }

static int cmp_scored(const void *a, const void *b) {
  const scored *x = (const scored *)a, *y = (const scored *)b;
  if (better(x->s, x->id, y->s, y->id)) return -1;
  if (better(y->s, y->id, x->s, x->id)) return 1;
  return 0;
}

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

typedef struct {
  uint8_t *rank;   /* [n_item][nq] 0xff = not hit */
  uint8_t *seen;   /* [n_item] */
  uint32_t *cand;  /* [n_item] */
  float *S;        /* [nq][n_centroid] */
  float *qt;       /* [dim][64] */
  float *x;        /* [max_item_n_vec][dim] */
  scored *sc;      /* [n_item] */
} orc_ws;

static int ws_init(orc_ws *w, const orc_index *ix, uint32_t nq) {
  memset(w, 0, sizeof(*w));
  w->rank = (uint8_t *)malloc((size_t)ix->n_item * nq);
  w->seen = (uint8_t *)calloc(ix->n_item, 1);
  w->cand = (uint32_t *)malloc((size_t)ix->n_item * sizeof(uint32_t));
  w->S = (float *)malloc((size_t)nq * ix->n_centroid * sizeof(float));
  w->qt = (float *)malloc((size_t)ix->dim * 64 * sizeof(float));
  w->x = (float *)malloc((size_t)(ix->max_item_n_vec + 1) * ix->dim * sizeof(float));
  w->sc = (scored *)malloc((size_t)(ix->n_item + 1) * sizeof(scored));
  if (!w->rank || !w->seen || !w->cand || !w->S || !w->qt || !w->x || !w->sc) return -1;
  memset(w->rank, 0xff, (size_t)ix->n_item * nq);
  return 0;
}

static void ws_free(orc_ws *w) {
  free(w->rank); free(w->seen); free(w->cand); free(w->S); free(w->qt);
  free(w->x); free(w->sc);
}

static int search_one_ws(const orc_index *ix, orc_ws *w, const float *q,
                         uint32_t nq, uint32_t topk, uint32_t nprobe,
                         uint32_t probe_topk, int semantics, orc_trace *tr,
                         float *out_score, uint32_t *out_id) {
  uint32_t pid[64 * 64];
  float ps[64 * 64];
  const int impute = (semantics & ORC_CAND_IMPUTE) != 0;
  semantics &= ~ORC_CAND_IMPUTE;
  /* 1. centroid scores + probe */
  orc_centroid_scores(q, nq, ix->centroid, ix->n_centroid, ix->dim, w->S);
  orc_probe(w->S, nq, ix->n_centroid, nprobe, pid, ps);
  if (tr && tr->probe_id) {
    memcpy(tr->probe_id, pid, (size_t)nq * nprobe * sizeof(uint32_t));
    memcpy(tr->probe_score, ps, (size_t)nq * nprobe * sizeof(float));
  }
  /* 2. candidates: first (= best) probe rank of token q that lists doc c
   * (max_qvec_doc_score, FilterPP.hpp:99-142) */
  uint32_t n_cand = 0;
  for (uint32_t j = 0; j < nprobe; j++)
    for (uint32_t t = 0; t < nq; t++) {
      const uint32_t c = pid[t * nprobe + j];
      const uint32_t *lst = ix->ivf_ids + ix->ivf_off[c];
      for (uint32_t e = 0; e < ix->ivf_size[c]; e++) {
        const uint32_t it = lst[e];
        uint8_t *r = w->rank + (size_t)it * nq + t;
        if (*r == 0xff) {
          *r = (uint8_t)j;
          if (!w->seen[it]) { w->seen[it] = 1; w->cand[n_cand++] = it; }
        }
      }
    }
  qsort(w->cand, n_cand, sizeof(uint32_t), cmp_u32);
  /* 3. approximate score = sum over q of the per-token maxima (RAFT reduce,
   * FilterPP.hpp:366-379), summed exactly: each term as a 2^-32 fixed-point
   * integer, the integer sum rounded once to FP32 (order-independent).
   * With ORC_CAND_IMPUTE (not a reference option) a token that visits no
   * list holding the doc contributes its lowest probed centroid score
   * instead of 0. */
  for (uint32_t i = 0; i < n_cand; i++) {
    const uint32_t it = w->cand[i];
    uint8_t *r = w->rank + (size_t)it * nq;
    int64_t acc = 0;
    for (uint32_t t = 0; t < nq; t++) {
      if (r[t] != 0xff) acc += orc_fixed(ps[t * nprobe + r[t]]);
      else if (impute) acc += orc_fixed(ps[t * nprobe + nprobe - 1]);
      r[t] = 0xff;
    }
    w->seen[it] = 0;
    w->sc[i].s = orc_unfixed(acc);
    w->sc[i].id = it;
  }
  if (tr) {
    tr->n_cand = n_cand;
    if (tr->cand_id)
      for (uint32_t i = 0; i < n_cand && i < tr->cand_cap; i++) {
        tr->cand_id[i] = w->sc[i].id;
        tr->cand_score[i] = w->sc[i].s;
      }
  }
  /* 4. shortlist top-probe_topk (select_k, FilterPP.hpp:386-394) */
  qsort(w->sc, n_cand, sizeof(scored), cmp_scored);
  const uint32_t n_short = n_cand < probe_topk ? n_cand : probe_topk;
  /* 5. rerank: exact MaxSim of decompressed tokens */
  float table[256 * 8];
  orc_decode_table(ix->n_bit, ix->weight, table);
  transpose_query(q, nq, ix->dim, w->qt);
  float m[64];
  for (uint32_t i = 0; i < n_short; i++) {
    const uint32_t it = w->sc[i].id;
    const uint32_t L = ix->item_n_vec[it];
    const uint64_t off = ix->item_off[it];
    for (uint32_t t = 0; t < L; t++)
      decompress_vec(ix, table, off + t, w->x + (uint64_t)t * ix->dim);
    const int clamp = semantics == ORC_SEM_BASIC && L < ix->max_item_n_vec;
    const float ex = maxsim_tokens(w->qt, nq, w->x, L, ix->dim, clamp, m);
    if (tr && tr->short_id) {
      tr->short_id[i] = it;
      tr->short_approx[i] = w->sc[i].s;
      tr->short_exact[i] = ex;
    }
    w->sc[i].s = ex;
  }
  if (tr) tr->n_short = n_short;
  /* 6. final top-k (host std::sort, IGPGPURetrievalPP.hpp:153-161) */
  qsort(w->sc, n_short, sizeof(scored), cmp_scored);
  for (uint32_t k = 0; k < topk; k++) {
    if (k < n_short) { out_score[k] = w->sc[k].s; out_id[k] = w->sc[k].id; }
    else { out_score[k] = -INFINITY; out_id[k] = 0xffffffffu; }
  }
  return 0;
}

static int check_args(const orc_index *ix, uint32_t nq, uint32_t topk,
                      uint32_t nprobe, uint32_t probe_topk) {
  if (nq == 0 || nq > 64) return -1;
  if (nprobe == 0 || nprobe > 64 || nprobe > ix->n_centroid) return -1;
  if (probe_topk < topk) return -1;
  if (ix->dim > 256) return -1;
  return 0;
}

int orc_search_one(const orc_index *ix, const float *q, uint32_t nq,
                   uint32_t topk, uint32_t nprobe, uint32_t probe_topk,
                   int semantics, orc_trace *tr, float *out_score,
                   uint32_t *out_id) {
  if (check_args(ix, nq, topk, nprobe, probe_topk)) return -1;
  orc_ws w;
  if (ws_init(&w, ix, nq)) { ws_free(&w); return -2; }
  const int rc = search_one_ws(ix, &w, q, nq, topk, nprobe, probe_topk,
                               semantics, tr, out_score, out_id);
  ws_free(&w);
  return rc;
}

int orc_search(const orc_index *ix, const float *q, const uint64_t *q_tok_off,
               uint32_t n_query, uint32_t topk, uint32_t nprobe,
               uint32_t probe_topk, int semantics, int n_threads,
               float *out_score, uint32_t *out_id) {
  uint32_t nq_max = 0;
  for (uint32_t i = 0; i < n_query; i++) {
    const uint32_t nq = (uint32_t)(q_tok_off[i + 1] - q_tok_off[i]);
    if (check_args(ix, nq, topk, nprobe, probe_topk)) return -1;
    if (nq > nq_max) nq_max = nq;
  }
  int err = 0;
#pragma omp parallel num_threads(n_threads > 0 ? n_threads : 1)
  {
    orc_ws w;
    int ok = ws_init(&w, ix, nq_max) == 0;
    if (!ok) {
#pragma omp atomic write
      err = -2;
    }
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < (int64_t)n_query; i++) {
      if (!ok) continue;
      const uint32_t nq = (uint32_t)(q_tok_off[i + 1] - q_tok_off[i]);
      search_one_ws(ix, &w, q + q_tok_off[i] * ix->dim, nq, topk, nprobe,
                    probe_topk, semantics, NULL, out_score + (uint64_t)i * topk,
                    out_id + (uint64_t)i * topk);
    }
    ws_free(&w);
  }
  return err;
}

typedef struct { double s; uint32_t id; } scored64;

static int cmp_scored64(const void *a, const void *b) {
  const scored64 *x = (const scored64 *)a, *y = (const scored64 *)b;
  if (x->s > y->s || (x->s == y->s && x->id < y->id)) return -1;
  if (y->s > x->s || (x->s == y->s && y->id < x->id)) return 1;
  return 0;
}

int orc_exhaustive_f64(const float *q, const uint64_t *q_tok_off,
                       uint32_t n_query, const float *tok,
                       const uint32_t *item_n_vec, const uint64_t *item_off,
                       uint32_t n_item, uint32_t dim, uint32_t topk,
                       int n_threads, double *out_score, uint32_t *out_id) {
#pragma omp parallel num_threads(n_threads > 0 ? n_threads : 1)
  {
    scored64 *sc = (scored64 *)malloc((size_t)n_item * sizeof(scored64));
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < (int64_t)n_query; i++) {
      const uint32_t nq = (uint32_t)(q_tok_off[i + 1] - q_tok_off[i]);
      const float *qi = q + q_tok_off[i] * dim;
      for (uint32_t it = 0; it < n_item; it++) {
        sc[it].s = orc_maxsim_f64(qi, nq, tok + item_off[it] * dim,
                                  item_n_vec[it], dim);
        sc[it].id = it;
      }
      qsort(sc, n_item, sizeof(scored64), cmp_scored64);
      for (uint32_t k = 0; k < topk; k++) {
        out_score[(uint64_t)i * topk + k] = k < n_item ? sc[k].s : -INFINITY;
        out_id[(uint64_t)i * topk + k] = k < n_item ? sc[k].id : 0xffffffffu;
      }
    }
    free(sc);
  }
  return 0;
}
