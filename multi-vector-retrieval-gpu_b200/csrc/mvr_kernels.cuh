// mvr_kernels.cuh -- launchers of the plain FP32 search kernels.
#pragma once
#include <cuda_runtime.h>
#include "mvr_common.cuh"

namespace mvr {

// Per-query-slot scratch of the candidate filter (one slot per CTA of a
// filter launch).  stamp starts at 0, rank at 0xff; the filter restores rank.
struct FilterScratch {
  uint32_t *stamp;       // [slots][n_item] epoch of last visit
  uint8_t *rank;         // [slots][n_item][rank_stride] best probe rank
  uint64_t *key;         // [slots][n_item] candidate (score, id) keys
  uint32_t n_item;
  uint32_t rank_stride;  // 32 or 64 (>= query tokens, multiple of 16)
  uint32_t *qcnt;        // [slots] candidate keys emitted by the hash filter (0 between batches)
  uint32_t *ovf;         // [slots] 1: the hash filter overflowed
  uint64_t *hkey;        // [slots][key_stride] hash-filter candidate keys
  uint32_t key_stride;   // keys per query slot: kHashFill * the largest range count in use
};

// Candidate keys one query can hold in the hash filter: every doc range
// stops inserting at kHashFill candidates, beyond which the query overflows.
constexpr uint32_t kHashFill = 7168u;

// Doc ranges (CTAs) of one query in the hash filter, a power of two in
// [8, kHashParts]: enough that the expected candidate count, nq * nprobe *
// cand_per_probe, fills each range's hash table to at most 85 % of
// kHashFill (candidates spread evenly over the doc ranges, up to a few
// percent).  cand_per_probe: the largest candidates per probed list seen in
// the handle's previous search (docs listed under several probes count
// once), or an estimate from the index's mean list length before the first.
// Each range is a union of kHashParts / P consecutive ranges of the
// partition table.
inline uint32_t hash_parts(uint32_t nq, uint32_t nprobe, double cand_per_probe) {
  const double cand = (double)nq * nprobe * cand_per_probe;
  uint32_t p = 8;
  while (p < (uint32_t)kHashParts && cand > 0.85 * kHashFill * p) p *= 2;
  return p;
}

cudaError_t configure_kernels();
// ivf_part table of an index ([C][kHashParts + 1] u32)
cudaError_t make_ivf_part(const DevIndex &ix, uint32_t *out, cudaStream_t st);
int probe_splits(uint32_t n_tok, uint32_t n_cent_pad, int n_sm);
cudaError_t launch_probe(const DevIndex &ix, const float *q, uint32_t n_tok,
                         uint32_t nprobe, int n_split, uint32_t *part_id,
                         float *part_s, uint32_t *out_id, float *out_s,
                         cudaStream_t st, int *n_launch);
cudaError_t launch_filter(const DevIndex &ix, const uint32_t *probe_id,
                          const float *probe_s, uint32_t nprobe,
                          const uint64_t *q_off, uint32_t n_query,
                          uint32_t probe_topk, const FilterScratch &scr,
                          uint32_t epoch, uint32_t *short_id,
                          float *short_approx, uint32_t *n_short,
                          uint32_t *qstat /*[n_query][3]: n_cand, list entries
                                            visited, shortlist tokens*/,
                          cudaStream_t st, int *n_launch);
// The same filter with each query split over a cluster of 4 CTAs; with
// only_if set, only the queries whose flag is set run (and clear it).
cudaError_t launch_filter_cluster(const DevIndex &ix, const uint32_t *probe_id,
                                  const float *probe_s, uint32_t nprobe,
                                  const uint64_t *q_off, uint32_t n_query,
                                  uint32_t probe_topk, const FilterScratch &scr,
                                  const uint32_t *epoch_base, uint32_t epoch_add,
                                  uint32_t *short_id, float *short_approx, uint32_t *n_short,
                                  uint32_t *qstat, cudaStream_t st, int *n_launch,
                                  uint32_t *only_if, int impute);
// Main-path filter: shared-memory hash tables over doc ranges (hash_parts
// CTAs per query), a select kernel, and the rank-table filter for overflowed
// queries.  cta_off[0..n_query]: first CTA of every query (prefix sum of
// hash_parts), n_cta = cta_off[n_query].
// impute: an unmatched query token adds its lowest probed score to a
// candidate's approximate score (MVR_CAND_IMPUTE) instead of 0.
// scr: stamp / rank / key hold fb_slots slots of the rank-table fallback,
// which runs in chunks of fb_slots queries; hkey / qcnt / ovf hold n_query.
// epoch: device counter of the fallback's stamp epochs (advanced on device).
cudaError_t launch_filter_hash(const DevIndex &ix, const uint32_t *probe_id,
                               const float *probe_s, uint32_t nprobe,
                               const uint64_t *q_off, const uint64_t *cta_off, uint32_t n_cta,
                               uint32_t n_query, uint32_t fb_slots,
                               uint32_t probe_topk, const FilterScratch &scr,
                               uint32_t *epoch, uint32_t *short_id,
                               float *short_approx, uint32_t *n_short,
                               uint32_t *qstat, cudaStream_t st, int *n_launch, int impute);
cudaError_t launch_rerank(const DevIndex &ix, const float *q, const uint64_t *q_off,
                          uint32_t n_query, const uint32_t *short_id,
                          const uint32_t *n_short, uint32_t probe_topk,
                          int semantics, float *exact, unsigned *err, cudaStream_t st,
                          int *n_launch, uint64_t wait_ns);
cudaError_t launch_topk(const uint32_t *short_id, const float *exact,
                        const uint32_t *n_short, uint32_t n_query,
                        uint32_t probe_topk, uint32_t topk, float *out_s,
                        uint32_t *out_id, uint32_t *n_out /*nullable: min(n, topk)*/,
                        cudaStream_t st, int *n_launch);

}  // namespace mvr
