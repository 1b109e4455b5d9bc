// mvr_capi.cu -- the C ABI of libmvr (include/mvr.h): index residency in
// HBM, per-handle search workspaces, the batched asynchronous search
// pipeline and the index-build entry points.
#include "mvr.h"


#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "mvr_aux.cuh"
#include "mvr_common.cuh"
#include "mvr_io.hpp"
#include "mvr_kernels.cuh"
#include "mvr_tc.cuh"
#include "mvr_prune.cuh"

using namespace mvr;

namespace {

thread_local std::string g_err;

int set_err(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CUDA_TRY(expr)                                                              \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      return set_err(e_ == cudaErrorMemoryAllocation ? MVR_ERR_OOM : MVR_ERR_CUDA,  \
                     "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__,     \
                     __LINE__);                                                     \
    }                                                                               \
  } while (0)

#define MVR_TRY(expr)            \
  do {                           \
    int r_ = (expr);             \
    if (r_ != MVR_OK) return r_; \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <class T>
int dalloc(T **p, size_t n, std::vector<void *> *owner = nullptr) {
  *p = nullptr;
  if (n == 0) n = 1;
  CUDA_TRY(cudaMalloc((void **)p, n * sizeof(T)));
  if (owner) owner->push_back(*p);
  return MVR_OK;
}

void dfree(void *p) {
  if (p) cudaFree(p);
}

// One decode-table row per byte value: weights of its 8/b values, MSB-first
// (SQInfoPP ctor, DataStructPP.hpp:150-187).
std::vector<float> make_lut(uint32_t n_bit, const float *weight) {
  const uint32_t vpb = 8u / n_bit, mask = (1u << n_bit) - 1u;
  std::vector<float> lut(256 * vpb);
  for (uint32_t code = 0; code < 256; code++)
    for (uint32_t i = 0; i < vpb; i++)
      lut[code * vpb + i] = weight[(code >> (8u - n_bit * (i + 1u))) & mask];
  return lut;
}

__global__ void validate_kernel(const uint32_t *code, uint64_t n_vec, uint32_t n_cent,
                                const uint32_t *ids, uint64_t n_ele, uint32_t n_item,
                                unsigned *flag) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_vec; i += stride)
    if (code[i] >= n_cent) atomicOr(flag, 1u);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_ele; i += stride)
    if (ids[i] >= n_item) atomicOr(flag, 2u);
}

}  // namespace

// ----------------------------------------------------------------------
// handle
// ----------------------------------------------------------------------
struct Workspace {
  uint32_t slots = 0, fb_slots = 0, rank_stride = 0;
  uint32_t *stamp = nullptr;    // rank-table fallback: [fb_slots][n_item]
  uint8_t *rank = nullptr;      //   [fb_slots][n_item][rank_stride]
  uint64_t *key = nullptr;      //   [fb_slots][n_item]
  uint64_t *hkey = nullptr;     // hash filter: [slots][key_stride] candidate keys
  uint32_t key_stride = 0;      //   keys per slot: kHashFill * the largest range count
  uint32_t *qcnt = nullptr, *ovf = nullptr;  // [slots] hash-filter counters / overflow flags
  // per batch
  uint32_t batch_slots = 0, tok_cap = 0, np_cap = 0, short_cap = 0, topk_cap = 0;
  size_t part_cap = 0;
  float *q = nullptr, *q2 = nullptr;  // query tokens (host-buffer calls: two, alternating)
  uint32_t *probe_id = nullptr, *part_id = nullptr;
  float *probe_s = nullptr, *part_s = nullptr;
  uint32_t *short_id = nullptr, *n_short = nullptr;
  float *short_approx = nullptr, *exact = nullptr;
  float *out_s = nullptr;
  uint32_t *out_id = nullptr;
  size_t cand_cap = 0;            // tensor-core probe candidates (BF16 path)
  uint32_t *cand = nullptr;
  uint32_t r_cap = 0;             // FP32 re-score of the top-R (BF16 path)
  uint32_t *r_id = nullptr, *n_r = nullptr;
  float *r_score = nullptr, *r_exact = nullptr;
  // per call
  size_t off_cap = 0, stat_cap = 0;
  uint64_t *q_off = nullptr;    // device, all batches' relative token offsets, then
                                // their hash-filter CTA offsets (same layout)
  uint64_t *h_off = nullptr;    // pinned mirror
  uint32_t *qstat = nullptr;    // device [n_query][3]
  uint32_t *h_qstat = nullptr;  // pinned mirror
  // learned pruner (MVR_PRUNE), per batch
  uint32_t pr_slots = 0, pr_short = 0, pr_keep = 0;
  float *feat = nullptr;        // [slots][short][33] features
  float *pred = nullptr;        // [slots][short] predictions
  float *kept_s = nullptr;      // [slots][keep] best predictions
  uint32_t *kept_id = nullptr;  // [slots][keep]
  uint32_t *fin_id = nullptr;   // [slots][short] docs the rerank takes
  uint32_t *n_fin = nullptr;    // [slots]
};

struct mvr_index {
  int device = 0;
  int n_sm = 148;
  DevIndex dix{};
  std::vector<void *> bufs;
  uint32_t max_ivf_list = 0;
  uint64_t device_bytes = 0;
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> events;
  // host-buffer calls: query copies on their own stream, one event per batch
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> copy_events;
  uint32_t batch_cap = 0;
  uint32_t rescore = 0;          // FP32 re-score count of the BF16 path (0: 4 * topk)
  void *cen_bf16 = nullptr;      // [C][128] BF16 centroid rows
  void *lut_bf16 = nullptr;      // [256][8/b] BF16 decode table
  void *cen_sw = nullptr;        // [C_pad/128][32 KB] swizzled BF16 centroid tiles
  void *cen_perm = nullptr;      // [C][64] bf16x2 centroid rows, TMEM-rerank K order (b <= 2)
  TmWeights tw_bf16{};           // weight tables of the BF16 tensor-memory MaxSim (b <= 2)
  float x_bound = 0.f;           // bound on the norm of every decoded doc token
  void *cen8 = nullptr;          // [C][128] E4M3 centroid rows, FP8-rerank K order (b = 2, 4)
  TmWeights tw_fp8{};            // E4M3 weight tables of the FP8 MaxSim (b = 2, 4)
  unsigned *d_err = nullptr;     // device error flags of the tensor-core kernels
  uint32_t *d_epoch = nullptr;   // stamp-epoch counter of the rank-table fallback (device)
  uint64_t epoch_used = 0;       // epochs consumed since the stamps were last cleared
  uint64_t ws_gen = 0;           // bumped whenever a workspace buffer is reallocated
  // hash filter sizing: candidates per probed list, the largest over the
  // queries of the previous search call (0: none yet)
  double cand_per_probe = 0.0;
  uint64_t wait_ns = 1000000000ull;  // bound of the FP8 rerank's pipeline waits
  uint32_t ws_docs = 256;            // shortlisted docs per CTA of the FP8 rerank
  // learned pruner (mvr_index_set_pruner): BF16 weight tiles, b1/b2/w3/b3
  uint8_t *prune_wts = nullptr;
  float *prune_vecs = nullptr;
  uint32_t prune_keep = 0;
  float prune_margin = 0.f;
  unsigned long long *d_fallback = nullptr;  // queries of a call that scored their whole shortlist
  // CUDA-graph replay of repeated device-buffer searches (mvr_index_set_graphs)
  bool graphs = false;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;  // stream handoff (no timing)
  cudaEvent_t ev_g0 = nullptr, ev_g1 = nullptr;   // device time of a graph launch
  struct {
    cudaGraphExec_t exec = nullptr;
    const float *query = nullptr;
    float *out_s = nullptr;
    uint32_t *out_id = nullptr;
    uint32_t n_query = 0, topk = 0, nprobe = 0, probe_topk = 0, flags = 0, R = 0, B = 0;
    uint64_t gen = 0;
    double cand_per_probe = 0.0;  // the hash filter's layout was sized by this
    std::vector<uint64_t> off;
    int launches = 0;
  } graph;
  Workspace ws;

  void drop_graph() {
    if (graph.exec) cudaGraphExecDestroy(graph.exec);
    graph.exec = nullptr;
  }

  ~mvr_index() {
    DeviceGuard g(device);
    if (stream) cudaStreamSynchronize(stream);
    for (void *p : bufs) dfree(p);
    dfree(d_err);
    dfree(d_epoch);
    drop_graph();
    for (cudaEvent_t e : {ev_in, ev_out, ev_g0, ev_g1})
      if (e) cudaEventDestroy(e);
    free_scratch();
    free_batch();
    free_prune();
    dfree(prune_wts);
    dfree(prune_vecs);
    dfree(d_fallback);
    dfree(ws.q_off);
    dfree(ws.qstat);
    if (ws.h_off) cudaFreeHost(ws.h_off);
    if (ws.h_qstat) cudaFreeHost(ws.h_qstat);
    for (auto e : events) cudaEventDestroy(e);
    for (auto e : copy_events) cudaEventDestroy(e);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (stream) cudaStreamDestroy(stream);
  }
  void free_scratch() {
    dfree(ws.stamp); dfree(ws.rank); dfree(ws.key); dfree(ws.hkey); dfree(ws.qcnt); dfree(ws.ovf);
    ws.stamp = nullptr; ws.rank = nullptr; ws.key = nullptr; ws.hkey = nullptr;
    ws.qcnt = nullptr; ws.ovf = nullptr;
    ws.slots = 0;
  }
  void free_prune() {
    for (void *p : {(void *)ws.feat, (void *)ws.pred, (void *)ws.kept_s, (void *)ws.kept_id,
                    (void *)ws.fin_id, (void *)ws.n_fin})
      dfree(p);
    ws.feat = ws.pred = ws.kept_s = nullptr;
    ws.kept_id = ws.fin_id = ws.n_fin = nullptr;
    ws.pr_slots = ws.pr_short = ws.pr_keep = 0;
  }
  void free_batch() {
    for (void *p : {(void *)ws.q, (void *)ws.q2, (void *)ws.probe_id, (void *)ws.part_id, (void *)ws.probe_s,
                    (void *)ws.part_s, (void *)ws.short_id, (void *)ws.n_short,
                    (void *)ws.short_approx, (void *)ws.exact, (void *)ws.out_s, (void *)ws.out_id,
                    (void *)ws.r_id, (void *)ws.n_r, (void *)ws.r_score, (void *)ws.r_exact,
                    (void *)ws.cand})
      dfree(p);
    ws.cand = nullptr;
    ws.cand_cap = 0;
    ws.r_id = ws.n_r = nullptr;
    ws.r_score = ws.r_exact = nullptr;
    ws.r_cap = 0;
    ws.q = ws.q2 = nullptr; ws.probe_id = ws.part_id = nullptr; ws.probe_s = ws.part_s = nullptr;
    ws.short_id = ws.n_short = nullptr; ws.short_approx = ws.exact = nullptr;
    ws.out_s = nullptr; ws.out_id = nullptr;
    ws.batch_slots = ws.tok_cap = ws.np_cap = ws.short_cap = ws.topk_cap = 0;
    ws.part_cap = 0;
  }
};

namespace {

// Queries per device batch: 8 per SM (1,184 on B200) -- large batches fill
// the tensor-core probe's token tiles and the re-score's CTAs; the hash
// filter's key space is kHashFill * 8 B = 57 KB per query per doc range
// (8 to 64 ranges).
uint32_t default_batch(const mvr_index *h) { return 8u * (uint32_t)h->n_sm; }

// Slots of the rank-table fallback (n_item * (4 + 32|64 + 8) bytes each,
// kept within ~8 GB and at most half the batch, so a batch always takes at
// least two chunks); it runs the batch's overflowed queries chunk by chunk.
uint32_t fallback_slots(const mvr_index *h, uint32_t slots, uint32_t rank_stride) {
  const double per_slot = (double)h->dix.n_item * (12.0 + rank_stride);
  uint32_t f = std::min((slots + 1) / 2, 2u * (uint32_t)h->n_sm);
  while (f > 1 && per_slot * f > 8.0 * (1ull << 30)) f--;
  return std::max(1u, f);
}

int ensure_scratch(mvr_index *h, uint32_t slots, uint32_t rank_stride, uint32_t key_stride) {
  Workspace &w = h->ws;
  if (w.slots >= slots && w.rank_stride >= rank_stride && w.key_stride >= key_stride)
    return MVR_OK;
  key_stride = std::max(key_stride, w.key_stride);
  h->free_scratch();
  const size_t n = (size_t)h->dix.n_item;
  const uint32_t fb = fallback_slots(h, slots, rank_stride);
  MVR_TRY(dalloc(&w.stamp, fb * n));
  MVR_TRY(dalloc(&w.rank, fb * n * rank_stride));
  MVR_TRY(dalloc(&w.key, fb * n));
  MVR_TRY(dalloc(&w.hkey, (size_t)slots * key_stride));
  MVR_TRY(dalloc(&w.qcnt, slots));
  MVR_TRY(dalloc(&w.ovf, slots));
  CUDA_TRY(cudaMemsetAsync(w.qcnt, 0, slots * sizeof(uint32_t), h->stream));
  CUDA_TRY(cudaMemsetAsync(w.ovf, 0, slots * sizeof(uint32_t), h->stream));
  CUDA_TRY(cudaMemsetAsync(w.stamp, 0, fb * n * sizeof(uint32_t), h->stream));
  CUDA_TRY(cudaMemsetAsync(w.rank, 0xff, fb * n * rank_stride, h->stream));
  CUDA_TRY(cudaMemsetAsync(h->d_epoch, 0, sizeof(uint32_t), h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  w.slots = slots;
  w.fb_slots = fb;
  w.rank_stride = rank_stride;
  w.key_stride = key_stride;
  h->epoch_used = 0;
  h->ws_gen++;
  return MVR_OK;
}

int ensure_prune(mvr_index *h, uint32_t slots, uint32_t short_cap, uint32_t keep) {
  Workspace &w = h->ws;
  if (w.pr_slots >= slots && w.pr_short >= short_cap && w.pr_keep >= keep) return MVR_OK;
  slots = std::max(slots, w.pr_slots);
  short_cap = std::max(short_cap, w.pr_short);
  keep = std::max(keep, w.pr_keep);
  h->free_prune();
  h->ws_gen++;
  MVR_TRY(dalloc(&w.feat, (size_t)slots * short_cap * 33));
  MVR_TRY(dalloc(&w.pred, (size_t)slots * short_cap));
  MVR_TRY(dalloc(&w.kept_s, (size_t)slots * keep));
  MVR_TRY(dalloc(&w.kept_id, (size_t)slots * keep));
  MVR_TRY(dalloc(&w.fin_id, (size_t)slots * short_cap));
  MVR_TRY(dalloc(&w.n_fin, (size_t)slots));
  w.pr_slots = slots;
  w.pr_short = short_cap;
  w.pr_keep = keep;
  return MVR_OK;
}

int ensure_batch(mvr_index *h, uint32_t slots, uint32_t tok_cap, uint32_t nprobe,
                 uint32_t short_cap, uint32_t topk, size_t part_need, uint32_t r_cap,
                 size_t cand_need) {
  Workspace &w = h->ws;
  if (w.batch_slots >= slots && w.tok_cap >= tok_cap && w.np_cap >= nprobe &&
      w.short_cap >= short_cap && w.topk_cap >= topk && w.part_cap >= part_need &&
      w.r_cap >= r_cap && w.cand_cap >= cand_need)
    return MVR_OK;
  r_cap = std::max(r_cap, w.r_cap);
  cand_need = std::max(cand_need, w.cand_cap);
  const uint32_t s = std::max(slots, w.batch_slots);
  tok_cap = std::max(tok_cap, w.tok_cap);
  nprobe = std::max(nprobe, w.np_cap);
  short_cap = std::max(short_cap, w.short_cap);
  topk = std::max(topk, w.topk_cap);
  part_need = std::max(part_need, w.part_cap);
  h->free_batch();
  h->ws_gen++;
  MVR_TRY(dalloc(&w.q, (size_t)tok_cap * kDim));
  MVR_TRY(dalloc(&w.q2, (size_t)tok_cap * kDim));
  MVR_TRY(dalloc(&w.probe_id, (size_t)tok_cap * nprobe));
  MVR_TRY(dalloc(&w.probe_s, (size_t)tok_cap * nprobe));
  MVR_TRY(dalloc(&w.part_id, part_need));
  MVR_TRY(dalloc(&w.part_s, part_need));
  MVR_TRY(dalloc(&w.short_id, (size_t)s * short_cap));
  MVR_TRY(dalloc(&w.short_approx, (size_t)s * short_cap));
  MVR_TRY(dalloc(&w.exact, (size_t)s * short_cap));
  MVR_TRY(dalloc(&w.n_short, (size_t)s));
  MVR_TRY(dalloc(&w.out_s, (size_t)s * topk));
  MVR_TRY(dalloc(&w.out_id, (size_t)s * topk));
  MVR_TRY(dalloc(&w.r_id, (size_t)s * r_cap));
  MVR_TRY(dalloc(&w.r_score, (size_t)s * r_cap));
  MVR_TRY(dalloc(&w.r_exact, (size_t)s * r_cap));
  MVR_TRY(dalloc(&w.n_r, (size_t)s));
  MVR_TRY(dalloc(&w.cand, cand_need));
  w.cand_cap = cand_need;
  w.r_cap = r_cap;
  w.batch_slots = s;
  w.tok_cap = tok_cap;
  w.np_cap = nprobe;
  w.short_cap = short_cap;
  w.topk_cap = topk;
  w.part_cap = part_need;
  return MVR_OK;
}

constexpr int kStages = 6;

int ensure_call(mvr_index *h, size_t n_off, size_t n_stat, size_t n_events) {
  Workspace &w = h->ws;
  if (w.off_cap < n_off || w.stat_cap < n_stat || h->events.size() < n_events) h->ws_gen++;
  if (w.off_cap < n_off) {
    dfree(w.q_off);
    w.q_off = nullptr;
    if (w.h_off) cudaFreeHost(w.h_off);
    w.h_off = nullptr;
    MVR_TRY(dalloc(&w.q_off, n_off));
    CUDA_TRY(cudaMallocHost((void **)&w.h_off, n_off * sizeof(uint64_t)));
    w.off_cap = n_off;
  }
  if (w.stat_cap < n_stat) {
    dfree(w.qstat);
    w.qstat = nullptr;
    if (w.h_qstat) cudaFreeHost(w.h_qstat);
    w.h_qstat = nullptr;
    MVR_TRY(dalloc(&w.qstat, n_stat));
    CUDA_TRY(cudaMallocHost((void **)&w.h_qstat, n_stat * sizeof(uint32_t)));
    w.stat_cap = n_stat;
  }
  while (h->events.size() < n_events) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    h->events.push_back(e);
  }
  while (h->copy_events.size() * kStages + 1 < n_events) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->copy_events.push_back(e);
  }
  return MVR_OK;
}

size_t part_entries(const mvr_index *h, uint32_t n_tok, uint32_t nprobe, int *splits_out) {
  const int splits = probe_splits(n_tok, h->dix.n_centroid_pad, h->n_sm);
  *splits_out = splits;
  return splits > 1 ? (size_t)splits * n_tok * nprobe : 1;
}

int check_search_args(const mvr_index *h, uint32_t n_query, uint32_t topk, uint32_t nprobe,
                      uint32_t probe_topk) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  if (probe_topk < topk)
    return set_err(MVR_ERR_INVALID_ARG,
                   "probe_topk (%u) is smaller than topk (%u)", probe_topk, topk);
  if (topk == 0 || topk > (uint32_t)kMaxTopk)
    return set_err(MVR_ERR_INVALID_ARG, "topk must be in [1, %d], got %u", kMaxTopk, topk);
  if (probe_topk > (uint32_t)kMaxShort)
    return set_err(MVR_ERR_INVALID_ARG, "probe_topk must be <= %d, got %u", kMaxShort, probe_topk);
  if (nprobe == 0 || nprobe > h->dix.n_centroid)
    return set_err(MVR_ERR_INVALID_ARG, "nprobe (%u) must be in [1, n_centroid=%u]", nprobe,
                   h->dix.n_centroid);
  if (nprobe > (uint32_t)kMaxProbe)
    return set_err(MVR_ERR_UNSUPPORTED, "nprobe > %d is not supported", kMaxProbe);
  (void)n_query;
  return MVR_OK;
}

int build_offsets(const uint64_t *tok_off, uint32_t n_query, uint32_t query_n_vec,
                  std::vector<uint64_t> &off, uint32_t *nq_max) {
  off.resize((size_t)n_query + 1);
  *nq_max = 0;
  if (!tok_off) {
    if (query_n_vec == 0 || query_n_vec > (uint32_t)kMaxQueryTok)
      return set_err(MVR_ERR_INVALID_ARG, "query_n_vec must be in [1, %d], got %u", kMaxQueryTok,
                     query_n_vec);
    for (uint32_t i = 0; i <= n_query; i++) off[i] = (uint64_t)i * query_n_vec;
    *nq_max = query_n_vec;
    return MVR_OK;
  }
  if (tok_off[0] != 0) return set_err(MVR_ERR_INVALID_ARG, "tok_off[0] must be 0");
  for (uint32_t i = 0; i < n_query; i++) {
    if (tok_off[i + 1] <= tok_off[i] || tok_off[i + 1] - tok_off[i] > (uint64_t)kMaxQueryTok)
      return set_err(MVR_ERR_INVALID_ARG, "query %u has %lld tokens (allowed 1..%d)", i,
                     (long long)(tok_off[i + 1] - tok_off[i]), kMaxQueryTok);
    *nq_max = std::max(*nq_max, (uint32_t)(tok_off[i + 1] - tok_off[i]));
  }
  std::memcpy(off.data(), tok_off, off.size() * sizeof(uint64_t));
  return MVR_OK;
}

// The shared batched pipeline.  host_io: queries/results are host buffers
// (copied per batch inside the call: each batch's queries on the handle's
// copy stream while the previous batch computes); otherwise device buffers.
// Events: kStages+0 per batch at the stage boundaries plus one closing event;
// stage k of a batch = events[bt*kStages+k] .. events[bt*kStages+k+1]:
//   0 query copy, 1 centroid scoring + probe, 2 candidate filter + shortlist,
//   3 rerank (FP32, or BF16 tensor-core), 4 FP32 re-score + top-k, 5 result copy.

int search_impl(mvr_index *h, const float *query, const uint64_t *tok_off_in, uint32_t n_query,
                uint32_t query_n_vec, uint32_t topk, uint32_t nprobe, uint32_t probe_topk,
                uint32_t flags, float *out_s, uint32_t *out_id, double *query_time_s,
                double *stage_s, mvr_stats *stats, cudaStream_t st, bool host_io) {
  const auto t_start = std::chrono::steady_clock::now();
  MVR_TRY(check_search_args(h, n_query, topk, nprobe, probe_topk));
  if (n_query == 0) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return MVR_OK;
  }
  if (!query || !out_s || !out_id) return set_err(MVR_ERR_INVALID_ARG, "null query/result buffer");
  if (flags & ~(MVR_SEM_BASIC | MVR_PREC_BF16 | MVR_PREC_FP8 | MVR_CAND_IMPUTE | MVR_PRUNE))
    return set_err(MVR_ERR_INVALID_ARG, "unknown flags %u", flags);
  const int sem = (flags & MVR_SEM_BASIC) ? 1 : 0;
  const bool fp8 = (flags & MVR_PREC_FP8) != 0 && h->cen8 != nullptr;
  const bool bf16 = (flags & (MVR_PREC_BF16 | MVR_PREC_FP8)) != 0;  // mixed-precision path
  uint32_t R = h->rescore ? h->rescore : 4 * topk;
  R = std::min(std::max(R, topk), probe_topk);
  std::vector<uint64_t> off;
  uint32_t nq_max = 0;
  MVR_TRY(build_offsets(tok_off_in, n_query, query_n_vec, off, &nq_max));
  const bool prune = (flags & MVR_PRUNE) != 0;
  if (prune) {
    // the features come from the FP8 centroid table (2- and 4-bit indexes);
    // the pruned docs go to the FP8 MaxSim (with MVR_PREC_FP8) or straight
    // to the exact FP32 rerank (no precision flag)
    if (!h->cen8)
      return set_err(MVR_ERR_UNSUPPORTED, "MVR_PRUNE needs a 2- or 4-bit index");
    if (bf16 && !(flags & MVR_PREC_FP8))
      return set_err(MVR_ERR_UNSUPPORTED, "MVR_PRUNE: with a precision flag, MVR_PREC_FP8");
    if (!h->prune_wts) return set_err(MVR_ERR_INVALID_ARG, "MVR_PRUNE: no pruner set");
    if (nq_max > 32) return set_err(MVR_ERR_UNSUPPORTED, "MVR_PRUNE: queries of up to 32 tokens");
  }
  const uint32_t keep = prune ? std::min(h->prune_keep, probe_topk) : 0u;
  DeviceGuard g(h->device);

  const uint32_t B = h->batch_cap ? h->batch_cap : default_batch(h);
  const uint32_t n_batch = (n_query + B - 1) / B;
  uint32_t tok_cap = 0;
  size_t part_need = 1, cand_need = 1;
  const bool tc_probe = bf16 && nprobe <= 16;  // tensor-core scoring + exact re-score
  for (uint32_t bt = 0; bt < n_batch; bt++) {
    const uint32_t s = bt * B, e = std::min(n_query, s + B);
    const uint32_t T = (uint32_t)(off[e] - off[s]);
    tok_cap = std::max(tok_cap, T);
    int sp;
    part_need = std::max(part_need, part_entries(h, T, nprobe, &sp));
    uint32_t tsp;
    if (tc_probe)
      cand_need = std::max(cand_need, (size_t)T * probe_tc_cand_per_token(T, h->dix.n_centroid, h->n_sm, &tsp));
  }
  const uint32_t rank_stride = nq_max <= 32 ? 32u : 64u;
  // before the first search: about a third of a mean-length list's docs are
  // new candidates (measured on the synthetic corpora)
  const double cpe = h->cand_per_probe > 0.0
                         ? h->cand_per_probe
                         : 0.35 * (double)h->dix.n_ele_ivf / std::max(1u, h->dix.n_centroid);
  const uint32_t parts_max = hash_parts(nq_max, nprobe, cpe);
  MVR_TRY(ensure_scratch(h, std::min(B, n_query), rank_stride, parts_max * kHashFill));
  MVR_TRY(ensure_batch(h, std::min(B, n_query), tok_cap, nprobe, probe_topk, topk, part_need, R,
                       cand_need));
  MVR_TRY(ensure_call(h, 2 * ((size_t)n_query + n_batch), (size_t)n_query * 3,
                      (size_t)kStages * n_batch + 1));
  if (prune) MVR_TRY(ensure_prune(h, std::min(B, n_query), probe_topk, keep));
  Workspace &w = h->ws;

  // stamp epochs this call takes (one per fallback chunk of every batch);
  // clear the stamps before the device counter could wrap
  uint64_t call_epochs = 0;
  for (uint32_t bt = 0; bt < n_batch; bt++) {
    const uint32_t nb = std::min(n_query, (bt + 1) * B) - bt * B;
    call_epochs += (nb + w.fb_slots - 1) / w.fb_slots;
  }
  if (h->epoch_used + call_epochs >= (1ull << 31)) {
    CUDA_TRY(cudaStreamSynchronize(st));
    CUDA_TRY(cudaMemsetAsync(w.stamp, 0, (size_t)w.fb_slots * h->dix.n_item * sizeof(uint32_t),
                             h->stream));
    CUDA_TRY(cudaMemsetAsync(h->d_epoch, 0, sizeof(uint32_t), h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->epoch_used = 0;
  }
  h->epoch_used += call_epochs;

  // relative token offsets of every batch, then the first hash-filter CTA
  // of every query of the batch (prefix sum of hash_parts)
  const size_t n_off = (size_t)n_query + n_batch;
  std::vector<uint32_t> n_cta(n_batch);
  for (uint32_t bt = 0, pos = 0; bt < n_batch; bt++) {
    const uint32_t s = bt * B, e = std::min(n_query, s + B);
    uint64_t cta = 0;
    for (uint32_t i = s; i <= e; i++, pos++) {
      w.h_off[pos] = off[i] - off[s];
      w.h_off[n_off + pos] = cta;
      if (i < e) cta += hash_parts((uint32_t)(off[i + 1] - off[i]), nprobe, cpe);
    }
    n_cta[bt] = (uint32_t)cta;
  }

  FilterScratch scr{w.stamp, w.rank,   w.key,  h->dix.n_item, w.rank_stride,
                    w.qcnt,  w.ovf,    w.hkey, w.key_stride};
  int launches = 0;
  uint64_t h2d = 2 * n_off * sizeof(uint64_t), d2h = 0;
  auto ev = [&](uint32_t bt, int k) { return h->events[(size_t)bt * kStages + k]; };
  // every device operation of the call, in stream order on `rs`
  // (events recorded while capturing become external event-record nodes)
  auto enqueue = [&](cudaStream_t rs, bool capturing) -> int {
    if (prune) CUDA_TRY(cudaMemsetAsync(h->d_fallback, 0, sizeof(unsigned long long), rs));
    auto rec = [&](cudaEvent_t e) {
      return capturing ? cudaEventRecordWithFlags(e, rs, cudaEventRecordExternal)
                       : cudaEventRecord(e, rs);
    };
    CUDA_TRY(cudaMemcpyAsync(w.q_off, w.h_off, 2 * n_off * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, rs));
    // host buffers: batch bt's query tokens go to device buffer bt % 2 on
    // the copy stream, one batch ahead of the kernels, once batch bt - 2
    // (the buffer's previous user) has finished
    // (a single batch has nothing to overlap: its copy stays on rs)
    const bool pipelined = host_io && n_batch > 1;
    auto qbuf = [&](uint32_t bt) { return (bt & 1) ? w.q2 : w.q; };
    auto copy_in = [&](uint32_t bt) -> int {
      const uint32_t s = bt * B, e = std::min(n_query, s + B);
      const uint32_t T = (uint32_t)(off[e] - off[s]);
      if (bt >= 2) CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, ev(bt - 2, 5), 0));
      CUDA_TRY(cudaMemcpyAsync(qbuf(bt), query + off[s] * kDim, (size_t)T * kDim * sizeof(float),
                               cudaMemcpyHostToDevice, h->copy_stream));
      CUDA_TRY(cudaEventRecord(h->copy_events[bt], h->copy_stream));
      h2d += (size_t)T * kDim * sizeof(float);
      return MVR_OK;
    };
    if (pipelined) {
      CUDA_TRY(cudaEventRecord(h->ev_in, rs));  // the copies after the caller's prior work
      CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev_in, 0));
      MVR_TRY(copy_in(0));
    }
    for (uint32_t bt = 0; bt < n_batch; bt++) {
      const uint32_t s = bt * B, e = std::min(n_query, s + B), nb = e - s;
      CUDA_TRY(rec(ev(bt, 0)));
      const uint32_t T = (uint32_t)(off[e] - off[s]);
      const uint64_t *qo = w.q_off + (size_t)s + bt;
      const float *qp;
      if (pipelined) {
        if (bt + 1 < n_batch) MVR_TRY(copy_in(bt + 1));
        CUDA_TRY(cudaStreamWaitEvent(rs, h->copy_events[bt], 0));
        qp = qbuf(bt);
      } else if (host_io) {
        CUDA_TRY(cudaMemcpyAsync(w.q, query + off[s] * kDim, (size_t)T * kDim * sizeof(float),
                                 cudaMemcpyHostToDevice, rs));
        h2d += (size_t)T * kDim * sizeof(float);
        qp = w.q;
      } else {
        qp = query + off[s] * kDim;
      }
      CUDA_TRY(rec(ev(bt, 1)));
      if (tc_probe) {
        uint32_t tsp;
        probe_tc_cand_per_token(T, h->dix.n_centroid, h->n_sm, &tsp);
        CUDA_TRY(launch_probe_tc(qp, T, h->cen_sw, h->dix.centroid, h->dix.n_centroid, nprobe,
                                 tsp, w.cand, w.probe_id, w.probe_s, h->d_err, rs, &launches));
      } else {
        int splits;
        part_entries(h, T, nprobe, &splits);
        CUDA_TRY(launch_probe(h->dix, qp, T, nprobe, splits, w.part_id, w.part_s, w.probe_id,
                              w.probe_s, rs, &launches));
      }
      CUDA_TRY(rec(ev(bt, 2)));
      CUDA_TRY(launch_filter_hash(h->dix, w.probe_id, w.probe_s, nprobe, qo, qo + n_off,
                                  n_cta[bt], nb, w.fb_slots,
                                  probe_topk, scr, h->d_epoch, w.short_id, w.short_approx,
                                  w.n_short, w.qstat + (size_t)s * 3, rs, &launches,
                                  (flags & MVR_CAND_IMPUTE) ? 1 : 0));
      CUDA_TRY(rec(ev(bt, 3)));
      float *os = host_io ? w.out_s : out_s + (size_t)s * topk;
      uint32_t *oi = host_io ? w.out_id : out_id + (size_t)s * topk;
      if (bf16) {
        // tensor-core MaxSim (FP8 or BF16) over the shortlist -- with
        // MVR_PRUNE over the docs the pruner keeps -- then the exact FP32
        // kernel re-scores its best R docs
        const uint32_t *sid = w.short_id, *nsh = w.n_short;
        if (prune) {
          CUDA_TRY(launch_prune_features(h->dix, h->cen8, qp, qo, nb, w.short_id, w.n_short,
                                         probe_topk, h->x_bound, w.feat, h->d_err, rs,
                                         &launches, h->wait_ns));
          CUDA_TRY(launch_prune_mlp(w.feat, w.n_short, nb, probe_topk, h->prune_wts,
                                    h->prune_vecs, w.pred, h->d_err, h->n_sm, rs, &launches));
          CUDA_TRY(launch_topk(w.short_id, w.pred, w.n_short, nb, probe_topk, keep, w.kept_s,
                               w.kept_id, nullptr, rs, &launches));
          CUDA_TRY(launch_prune_choose(h->dix, w.short_id, w.n_short, w.kept_id, w.kept_s, nb,
                                       probe_topk, keep, R, h->prune_margin, w.fin_id, w.n_fin,
                                       w.qstat + (size_t)s * 3, h->d_fallback, rs, &launches));
          sid = w.fin_id;
          nsh = w.n_fin;
        }
        if (fp8)
          CUDA_TRY(launch_rerank_ws(h->dix, h->cen8, h->tw_fp8, qp, qo, nb, sid, nsh,
                                    probe_topk, sem, nq_max, h->x_bound, w.exact, h->d_err, rs,
                                    &launches, h->wait_ns, h->ws_docs));
        else if (h->cen_perm)
          CUDA_TRY(launch_rerank_tmem(h->dix, h->cen_perm, h->tw_bf16, qp, qo, nb, sid, nsh,
                                      probe_topk, sem, nq_max, h->x_bound, w.exact,
                                      h->d_err, rs, &launches, false));
        else
          CUDA_TRY(launch_rerank_tc(h->dix, h->cen_bf16, h->lut_bf16, qp, qo, nb, w.short_id,
                                    w.n_short, probe_topk, sem, nq_max, w.exact, h->d_err, rs,
                                    &launches));
        CUDA_TRY(rec(ev(bt, 4)));
        CUDA_TRY(launch_topk(sid, w.exact, nsh, nb, probe_topk, R, w.r_score, w.r_id, w.n_r, rs,
                             &launches));
        CUDA_TRY(launch_rerank(h->dix, qp, qo, nb, w.r_id, w.n_r, R, sem, w.r_exact, h->d_err,
                               rs, &launches, h->wait_ns));
        CUDA_TRY(launch_topk(w.r_id, w.r_exact, w.n_r, nb, R, topk, os, oi, nullptr, rs,
                             &launches));
      } else {
        // exact FP32 MaxSim over the shortlist -- with MVR_PRUNE over the docs
        // the pruner keeps (its fallback: the whole shortlist)
        const uint32_t *sid = w.short_id, *nsh = w.n_short;
        if (prune) {
          CUDA_TRY(launch_prune_features(h->dix, h->cen8, qp, qo, nb, w.short_id, w.n_short,
                                         probe_topk, h->x_bound, w.feat, h->d_err, rs,
                                         &launches, h->wait_ns));
          CUDA_TRY(launch_prune_mlp(w.feat, w.n_short, nb, probe_topk, h->prune_wts,
                                    h->prune_vecs, w.pred, h->d_err, h->n_sm, rs, &launches));
          CUDA_TRY(launch_topk(w.short_id, w.pred, w.n_short, nb, probe_topk, keep, w.kept_s,
                               w.kept_id, nullptr, rs, &launches));
          CUDA_TRY(launch_prune_choose(h->dix, w.short_id, w.n_short, w.kept_id, w.kept_s, nb,
                                       probe_topk, keep, R, h->prune_margin, w.fin_id, w.n_fin,
                                       w.qstat + (size_t)s * 3, h->d_fallback, rs, &launches));
          sid = w.fin_id;
          nsh = w.n_fin;
        }
        CUDA_TRY(launch_rerank(h->dix, qp, qo, nb, sid, nsh, probe_topk, sem, w.exact, h->d_err,
                               rs, &launches, h->wait_ns));
        CUDA_TRY(rec(ev(bt, 4)));
        CUDA_TRY(launch_topk(sid, w.exact, nsh, nb, probe_topk, topk, os, oi, nullptr, rs,
                             &launches));
      }
      CUDA_TRY(rec(ev(bt, 5)));
      if (host_io) {
        CUDA_TRY(cudaMemcpyAsync(out_s + (size_t)s * topk, w.out_s,
                                 (size_t)nb * topk * sizeof(float), cudaMemcpyDeviceToHost, rs));
        CUDA_TRY(cudaMemcpyAsync(out_id + (size_t)s * topk, w.out_id,
                                 (size_t)nb * topk * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 rs));
        d2h += (size_t)nb * topk * 8;
      }
    }
    CUDA_TRY(rec(h->events[(size_t)n_batch * kStages]));
    return MVR_OK;
  };

  const bool use_graph = h->graphs && !host_io;
  if (!use_graph) {
    MVR_TRY(enqueue(st, false));
  } else {
    // device buffers with graphs on: replay the recorded call when every
    // argument repeats, else record it (on the handle's stream, ordered
    // after the caller's stream) and keep the instantiated graph
    auto &G = h->graph;
    const bool same = G.exec && G.query == query && G.out_s == out_s && G.out_id == out_id &&
                      G.n_query == n_query && G.topk == topk && G.nprobe == nprobe &&
                      G.probe_topk == probe_topk && G.flags == flags && G.R == R && G.B == B &&
                      G.gen == h->ws_gen && G.off == off && G.cand_per_probe == cpe;
    CUDA_TRY(cudaEventRecord(h->ev_in, st));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_in, 0));
    if (!same) {
      h->drop_graph();
      CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue(h->stream, true);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
      if (rc != MVR_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ec != cudaSuccess) return set_err(MVR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
      const cudaError_t ei = cudaGraphInstantiate(&G.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        G.exec = nullptr;
        return set_err(MVR_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
      }
      G.query = query; G.out_s = out_s; G.out_id = out_id; G.n_query = n_query; G.topk = topk;
      G.nprobe = nprobe; G.probe_topk = probe_topk; G.flags = flags; G.R = R; G.B = B;
      G.gen = h->ws_gen; G.off = off; G.launches = launches; G.cand_per_probe = cpe;
    }
    launches = G.launches;
    CUDA_TRY(cudaEventRecord(h->ev_g0, h->stream));
    CUDA_TRY(cudaGraphLaunch(G.exec, h->stream));
    CUDA_TRY(cudaEventRecord(h->ev_g1, h->stream));
    CUDA_TRY(cudaEventRecord(h->ev_out, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(st, h->ev_out, 0));
  }
  CUDA_TRY(cudaMemcpyAsync(w.h_qstat, w.qstat, (size_t)n_query * 3 * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, st));
  unsigned herr = 0;
  unsigned long long n_fallback = 0;
  CUDA_TRY(cudaMemcpyAsync(&herr, h->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  if (prune)
    CUDA_TRY(cudaMemcpyAsync(&n_fallback, h->d_fallback, sizeof(n_fallback), cudaMemcpyDeviceToHost,
                             st));
  CUDA_TRY(cudaStreamSynchronize(st));
  CUDA_TRY(cudaGetLastError());
  if (herr) {
    CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(unsigned)));
    if (herr & 32u)
      return set_err(MVR_ERR_CUDA, "FP32 rerank: a pipeline wait timed out");
    if (herr & 16u)
      return set_err(MVR_ERR_CUDA, "FP8 rerank: query and doc token norms beyond the "
                                   "positive-offset range (2^21)");
    return set_err(MVR_ERR_CUDA, "tensor-core %s: a completion wait timed out",
                   (herr & 2u) ? "centroid scoring" : (herr & 8u) ? "pruner MLP" : "rerank");
  }

  {  // candidates per probed list, sizing the next call's hash filter
    double r = 0.0;
    for (uint32_t i = 0; i < n_query; i++) {
      const uint64_t probes = (off[i + 1] - off[i]) * (uint64_t)nprobe;
      if (probes) r = std::max(r, (double)w.h_qstat[i * 3 + 0] / (double)probes);
    }
    if (r > 0.0) h->cand_per_probe = r;
  }

  float total_ms = 0.f, max_ms = 0.f;
  if (use_graph)  // the graph launch as a whole, bracketed outside the graph
    CUDA_TRY(cudaEventElapsedTime(&total_ms, h->ev_g0, h->ev_g1));
  else
    CUDA_TRY(cudaEventElapsedTime(&total_ms, h->events[0], h->events[(size_t)n_batch * kStages]));
  // per-batch stage times from the events inside the pipeline (in a replayed
  // graph: its external event-record nodes; if the runtime cannot time
  // those, the stage times stay 0 and the total above still holds)
  auto elapsed = [&](float *ms, cudaEvent_t a, cudaEvent_t b) {
    if (cudaEventElapsedTime(ms, a, b) != cudaSuccess) {
      cudaGetLastError();
      *ms = 0.f;
    }
  };
  double stage_tot[kStages] = {0};
  for (uint32_t bt = 0; bt < n_batch; bt++) {
    float ms = 0.f, st_ms[kStages];
    elapsed(&ms, ev(bt, 0), h->events[(size_t)(bt + 1) * kStages]);
    for (int k = 0; k < kStages; k++) {
      elapsed(&st_ms[k], ev(bt, k), h->events[(size_t)bt * kStages + k + 1]);
      stage_tot[k] += st_ms[k];
    }
    max_ms = std::max(max_ms, ms);
    const uint32_t s = bt * B, e = std::min(n_query, s + B);
    for (uint32_t i = s; i < e; i++) {
      if (query_time_s) query_time_s[i] = ms * 1e-3;
      if (stage_s)
        for (int k = 0; k < kStages; k++) stage_s[(size_t)i * kStages + k] = st_ms[k] * 1e-3;
    }
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->device_ms = total_ms;
    stats->batch_ms_max = max_ms;
    stats->n_batch = n_batch;
    stats->gpu_launches = (uint32_t)launches;
    stats->h2d_bytes = h2d;
    stats->d2h_bytes = d2h;
    for (uint32_t i = 0; i < n_query; i++) {
      stats->n_cand_total += w.h_qstat[i * 3 + 0];
      stats->n_list_ent += w.h_qstat[i * 3 + 1];
      stats->n_rerank_tok += w.h_qstat[i * 3 + 2];
    }
    for (int k = 0; k < kStages; k++) stats->stage_ms[k] = stage_tot[k];
    stats->n_prune_fallback = n_fallback;
    stats->wall_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  }
  return MVR_OK;
}

int finish_index(mvr_index *h, const uint32_t *item_n_vec_host, const uint32_t *ivf_size_host,
                 const float *weight, std::unique_ptr<mvr_index> &owner, mvr_index **out) {
  DevIndex &d = h->dix;
  uint32_t mx = 0;
  for (uint32_t i = 0; i < d.n_item; i++) mx = std::max(mx, item_n_vec_host[i]);
  d.max_item_n_vec = mx;
  uint32_t ml = 0;
  for (uint32_t c = 0; c < d.n_centroid; c++) ml = std::max(ml, ivf_size_host[c]);
  h->max_ivf_list = ml;
  const std::vector<float> lut = make_lut(d.n_bit, weight);
  float *dl;
  MVR_TRY(dalloc(&dl, lut.size(), &h->bufs));
  CUDA_TRY(cudaMemcpy(dl, lut.data(), lut.size() * sizeof(float), cudaMemcpyHostToDevice));
  d.lut = dl;
  uint16_t *cb, *lb;
  MVR_TRY(dalloc(&cb, (size_t)d.n_centroid * kDim, &h->bufs));
  MVR_TRY(dalloc(&lb, lut.size(), &h->bufs));
  CUDA_TRY(make_bf16(d.centroid, (size_t)d.n_centroid * kDim, cb, h->stream));
  CUDA_TRY(make_bf16(dl, lut.size(), lb, h->stream));
  h->cen_bf16 = cb;
  h->lut_bf16 = lb;
  uint8_t *sw;
  MVR_TRY(dalloc(&sw, (size_t)d.n_centroid_pad * 256, &h->bufs));
  CUDA_TRY(make_centroid_tiles(d.centroid, d.n_centroid, d.n_centroid_pad / 64, sw, h->stream));
  h->cen_sw = sw;
  if (tmem_rerank_supported(d.n_bit) || fp8_rerank_supported(d.n_bit)) {
    float wmax = 0.f;
    for (uint32_t k = 0; k < (1u << d.n_bit); k++) wmax = std::max(wmax, std::fabs(weight[k]));
    float cmax = 0.f;
    CUDA_TRY(max_centroid_norm(d.centroid, d.n_centroid, h->d_err, &cmax, h->stream));
    CUDA_TRY(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->stream));  // was scratch
    h->x_bound = cmax + std::sqrt((float)kDim) * wmax;
  }
  if (tmem_rerank_supported(d.n_bit)) {
    uint32_t *cp;
    MVR_TRY(dalloc(&cp, (size_t)d.n_centroid * 64, &h->bufs));
    CUDA_TRY(make_centroid_perm(d.centroid, d.n_centroid, d.n_bit, cp, h->stream));
    h->cen_perm = cp;
    h->tw_bf16 = make_tm_weights(d.n_bit, weight, false);
  }
  if (fp8_rerank_supported(d.n_bit)) {
    uint8_t *c8;
    // one zero row past the last centroid: the FP8 rerank's padding rows
    MVR_TRY(dalloc(&c8, (size_t)(d.n_centroid + 1) * kDim, &h->bufs));
    CUDA_TRY(cudaMemsetAsync(c8 + (size_t)d.n_centroid * kDim, 0, kDim, h->stream));
    CUDA_TRY(make_centroid_fp8(d.centroid, d.n_centroid, d.n_bit, c8, h->stream));
    h->cen8 = c8;
    h->tw_fp8 = make_tm_weights(d.n_bit, weight, true);
  }
  uint32_t *ipart;
  MVR_TRY(dalloc(&ipart, (size_t)d.n_centroid * (kHashParts + 1), &h->bufs));
  CUDA_TRY(make_ivf_part(d, ipart, h->stream));
  d.ivf_part = ipart;
  float *ct;
  MVR_TRY(dalloc(&ct, (size_t)kDim * d.n_centroid_pad, &h->bufs));
  CUDA_TRY(launch_transpose_centroid(d.centroid, d.n_centroid, d.n_centroid_pad, ct, h->stream));
  d.centroid_t = ct;
  unsigned *flag;
  MVR_TRY(dalloc(&flag, 1));
  std::unique_ptr<void, void (*)(void *)> flag_guard(flag, dfree);
  CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned), h->stream));
  validate_kernel<<<4 * h->n_sm, 256, 0, h->stream>>>(d.vq_code, d.n_vec, d.n_centroid, d.ivf_ids,
                                                     d.n_ele_ivf, d.n_item, flag);
  CUDA_TRY(cudaGetLastError());
  unsigned hflag = 0;
  CUDA_TRY(cudaMemcpyAsync(&hflag, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (hflag & 1u) return set_err(MVR_ERR_INVALID_ARG, "vq_code holds a centroid id >= n_centroid");
  if (hflag & 2u) return set_err(MVR_ERR_INVALID_ARG, "ivf holds a doc id >= n_item");
  h->device_bytes = 0;
  h->device_bytes += (size_t)d.n_centroid * kDim * 4 * 1 + (size_t)kDim * d.n_centroid_pad * 4;
  h->device_bytes += d.n_vec * (4 + d.bytes_per_vec) + (size_t)d.n_item * 12;
  h->device_bytes += (size_t)d.n_centroid * 12 + d.n_ele_ivf * 4 + lut.size() * 4;
  h->batch_cap = 0;
  *out = owner.release();
  return MVR_OK;
}

int check_index_args(uint32_t n_item, uint32_t n_centroid, uint32_t dim, uint64_t n_vec,
                     uint32_t n_bit) {
  if (dim != (uint32_t)kDim)
    return set_err(MVR_ERR_UNSUPPORTED, "vector dimension %u is not supported (only %d)", dim, kDim);
  if (n_bit != 1 && n_bit != 2 && n_bit != 4 && n_bit != 8)
    return set_err(MVR_ERR_INVALID_ARG, "n_bit must be 1, 2, 4 or 8, got %u", n_bit);
  if (n_item == 0 || n_centroid == 0 || n_vec == 0)
    return set_err(MVR_ERR_INVALID_ARG, "empty index (n_item=%u n_centroid=%u n_vec=%llu)", n_item,
                   n_centroid, (unsigned long long)n_vec);
  return MVR_OK;
}

int new_handle(int device, std::unique_ptr<mvr_index> &h) {
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    cudaGetLastError();
    return set_err(MVR_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= n_dev)
    return set_err(MVR_ERR_INVALID_ARG, "device %d out of range (have %d)", device, n_dev);
  h.reset(new mvr_index());
  h->device = device;
  CUDA_TRY(cudaSetDevice(device));
  CUDA_TRY(cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(configure_kernels());
  CUDA_TRY(configure_tc_kernels());
  CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  MVR_TRY(dalloc(&h->d_err, 1));
  CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(unsigned)));
  MVR_TRY(dalloc(&h->d_epoch, 1));
  CUDA_TRY(cudaMemset(h->d_epoch, 0, sizeof(uint32_t)));
  CUDA_TRY(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreate(&h->ev_g0));
  CUDA_TRY(cudaEventCreate(&h->ev_g1));
  return MVR_OK;
}

template <class T>
int upload(const T *src, size_t n, T **dst, std::vector<void *> &owner, cudaMemcpyKind kind,
           size_t pad = 0) {
  MVR_TRY(dalloc(dst, n + pad, &owner));
  if (n) CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), kind));
  if (pad) CUDA_TRY(cudaMemset(*dst + n, 0, pad * sizeof(T)));
  return MVR_OK;
}

int from_arrays_impl(const uint32_t *item_n_vec_l, uint32_t n_item, const float *centroid_l,
                     uint32_t n_centroid, uint32_t dim, const uint32_t *vq_code_l, uint64_t n_vec,
                     const uint64_t *ivf_offset_l, const uint32_t *ivf_size_l, const uint32_t *ivf,
                     uint64_t n_ele_ivf, const float *weight_l, uint32_t n_bit,
                     const uint8_t *residual_code_l, int device, mvr_index **out, bool on_device) {
  if (!out) return set_err(MVR_ERR_INVALID_ARG, "null output handle");
  *out = nullptr;
  MVR_TRY(check_index_args(n_item, n_centroid, dim, n_vec, n_bit));
  if (!item_n_vec_l || !centroid_l || !vq_code_l || !ivf_offset_l || !ivf_size_l || !weight_l ||
      !residual_code_l || (n_ele_ivf && !ivf))
    return set_err(MVR_ERR_INVALID_ARG, "null index array");
  DeviceGuard g(device);
  std::unique_ptr<mvr_index> h;
  MVR_TRY(new_handle(device, h));
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;

  // host copies of the small arrays the host logic needs
  std::vector<uint32_t> inv(n_item), isz(n_centroid);
  std::vector<uint64_t> ioff(n_centroid);
  CUDA_TRY(cudaMemcpy(inv.data(), item_n_vec_l, n_item * 4ull, on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
  CUDA_TRY(cudaMemcpy(isz.data(), ivf_size_l, n_centroid * 4ull, on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
  CUDA_TRY(cudaMemcpy(ioff.data(), ivf_offset_l, n_centroid * 8ull, on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
  std::vector<float> weight(1u << n_bit);
  CUDA_TRY(cudaMemcpy(weight.data(), weight_l, weight.size() * 4, on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
  uint64_t tot = 0;
  std::vector<uint64_t> item_off(n_item);
  for (uint32_t i = 0; i < n_item; i++) { item_off[i] = tot; tot += inv[i]; }
  if (tot != n_vec)
    return set_err(MVR_ERR_INVALID_ARG, "sum of item_n_vec (%llu) != n_vec (%llu)",
                   (unsigned long long)tot, (unsigned long long)n_vec);
  for (uint32_t c = 0; c < n_centroid; c++)
    if (ioff[c] + isz[c] > n_ele_ivf)
      return set_err(MVR_ERR_INVALID_ARG, "ivf list %u exceeds n_ele_ivf", c);

  DevIndex &d = h->dix;
  d.n_item = n_item;
  d.n_centroid = n_centroid;
  d.n_centroid_pad = (n_centroid + 127u) / 128u * 128u;
  d.n_bit = n_bit;
  d.bytes_per_vec = kDim * n_bit / 8;
  d.n_vec = n_vec;
  d.n_ele_ivf = n_ele_ivf;
  float *cen;
  uint32_t *code, *dinv, *dsz, *dids;
  uint8_t *res;
  uint64_t *doff, *dioff;
  MVR_TRY(upload(centroid_l, (size_t)n_centroid * kDim, &cen, h->bufs, kind));
  // 16 zero bytes past the codes: the FP8 rerank copies each doc group's
  // codes in 16-byte-aligned bulk copies that may round up past the last one
  MVR_TRY(upload(vq_code_l, (size_t)n_vec, &code, h->bufs, kind, 4));
  MVR_TRY(upload(residual_code_l, (size_t)n_vec * d.bytes_per_vec, &res, h->bufs, kind));
  MVR_TRY(upload(inv.data(), n_item, &dinv, h->bufs, cudaMemcpyHostToDevice));
  MVR_TRY(upload(item_off.data(), n_item, &doff, h->bufs, cudaMemcpyHostToDevice));
  MVR_TRY(upload(ioff.data(), n_centroid, &dioff, h->bufs, cudaMemcpyHostToDevice));
  MVR_TRY(upload(isz.data(), n_centroid, &dsz, h->bufs, cudaMemcpyHostToDevice));
  MVR_TRY(upload(ivf, (size_t)n_ele_ivf, &dids, h->bufs, kind));
  d.centroid = cen;
  d.vq_code = code;
  d.residual = res;
  d.item_n_vec = dinv;
  d.item_off = doff;
  d.ivf_off = dioff;
  d.ivf_size = dsz;
  d.ivf_ids = dids;
  return finish_index(h.get(), inv.data(), isz.data(), weight.data(), h, out);
}

bool npy_u32(const NpyArray &a, std::vector<uint32_t> &out) {
  const uint64_t n = a.numel();
  out.resize(n);
  const std::string t = a.descr.substr(1);
  if (t == "u4" || t == "i4") {
    std::memcpy(out.data(), a.data.data(), n * 4);
  } else if (t == "u8" || t == "i8") {
    const int64_t *p = reinterpret_cast<const int64_t *>(a.data.data());
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)p[i];
  } else {
    return false;
  }
  return true;
}

}  // namespace

// Read access to a handle's device and HBM-resident index arrays for other
// translation units of the library (not part of the C ABI).
namespace mvr {
const DevIndex *handle_index(const mvr_index *h, int *device) {
  if (device) *device = h->device;
  return &h->dix;
}
// Sets the calling thread's mvr_last_error() text; returns code.
int record_error(int code, const char *msg) { return set_err(code, "%s", msg); }
}  // namespace mvr

// ----------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------
extern "C" {

const char *mvr_last_error(void) { return g_err.c_str(); }

int mvr_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int mvr_index_from_arrays(const uint32_t *item_n_vec_l, uint32_t n_item, const float *centroid_l,
                          uint32_t n_centroid, uint32_t dim, const uint32_t *vq_code_l,
                          uint64_t n_vec, const uint64_t *ivf_offset_l, const uint32_t *ivf_size_l,
                          const uint32_t *ivf, uint64_t n_ele_ivf, const float *weight_l,
                          uint32_t n_bit, const uint8_t *residual_code_l, int device,
                          mvr_index **out) {
  return from_arrays_impl(item_n_vec_l, n_item, centroid_l, n_centroid, dim, vq_code_l, n_vec,
                          ivf_offset_l, ivf_size_l, ivf, n_ele_ivf, weight_l, n_bit,
                          residual_code_l, device, out, false);
}

int mvr_index_from_device_arrays(const uint32_t *item_n_vec_l, uint32_t n_item,
                                 const float *centroid_l, uint32_t n_centroid, uint32_t dim,
                                 const uint32_t *vq_code_l, uint64_t n_vec,
                                 const uint64_t *ivf_offset_l, const uint32_t *ivf_size_l,
                                 const uint32_t *ivf, uint64_t n_ele_ivf, const float *weight_l,
                                 uint32_t n_bit, const uint8_t *residual_code_l, int device,
                                 mvr_index **out) {
  return from_arrays_impl(item_n_vec_l, n_item, centroid_l, n_centroid, dim, vq_code_l, n_vec,
                          ivf_offset_l, ivf_size_l, ivf, n_ele_ivf, weight_l, n_bit,
                          residual_code_l, device, out, true);
}

int mvr_index_load(const char *index_dir, uint32_t n_centroid, uint32_t n_bit, int device,
                   mvr_index **out) {
  if (!index_dir || !out) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  const std::string dir(index_dir);
  return mvr_index_load_files((dir + "/item_n_vec_l.npy").c_str(), (dir + "/centroid_l.npy").c_str(),
                              (dir + "/vq_code_l.npy").c_str(), (dir + "/ivf.index").c_str(),
                              (dir + "/weight_l.npy").c_str(), (dir + "/residual_code_l.npy").c_str(),
                              n_centroid, n_bit, device, out);
}

int mvr_index_load_files(const char *item_n_vec_l_fname, const char *centroid_l_fname,
                         const char *vq_code_l_fname, const char *ivf_index_fname,
                         const char *weight_l_fname, const char *residual_code_l_fname,
                         uint32_t n_centroid, uint32_t n_bit, int device, mvr_index **out) {
  if (!item_n_vec_l_fname || !centroid_l_fname || !vq_code_l_fname || !ivf_index_fname ||
      !weight_l_fname || !residual_code_l_fname || !out)
    return set_err(MVR_ERR_INVALID_ARG, "null argument");
  std::string err;
  NpyArray a_inv, a_cen, a_code, a_w, a_res;
  if (!npy_load(item_n_vec_l_fname, a_inv, err) || !npy_load(centroid_l_fname, a_cen, err) ||
      !npy_load(vq_code_l_fname, a_code, err) || !npy_load(weight_l_fname, a_w, err) ||
      !npy_load(residual_code_l_fname, a_res, err))
    return set_err(MVR_ERR_IO, "%s", err.c_str());
  IvfCsr ivf;
  if (!ivf_load(ivf_index_fname, ivf, err)) return set_err(MVR_ERR_IO, "%s", err.c_str());
  std::vector<uint32_t> inv, code;
  if (a_inv.shape.size() != 1 || !npy_u32(a_inv, inv))
    return set_err(MVR_ERR_IO, "item_n_vec_l.npy: expected 1-D integer array (%s)", a_inv.descr.c_str());
  if (a_code.shape.size() != 1 || !npy_u32(a_code, code))
    return set_err(MVR_ERR_IO, "vq_code_l.npy: expected 1-D integer array (%s)", a_code.descr.c_str());
  if (a_cen.shape.size() != 2 || a_cen.descr.substr(1) != "f4")
    return set_err(MVR_ERR_IO, "centroid_l.npy: expected 2-D float32 array");
  if (a_w.shape.size() != 1 || a_w.descr.substr(1) != "f4")
    return set_err(MVR_ERR_IO, "weight_l.npy: expected 1-D float32 array");
  if (a_res.descr.substr(1) != "u1")
    return set_err(MVR_ERR_IO, "residual_code_l.npy: expected uint8 array");
  const uint32_t C = (uint32_t)a_cen.shape[0], dim = (uint32_t)a_cen.shape[1];
  if (C != n_centroid)
    return set_err(MVR_ERR_INVALID_ARG, "centroid_l.npy has %u centroids, expected %u", C, n_centroid);
  if (ivf.n_centroid != n_centroid)
    return set_err(MVR_ERR_IO, "ivf.index has %u lists, expected %u", ivf.n_centroid, n_centroid);
  if (a_w.shape[0] != (1ull << n_bit))
    return set_err(MVR_ERR_INVALID_ARG, "weight_l.npy has %llu weights, n_bit=%u needs %u",
                   (unsigned long long)a_w.shape[0], n_bit, 1u << n_bit);
  MVR_TRY(check_index_args((uint32_t)inv.size(), C, dim, code.size(), n_bit));
  const uint64_t bpv = (uint64_t)dim * n_bit / 8;
  if (a_res.numel() != code.size() * bpv)
    return set_err(MVR_ERR_IO, "residual_code_l.npy has %llu bytes, expected %llu",
                   (unsigned long long)a_res.numel(), (unsigned long long)(code.size() * bpv));
  return mvr_index_from_arrays(inv.data(), (uint32_t)inv.size(),
                               reinterpret_cast<const float *>(a_cen.data.data()), C, dim,
                               code.data(), code.size(), ivf.offset.data(), ivf.size.data(),
                               ivf.ids.data(), ivf.n_ele,
                               reinterpret_cast<const float *>(a_w.data.data()), n_bit,
                               a_res.data.data(), device, out);
}

int mvr_index_free(mvr_index *h) {
  delete h;
  return MVR_OK;
}

int mvr_index_get_info(const mvr_index *h, mvr_index_info *info) {
  if (!h || !info) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  info->n_item = h->dix.n_item;
  info->n_centroid = h->dix.n_centroid;
  info->dim = kDim;
  info->n_bit = h->dix.n_bit;
  info->n_vec = h->dix.n_vec;
  info->n_ele_ivf = h->dix.n_ele_ivf;
  info->max_item_n_vec = h->dix.max_item_n_vec;
  info->max_ivf_list = h->max_ivf_list;
  info->device_bytes = h->device_bytes;
  info->device = h->device;
  return MVR_OK;
}

int mvr_index_set_batch(mvr_index *h, uint32_t max_batch_queries) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  h->batch_cap = max_batch_queries;
  return MVR_OK;
}

int mvr_index_set_graphs(mvr_index *h, int enable) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  h->graphs = enable != 0;
  if (!h->graphs) {
    DeviceGuard g(h->device);
    h->drop_graph();
  }
  return MVR_OK;
}

int mvr_index_set_pruner(mvr_index *h, const float *params, uint32_t keep, float margin) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  DeviceGuard g(h->device);
  h->drop_graph();
  if (!params) {
    dfree(h->prune_wts);
    dfree(h->prune_vecs);
    h->prune_wts = nullptr;
    h->prune_vecs = nullptr;
    return MVR_OK;
  }
  if (keep == 0) return set_err(MVR_ERR_INVALID_ARG, "keep must be >= 1");
  if (!fp8_rerank_supported(h->dix.n_bit))
    return set_err(MVR_ERR_UNSUPPORTED, "the pruner's features need a 2- or 4-bit index");
  if (!h->prune_wts) {
    MVR_TRY(dalloc(&h->prune_wts, prune_weight_bytes()));
    MVR_TRY(dalloc(&h->prune_vecs, 769));
  }
  if (!h->d_fallback) MVR_TRY(dalloc(&h->d_fallback, 1));
  float *tmp = nullptr;
  MVR_TRY(dalloc(&tmp, kNumParams));
  cudaError_t e = cudaMemcpy(tmp, params, kNumParams * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = prune_prepare(tmp, h->prune_wts, h->prune_vecs, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dfree(tmp);
  CUDA_TRY(e);
  h->prune_keep = keep;
  h->prune_margin = margin;
  return MVR_OK;
}

int mvr_index_set_rerank_tile(mvr_index *h, uint32_t docs_per_cta) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  if (docs_per_cta == 0) docs_per_cta = 256;
  if (!ws_docs_supported(docs_per_cta))
    return set_err(MVR_ERR_INVALID_ARG, "docs per CTA %u: 32, 64, 128 or 256", docs_per_cta);
  DeviceGuard g(h->device);
  h->ws_docs = docs_per_cta;
  h->drop_graph();
  return MVR_OK;
}

int mvr_index_set_wait_limit(mvr_index *h, uint64_t wait_ns) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  DeviceGuard g(h->device);
  h->wait_ns = wait_ns ? wait_ns : 1000000000ull;
  h->drop_graph();  // recorded launches carry the old bound
  return MVR_OK;
}

int mvr_index_set_rescore(mvr_index *h, uint32_t n_rescore) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  h->rescore = n_rescore;
  return MVR_OK;
}

int mvr_search(mvr_index *h, const float *query_l, const uint64_t *tok_off, uint32_t n_query,
               uint32_t query_n_vec, uint32_t topk, uint32_t nprobe, uint32_t probe_topk,
               uint32_t flags, float *result_score_l, uint32_t *result_id_l, double *query_time_s,
               mvr_stats *stats) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  return search_impl(h, query_l, tok_off, n_query, query_n_vec, topk, nprobe, probe_topk, flags,
                     result_score_l, result_id_l, query_time_s, nullptr, stats, h->stream, true);
}

int mvr_search_staged(mvr_index *h, const float *query_l, const uint64_t *tok_off,
                      uint32_t n_query, uint32_t query_n_vec, uint32_t topk, uint32_t nprobe,
                      uint32_t probe_topk, uint32_t flags, float *result_score_l,
                      uint32_t *result_id_l, double *query_time_s, double *stage_time_s,
                      mvr_stats *stats) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  return search_impl(h, query_l, tok_off, n_query, query_n_vec, topk, nprobe, probe_topk, flags,
                     result_score_l, result_id_l, query_time_s, stage_time_s, stats, h->stream,
                     true);
}

int mvr_search_device(mvr_index *h, const float *d_query_l, const uint64_t *tok_off,
                      uint32_t n_query, uint32_t query_n_vec, uint32_t topk, uint32_t nprobe,
                      uint32_t probe_topk, uint32_t flags, float *d_result_score_l,
                      uint32_t *d_result_id_l, void *cuda_stream, mvr_stats *stats) {
  if (!h) return set_err(MVR_ERR_INVALID_ARG, "null index handle");
  cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : (cudaStream_t)0;
  return search_impl(h, d_query_l, tok_off, n_query, query_n_vec, topk, nprobe, probe_topk, flags,
                     d_result_score_l, d_result_id_l, nullptr, nullptr, stats, st, false);
}

int mvr_search_trace(mvr_index *h, const float *query, uint32_t nq, uint32_t topk,
                     uint32_t nprobe, uint32_t probe_topk, uint32_t flags, mvr_trace *tr) {
  if (!h || !query || !tr) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (!tr->topk_score || !tr->topk_id) return set_err(MVR_ERR_INVALID_ARG, "null trace result buffer");
  if (flags & MVR_PRUNE)
    return set_err(MVR_ERR_UNSUPPORTED, "trace the pruner through short_pred, not MVR_PRUNE");
  if ((tr->short_feat || tr->short_pred) && (!h->cen8 || nq > 32))
    return set_err(MVR_ERR_UNSUPPORTED, "pruner features: a 2- or 4-bit index, <= 32 tokens");
  if (tr->short_pred && !h->prune_wts) return set_err(MVR_ERR_INVALID_ARG, "no pruner set");
  MVR_TRY(search_impl(h, query, nullptr, 1, nq, topk, nprobe, probe_topk, flags, tr->topk_score,
                      tr->topk_id, nullptr, nullptr, nullptr, h->stream, true));
  DeviceGuard g(h->device);
  Workspace &w = h->ws;
  if (tr->probe_id)
    CUDA_TRY(cudaMemcpy(tr->probe_id, w.probe_id, (size_t)nq * nprobe * 4, cudaMemcpyDeviceToHost));
  if (tr->probe_score)
    CUDA_TRY(cudaMemcpy(tr->probe_score, w.probe_s, (size_t)nq * nprobe * 4, cudaMemcpyDeviceToHost));
  uint32_t n_short = 0;
  CUDA_TRY(cudaMemcpy(&n_short, w.n_short, 4, cudaMemcpyDeviceToHost));
  const uint32_t n_cand = w.h_qstat[0];
  tr->n_cand = n_cand;
  tr->n_short = n_short;
  if (tr->cand_id || tr->cand_score) {
    // the query's keys: the hash filter's, or the rank-table fallback's when
    // the query overflowed the hash tables
    uint32_t ovf = 0;
    CUDA_TRY(cudaMemcpy(&ovf, w.ovf, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<uint64_t> keys(n_cand);
    if (n_cand)
      CUDA_TRY(cudaMemcpy(keys.data(), ovf ? w.key : w.hkey, (size_t)n_cand * 8,
                          cudaMemcpyDeviceToHost));
    std::sort(keys.begin(), keys.end(),
              [](uint64_t a, uint64_t b) { return key_id(a) < key_id(b); });
    for (uint32_t i = 0; i < n_cand && i < tr->cand_cap; i++) {
      if (tr->cand_id) tr->cand_id[i] = key_id(keys[i]);
      if (tr->cand_score) tr->cand_score[i] = key_score(keys[i]);
    }
  }
  std::vector<uint32_t> sid(n_short);
  std::vector<float> sa(n_short), se(n_short);
  if (n_short) {
    CUDA_TRY(cudaMemcpy(sid.data(), w.short_id, n_short * 4ull, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(sa.data(), w.short_approx, n_short * 4ull, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(se.data(), w.exact, n_short * 4ull, cudaMemcpyDeviceToHost));
  }
  std::vector<uint32_t> ord(n_short);
  for (uint32_t i = 0; i < n_short; i++) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return sid[a] < sid[b]; });
  for (uint32_t i = 0; i < n_short; i++) {
    if (tr->short_id) tr->short_id[i] = sid[ord[i]];
    if (tr->short_approx) tr->short_approx[i] = sa[ord[i]];
    if (tr->short_exact) tr->short_exact[i] = se[ord[i]];
  }
  if ((tr->short_feat || tr->short_pred) && n_short) {
    // the shortlist's pruner features (and predictions), as the search
    // computes them
    float *d_feat = nullptr, *d_pred = nullptr;
    int l = 0;
    MVR_TRY(dalloc(&d_feat, (size_t)probe_topk * 33));
    MVR_TRY(dalloc(&d_pred, probe_topk));
    std::vector<float> f((size_t)n_short * 33), p(n_short);
    cudaError_t e = launch_prune_features(h->dix, h->cen8, w.q, w.q_off, 1, w.short_id, w.n_short,
                                          probe_topk, h->x_bound, d_feat, h->d_err, h->stream, &l,
                                          h->wait_ns);
    if (e == cudaSuccess && tr->short_pred)
      e = launch_prune_mlp(d_feat, w.n_short, 1, probe_topk, h->prune_wts, h->prune_vecs, d_pred,
                           h->d_err, h->n_sm, h->stream, &l);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(f.data(), d_feat, f.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(p.data(), d_pred, p.size() * 4, cudaMemcpyDeviceToHost);
    unsigned herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, h->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    dfree(d_feat);
    dfree(d_pred);
    CUDA_TRY(e);
    if (herr) {
      CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(unsigned)));
      return set_err(MVR_ERR_CUDA, "pruner features: a completion wait timed out");
    }
    for (uint32_t i = 0; i < n_short; i++) {
      if (tr->short_feat)
        std::memcpy(tr->short_feat + (size_t)i * 33, f.data() + (size_t)ord[i] * 33, 33 * 4);
      if (tr->short_pred) tr->short_pred[i] = p[ord[i]];
    }
  }
  return MVR_OK;
}

static int gather_vec_ids(mvr_index *h, const uint64_t *vec_id, uint64_t n, uint64_t **d_ids) {
  for (uint64_t i = 0; i < n; i++)
    if (vec_id[i] >= h->dix.n_vec)
      return set_err(MVR_ERR_INVALID_ARG, "token id %llu >= n_vec %llu",
                     (unsigned long long)vec_id[i], (unsigned long long)h->dix.n_vec);
  MVR_TRY(dalloc(d_ids, n));
  CUDA_TRY(cudaMemcpy(*d_ids, vec_id, n * 8, cudaMemcpyHostToDevice));
  return MVR_OK;
}

int mvr_decompress(mvr_index *h, const uint64_t *vec_id, uint64_t n, float *out) {
  if (!h || (n && (!vec_id || !out))) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (n == 0) return MVR_OK;
  DeviceGuard g(h->device);
  uint64_t *ids;
  MVR_TRY(gather_vec_ids(h, vec_id, n, &ids));
  std::unique_ptr<void, void (*)(void *)> ig(ids, dfree);
  float *d_out;
  MVR_TRY(dalloc(&d_out, n * kDim));
  std::unique_ptr<void, void (*)(void *)> og(d_out, dfree);
  CUDA_TRY(launch_decompress(h->dix, ids, n, d_out, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(out, d_out, n * kDim * sizeof(float), cudaMemcpyDeviceToHost));
  return MVR_OK;
}

int mvr_unpack_buckets(mvr_index *h, const uint64_t *vec_id, uint64_t n, uint8_t *out) {
  if (!h || (n && (!vec_id || !out))) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (n == 0) return MVR_OK;
  DeviceGuard g(h->device);
  uint64_t *ids;
  MVR_TRY(gather_vec_ids(h, vec_id, n, &ids));
  std::unique_ptr<void, void (*)(void *)> ig(ids, dfree);
  uint8_t *d_out;
  MVR_TRY(dalloc(&d_out, n * kDim));
  std::unique_ptr<void, void (*)(void *)> og(d_out, dfree);
  CUDA_TRY(launch_unpack(h->dix, ids, n, d_out, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(out, d_out, n * kDim, cudaMemcpyDeviceToHost));
  return MVR_OK;
}

int mvr_assign_device(const float *d_vec, uint64_t n_vec, const float *d_centroid,
                      uint32_t n_centroid, uint32_t dim, uint32_t *d_code, float *d_score,
                      void *cuda_stream) {
  if (dim != (uint32_t)kDim) return set_err(MVR_ERR_UNSUPPORTED, "dim %u not supported", dim);
  if (!d_vec || !d_centroid || !d_code || n_centroid == 0)
    return set_err(MVR_ERR_INVALID_ARG, "null argument or no centroids");
  if (mvr_device_count() == 0) return set_err(MVR_ERR_CUDA, "no CUDA device available");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(configure_kernels());
  DevIndex d{};
  d.n_centroid = n_centroid;
  d.n_centroid_pad = (n_centroid + 127u) / 128u * 128u;
  float *ct;
  MVR_TRY(dalloc(&ct, (size_t)kDim * d.n_centroid_pad));
  std::unique_ptr<void, void (*)(void *)> cg(ct, dfree);
  CUDA_TRY(launch_transpose_centroid(d_centroid, n_centroid, d.n_centroid_pad, ct, st));
  d.centroid_t = ct;
  float *score = d_score;
  std::unique_ptr<void, void (*)(void *)> sg(nullptr, dfree);
  if (!score) {
    const uint64_t chunk_max = std::min<uint64_t>(n_vec, 2ull << 20);
    MVR_TRY(dalloc(&score, chunk_max));
    sg.reset(score);
  }
  int launches = 0;
  for (uint64_t s = 0; s < n_vec; s += (2ull << 20)) {  // grid.y <= 32768
    const uint32_t T = (uint32_t)std::min<uint64_t>(2ull << 20, n_vec - s);
    CUDA_TRY(launch_probe(d, d_vec + s * kDim, T, 1, 1, nullptr, nullptr, d_code + s,
                          d_score ? d_score + s : score, st, &launches));
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  return MVR_OK;
}

int mvr_assign_tc_device(const float *d_vec, uint64_t n_vec, const float *d_centroid,
                         uint32_t n_centroid, uint32_t dim, uint32_t *d_code, float *d_score,
                         void *cuda_stream) {
  if (dim != (uint32_t)kDim) return set_err(MVR_ERR_UNSUPPORTED, "dim %u not supported", dim);
  if (!d_vec || !d_centroid || !d_code || n_centroid == 0)
    return set_err(MVR_ERR_INVALID_ARG, "null argument or no centroids");
  if (mvr_device_count() == 0) return set_err(MVR_ERR_CUDA, "no CUDA device available");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(configure_tc_kernels());
  int dev = 0, n_sm = 148;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  // swizzled BF16 centroid tiles (64 centroids x 256 B each)
  const uint32_t n_tiles = (n_centroid + 63u) / 64u;
  uint8_t *sw;
  MVR_TRY(dalloc(&sw, (size_t)n_tiles * 64 * 256));
  std::unique_ptr<void, void (*)(void *)> swg(sw, dfree);
  CUDA_TRY(make_centroid_tiles(d_centroid, n_centroid, n_tiles, sw, st));
  // token chunks of <= 1M (probe grid.y <= 8192); candidate lists sized
  // for the largest chunk's split count
  const uint64_t kChunk = 1ull << 20;
  size_t cand_need = 1;
  for (uint64_t s = 0; s < n_vec; s += kChunk) {
    const uint32_t T = (uint32_t)std::min<uint64_t>(kChunk, n_vec - s);
    uint32_t sp;
    cand_need = std::max(cand_need, (size_t)T * probe_tc_cand_per_token(T, n_centroid, n_sm, &sp));
  }
  uint32_t *cand;
  MVR_TRY(dalloc(&cand, cand_need));
  std::unique_ptr<void, void (*)(void *)> cg(cand, dfree);
  float *score = d_score;
  std::unique_ptr<void, void (*)(void *)> sg(nullptr, dfree);
  if (!score) {
    MVR_TRY(dalloc(&score, std::min<uint64_t>(std::max<uint64_t>(n_vec, 1), kChunk)));
    sg.reset(score);
  }
  unsigned *err;
  MVR_TRY(dalloc(&err, 1));
  std::unique_ptr<void, void (*)(void *)> eg(err, dfree);
  CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned), st));
  int launches = 0;
  for (uint64_t s = 0; s < n_vec; s += kChunk) {
    const uint32_t T = (uint32_t)std::min<uint64_t>(kChunk, n_vec - s);
    uint32_t sp;
    probe_tc_cand_per_token(T, n_centroid, n_sm, &sp);
    CUDA_TRY(launch_probe_tc(d_vec + s * kDim, T, sw, d_centroid, n_centroid, 1, sp, cand,
                             d_code + s, d_score ? d_score + s : score, err, st, &launches));
  }
  unsigned herr = 0;
  CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return set_err(MVR_ERR_CUDA, "tensor-core scoring gave up waiting (flags %u)", herr);
  return MVR_OK;
}

int mvr_pack_residual_device(const float *d_vec, uint64_t n_vec, const float *d_centroid,
                             uint32_t dim, const uint32_t *d_code, const float *cutoff_l,
                             uint32_t n_bit, uint8_t *d_out, void *cuda_stream) {
  if (dim != (uint32_t)kDim) return set_err(MVR_ERR_UNSUPPORTED, "dim %u not supported", dim);
  if (n_bit != 1 && n_bit != 2 && n_bit != 4 && n_bit != 8)
    return set_err(MVR_ERR_INVALID_ARG, "n_bit must be 1, 2, 4 or 8");
  if (!d_vec || !d_centroid || !d_code || !cutoff_l || !d_out)
    return set_err(MVR_ERR_INVALID_ARG, "null argument");
  Cutoffs cut{};
  for (uint32_t i = 0; i + 1 < (1u << n_bit); i++) cut.v[i] = cutoff_l[i];
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(launch_pack_residual(d_vec, n_vec, d_centroid, d_code, cut, n_bit, d_out, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return MVR_OK;
}

int mvr_residual_quantiles_device(const float *d_vec, uint64_t n_vec, const float *d_centroid,
                                  uint32_t dim, const uint32_t *d_code, uint32_t n_bit,
                                  float *cutoff_out, float *weight_out, void *cuda_stream) {
  if (dim != (uint32_t)kDim) return set_err(MVR_ERR_UNSUPPORTED, "dim %u not supported", dim);
  if (n_bit != 1 && n_bit != 2 && n_bit != 4 && n_bit != 8)
    return set_err(MVR_ERR_INVALID_ARG, "n_bit must be 1, 2, 4 or 8");
  if (!d_vec || !d_centroid || !d_code || !cutoff_out || !weight_out)
    return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (n_vec == 0) return set_err(MVR_ERR_INVALID_ARG, "no vectors");
  const uint32_t nq = 1u << n_bit;
  const double n = (double)(n_vec * (uint64_t)kDim);
  std::vector<uint64_t> rank;
  for (uint32_t c = 0; c + 1 < nq; c++) rank.push_back((uint64_t)std::floor((1.0 * (c + 1) / nq) * n));
  for (uint32_t w = 0; w < nq; w++) rank.push_back((uint64_t)std::floor((1.0 * w / nq + 0.5 / nq) * n));
  std::vector<float> v(rank.size());
  CUDA_TRY(residual_select(d_vec, n_vec, d_centroid, d_code, rank.data(), (uint32_t)rank.size(),
                           v.data(), (cudaStream_t)cuda_stream));
  for (uint32_t c = 0; c + 1 < nq; c++) cutoff_out[c] = v[c];
  for (uint32_t w = 0; w < nq; w++) weight_out[w] = v[nq - 1 + w];
  return MVR_OK;
}

int mvr_kmeans_accumulate_device(const float *d_vec, uint64_t n_vec, uint32_t dim,
                                 const uint32_t *d_code, double *d_sum, uint64_t *d_count,
                                 void *cuda_stream) {
  if (dim != (uint32_t)kDim) return set_err(MVR_ERR_UNSUPPORTED, "dim %u not supported", dim);
  if (!d_vec || !d_code || !d_sum || !d_count) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(launch_kmeans_accumulate(d_vec, n_vec, d_code, d_sum, d_count, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return MVR_OK;
}

size_t mvr_mlp_work_floats(uint32_t n) { return mlp_work_floats(n); }

int mvr_mlp_train_step(const float *d_x, const float *d_y, uint32_t n, float *d_params,
                       float *d_adam_m, float *d_adam_v, float *d_work, float lr, uint32_t step,
                       float *d_loss, void *cuda_stream) {
  if (!d_x || !d_y || !d_params || !d_adam_m || !d_adam_v || !d_work)
    return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (n == 0 || step == 0) return set_err(MVR_ERR_INVALID_ARG, "empty minibatch or step 0");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(mlp_train_step(d_x, d_y, n, d_params, d_adam_m, d_adam_v, d_work, lr, step, d_loss, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return MVR_OK;
}

int mvr_mlp_forward(const float *d_x, uint32_t n, const float *d_params, float *d_work,
                    float *d_out, void *cuda_stream) {
  if (!d_x || !d_params || !d_work || !d_out) return set_err(MVR_ERR_INVALID_ARG, "null argument");
  if (n == 0) return MVR_OK;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  CUDA_TRY(mlp_forward_ref(d_x, n, d_params, d_work, d_out, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return MVR_OK;
}

}  // extern "C"
