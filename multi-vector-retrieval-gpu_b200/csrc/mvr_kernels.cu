// mvr_kernels.cu -- the plain FP32 search kernels of libmvr (sm_100a).
//
// Stage map (reference -> kernel):
//   centroid scoring S = Q.C^T + 1 and per-token top-nprobe
//       (GenerateVQScoreCandidatePP.hpp:118-179: cuBLAS SGEMM, thrust +1,
//        RAFT select_k)                       -> probe_topk_kernel (+ merge)
//   IVF gather, candidate flag/compaction, max-over-probes, sum over tokens,
//   top-probe_topk shortlist (FilterPP.hpp:19-142, 267-398)
//                                             -> filter_kernel
//   VQ/residual gather, decompress, SGEMM, max over doc tokens, sum over
//   query tokens (RerankPP.hpp:16-161, 368-475) -> rerank_kernel
//   host std::sort of the shortlist (IGPGPURetrievalPP.hpp:153-161)
//                                             -> topk_kernel
//
// Every dot product is a sequential __fmaf_rn chain over d = 0..127 from
// 0.0f, every other add is a single rounded FP32 add and every sum runs in a
// fixed order, so results are bit-identical to the CPU oracle's canonical
// arithmetic and independent of launch shape.
#include "mvr_common.cuh"
#include "mvr_kernels.cuh"
#include "mvr_mbar.cuh"

#include <cfloat>

namespace mvr {

// ---------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

constexpr unsigned kFull = 0xffffffffu;

// Insert (s, id) into the sorted per-warp list held one entry per lane
// (lanes < np).  thr is the list's worst entry, uniform across the warp.
__device__ __forceinline__ void warp_list_insert(float &ls, uint32_t &lid,
                                                 float &thr_s, uint32_t &thr_id,
                                                 float ns, uint32_t nid,
                                                 int lane, int np) {
  const bool ahead = lane < np && better(ls, lid, ns, nid);
  const int pos = __popc(__ballot_sync(kFull, ahead));
  const float up_s = __shfl_up_sync(kFull, ls, 1);
  const uint32_t up_id = __shfl_up_sync(kFull, lid, 1);
  if (lane > pos) {
    ls = up_s;
    lid = up_id;
  } else if (lane == pos) {
    ls = ns;
    lid = nid;
  }
  thr_s = __shfl_sync(kFull, ls, np - 1);
  thr_id = __shfl_sync(kFull, lid, np - 1);
}

// ---------------------------------------------------------------------
// K1: S = Q.C^T + 1 over a centroid range, running top-nprobe per token.
// CTA = 64 tokens x (tiles_per_split * 128) centroids, 256 threads.
// Thread (warp w, lane l): tokens w*8..w*8+7, centroids l*4..l*4+3 of the
// current 128-wide tile.  Qs[k][64] and double-buffered Cs[k][128] in smem.
// ---------------------------------------------------------------------
constexpr int kProbeTokTile = 64;
constexpr int kProbeCenTile = 128;
constexpr size_t kProbeSmem =
    (size_t)(kDim * kProbeTokTile + 2 * kDim * kProbeCenTile) * sizeof(float);

__global__ void __launch_bounds__(256, 1)
probe_topk_kernel(const float *__restrict__ q, uint32_t n_tok,
                  const float *__restrict__ ct, uint32_t n_cent,
                  uint32_t n_cent_pad, uint32_t nprobe,
                  uint32_t tiles_per_split, uint32_t *__restrict__ out_id,
                  float *__restrict__ out_s) {
  extern __shared__ __align__(16) float smem[];
  float *Qs = smem;                          // [128][64]
  float *Cs = smem + kDim * kProbeTokTile;   // [2][128][128]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t t0 = blockIdx.y * kProbeTokTile;
  const uint32_t n_tiles = n_cent_pad / kProbeCenTile;
  const uint32_t tile_begin = blockIdx.x * tiles_per_split;
  const uint32_t tile_end = min(n_tiles, tile_begin + tiles_per_split);

  for (int i = tid; i < kProbeTokTile * (kDim / 4); i += 256) {
    const int t = i % kProbeTokTile, k4 = i / kProbeTokTile;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t0 + t < n_tok) v = __ldg(reinterpret_cast<const float4 *>(q + (size_t)(t0 + t) * kDim) + k4);
    Qs[(k4 * 4 + 0) * kProbeTokTile + t] = v.x;
    Qs[(k4 * 4 + 1) * kProbeTokTile + t] = v.y;
    Qs[(k4 * 4 + 2) * kProbeTokTile + t] = v.z;
    Qs[(k4 * 4 + 3) * kProbeTokTile + t] = v.w;
  }

  auto load_tile = [&](uint32_t tile, int buf) {
    float *dst = Cs + buf * kDim * kProbeCenTile;
    const float *src = ct + (size_t)tile * kProbeCenTile;
    // 128 rows x 32 chunks of 16 B
#pragma unroll
    for (int i = 0; i < (kDim * kProbeCenTile / 4) / 256; i++) {
      const int ch = tid + i * 256;
      const int k = ch >> 5, c4 = ch & 31;
      cp_async16(dst + k * kProbeCenTile + c4 * 4, src + (size_t)k * n_cent_pad + c4 * 4);
    }
    cp_async_commit();
  };

  float Ls[8], thr_s[8];
  uint32_t Lid[8], thr_id[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    Ls[i] = -INFINITY; Lid[i] = 0xffffffffu;
    thr_s[i] = -INFINITY; thr_id[i] = 0xffffffffu;
  }
  const int np = (int)nprobe;

  if (tile_begin < tile_end) load_tile(tile_begin, 0);
  for (uint32_t tile = tile_begin; tile < tile_end; tile++) {
    const int buf = (tile - tile_begin) & 1;
    if (tile + 1 < tile_end) {
      load_tile(tile + 1, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();

    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    const float *qs = Qs + warp * 8;
    const float *cs = Cs + buf * kDim * kProbeCenTile + lane * 4;
#pragma unroll 4
    for (int k = 0; k < kDim; k++) {
      const float4 a0 = *reinterpret_cast<const float4 *>(qs + k * kProbeTokTile);
      const float4 a1 = *reinterpret_cast<const float4 *>(qs + k * kProbeTokTile + 4);
      const float4 b = *reinterpret_cast<const float4 *>(cs + k * kProbeCenTile);
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = __fmaf_rn(a[i], bb[j], acc[i][j]);
    }

    const uint32_t c0 = tile * kProbeCenTile + lane * 4;
#pragma unroll
    for (int i = 0; i < 8; i++) {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float s = __fadd_rn(acc[i][j], 1.0f);
        const uint32_t id = c0 + j;
        const bool cand = id < n_cent && better(s, id, thr_s[i], thr_id[i]);
        unsigned m = __ballot_sync(kFull, cand);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const float ns = __shfl_sync(kFull, s, src);
          const uint32_t nid = __shfl_sync(kFull, id, src);
          if (better(ns, nid, thr_s[i], thr_id[i]))
            warp_list_insert(Ls[i], Lid[i], thr_s[i], thr_id[i], ns, nid, lane, np);
        }
      }
    }
    __syncthreads();
  }

  const size_t split_off = (size_t)blockIdx.x * n_tok * nprobe;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t t = t0 + warp * 8 + i;
    if (t < n_tok && lane < np) {
      out_id[split_off + (size_t)t * nprobe + lane] = Lid[i];
      out_s[split_off + (size_t)t * nprobe + lane] = Ls[i];
    }
  }
}

// Merge n_split sorted partial lists per token (one warp per token).
__global__ void __launch_bounds__(256)
probe_merge_kernel(const uint32_t *__restrict__ part_id,
                   const float *__restrict__ part_s, uint32_t n_split,
                   uint32_t n_tok, uint32_t nprobe, uint32_t *__restrict__ out_id,
                   float *__restrict__ out_s) {
  const int lane = threadIdx.x & 31;
  const uint32_t t = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (t >= n_tok) return;
  const int np = (int)nprobe;
  float ls = -INFINITY, thr_s = -INFINITY;
  uint32_t lid = 0xffffffffu, thr_id = 0xffffffffu;
  for (uint32_t sp = 0; sp < n_split; sp++) {
    const size_t base = ((size_t)sp * n_tok + t) * nprobe;
    float ps = -INFINITY;
    uint32_t pid = 0xffffffffu;
    if (lane < np) { ps = part_s[base + lane]; pid = part_id[base + lane]; }
    for (int e = 0; e < np; e++) {
      const float ns = __shfl_sync(kFull, ps, e);
      const uint32_t nid = __shfl_sync(kFull, pid, e);
      if (!better(ns, nid, thr_s, thr_id)) break;  // partial lists are sorted
      warp_list_insert(ls, lid, thr_s, thr_id, ns, nid, lane, np);
    }
  }
  if (lane < np) {
    out_id[(size_t)t * nprobe + lane] = lid;
    out_s[(size_t)t * nprobe + lane] = ls;
  }
}

// ---------------------------------------------------------------------
// K2: candidate filter + shortlist, one CTA per query.
//
// Phase A visits the probed lists rank by rank (all tokens' j-th probe, then
// j+1, ...; probes are sorted best-first) so that the first visit of
// (doc, token) carries the max over probes; the rank j is recorded in a
// per-slot byte table rank[doc][token] (0xff = unvisited).  A doc enters the
// candidate set the first time any token visits it (per-slot epoch stamps,
// no O(n_item) reset).  Phase B sums the per-token maxima exactly (2^-32
// fixed point, rounded once to FP32) and restores the touched rank rows to
// 0xff.  Phase C/D radix-select the top
// probe_topk candidates by the 64-bit key (score desc, id asc).
// ---------------------------------------------------------------------
constexpr int kFilterThreads = 1024;
constexpr int kFilterCluster = 4;  // CTAs (SMs) per query of the rank-table filter

// v * 2^32 rounded to nearest-even, clamped to +-2^62 (exact for |v| >= 2^-9):
// the approximate score is the exact sum of these terms, rounded once to FP32
__device__ __forceinline__ long long to_fixed(float v) {
  double x = (double)v * 4294967296.0;
  x = fmin(fmax(x, -4611686018427387904.0), 4611686018427387904.0);
  return __double2ll_rn(x);
}
__device__ __forceinline__ float from_fixed(long long a) {
  return __ll2float_rn(a) * (1.0f / 4294967296.0f);
}

__device__ __forceinline__ uint32_t find_seg(const uint32_t *pref, int n, uint32_t e) {
  // largest i in [0, n) with pref[i] <= e   (pref[0] = 0, non-decreasing)
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return (uint32_t)lo;
}

// Cluster form: CL CTAs (one cluster) share one query.  Each CTA takes an
// interleaved share of every rank's list entries, of the candidates and of
// the keys; the candidate counter, the shortlist counter and the radix-select
// histograms are combined through distributed shared memory (CTA 0 holds the
// counters), and cluster barriers order the phases.  Splitting a query over
// CL SMs keeps only n_sm / CL queries' rank rows and stamps in flight, a
// working set that stays in L2.  CL = 1 is the single-CTA kernel.
template <int CL>
__device__ __forceinline__ void filter_sync() {
  if constexpr (CL == 1) {
    __syncthreads();
  } else {
    __threadfence();  // rank bytes / stamps / keys live in global memory
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
  }
}

template <int CL>
__device__ __forceinline__ uint32_t *cl_ptr(uint32_t *p, uint32_t rank) {
  if constexpr (CL == 1) {
    return p;
  } else {
    uint32_t *r;
    asm volatile("mapa.u64 %0, %1, %2;\n" : "=l"(r) : "l"(p), "r"(rank));
    return r;
  }
}

constexpr int kSelU = 8;  // candidate keys per thread in flight in the select passes

// Shared-memory state of select_emit.
struct SelectSmem {
  uint32_t (*hist)[256];  // [2][256]
  uint32_t *digit, *need, *done;
};

// Phases C/D of the filter: radix select of the probe_topk largest 64-bit
// keys among key[0, n_cand) (8-bit digits, high to low, stopping once the
// boundary digit is unique), then emission of the selected keys as the
// (unordered) shortlist of query b.  With CL > 1 the CL CTAs of a cluster
// each take an interleaved share of the keys and add their histograms
// through distributed shared memory; g_sel / g_stok are CTA 0's counters.
template <int CL>
__device__ void select_emit(const DevIndex &ix, const uint64_t *__restrict__ key, uint32_t n_cand,
                            uint32_t probe_topk, uint32_t b, uint32_t cr, const SelectSmem &sm,
                            uint32_t *g_sel, uint32_t *g_stok, uint32_t *__restrict__ short_id,
                            float *__restrict__ short_approx) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t cstride = CL * blockDim.x;
  const unsigned lt_mask = (1u << lane) - 1u;
  // ---- phase C: radix select of the probe_topk largest keys ----
  uint64_t prefix = 0, mask = 0;
  if (n_cand > probe_topk) {
    uint32_t need = probe_topk;
    for (int pass = 0; pass < 8; pass++) {
      const int shift = 56 - 8 * pass;
      uint32_t *h = sm.hist[pass & 1];
      for (int i = tid; i < 256; i += blockDim.x) h[i] = 0;
      __syncthreads();
      // kSelU keys per thread in flight
      for (uint32_t i0 = cr * blockDim.x; i0 < n_cand; i0 += kSelU * cstride) {
        uint64_t kv[kSelU];
#pragma unroll
        for (int u = 0; u < kSelU; u++) {
          const uint32_t i = i0 + u * cstride + tid;
          kv[u] = i < n_cand ? key[i] : ~0ull;
        }
#pragma unroll
        for (int u = 0; u < kSelU; u++) {
          const uint32_t i = i0 + u * cstride + tid;
          uint32_t dig = 256;
          if (i < n_cand && (kv[u] & mask) == prefix) dig = (uint32_t)(kv[u] >> shift) & 0xffu;
          const unsigned grp = __match_any_sync(kFull, dig);
          if (dig < 256 && lane == __ffs(grp) - 1) atomicAdd(&h[dig], (uint32_t)__popc(grp));
        }
      }
      filter_sync<CL>();  // every CTA's histogram of this pass complete
      if (warp == 0) {
        // lane l owns bins 255-8l .. 248-8l (high to low), summed over the cluster
        uint32_t cnt[8], sum = 0;
#pragma unroll
        for (int u = 0; u < 8; u++) cnt[u] = 0;
        for (int r = 0; r < CL; r++) {
          const uint32_t *hr = cl_ptr<CL>(h, (uint32_t)r);
#pragma unroll
          for (int u = 0; u < 8; u++) cnt[u] += hr[255 - 8 * lane - u];
        }
#pragma unroll
        for (int u = 0; u < 8; u++) sum += cnt[u];
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += v;
        }
        const uint32_t excl = incl - sum;
        if (excl < need && need <= incl) {
          uint32_t above = excl;
#pragma unroll
          for (int u = 0; u < 8; u++) {
            if (above < need && need <= above + cnt[u]) {
              *sm.digit = 255 - 8 * lane - u;
              *sm.need = need - above;
              *sm.done = (need - above == cnt[u]) ? 1u : 0u;
            }
            above += cnt[u];
          }
        }
      }
      __syncthreads();
      prefix |= (uint64_t)*sm.digit << shift;
      mask |= (uint64_t)0xff << shift;
      need = *sm.need;
      if (*sm.done) break;
    }
  }

  // ---- phase D: emit the shortlist (unordered) ----
  for (uint32_t j0 = cr * blockDim.x; j0 < n_cand; j0 += kSelU * cstride) {
    uint64_t kv[kSelU];
#pragma unroll
    for (int u = 0; u < kSelU; u++) {
      const uint32_t i = j0 + u * cstride + tid;
      kv[u] = i < n_cand ? key[i] : 0ull;
    }
#pragma unroll
    for (int u = 0; u < kSelU; u++) {
      const uint32_t i = j0 + u * cstride + tid;
      const uint64_t k = kv[u];
      const bool sel = i < n_cand && (k & mask) >= prefix;
      const unsigned m = __ballot_sync(kFull, sel);
      if (m) {
        uint32_t base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(g_sel, (uint32_t)__popc(m));
        base = __shfl_sync(kFull, base, __ffs(m) - 1);
        const uint32_t pos = base + __popc(m & lt_mask);
        uint32_t len = 0;
        if (sel && pos < probe_topk) {
          short_id[(size_t)b * probe_topk + pos] = key_id(k);
          short_approx[(size_t)b * probe_topk + pos] = key_score(k);
          len = ix.item_n_vec[key_id(k)];
        }
        const uint32_t tot = __reduce_add_sync(kFull, len);
        if (lane == 0 && tot) atomicAdd(g_stok, tot);
      }
    }
  }
}

template <int CL>
__global__ void __launch_bounds__(kFilterThreads, 1)
filter_kernel(DevIndex ix, const uint32_t *__restrict__ probe_id,
              const float *__restrict__ probe_s, uint32_t nprobe,
              const uint64_t *__restrict__ q_off, uint32_t probe_topk,
              FilterScratch scr, const uint32_t *__restrict__ epoch_base, uint32_t epoch_add,
              uint32_t *__restrict__ short_id, float *__restrict__ short_approx,
              uint32_t *__restrict__ n_short_out, uint32_t *__restrict__ qstat,
              uint32_t *__restrict__ only_if, int impute) {
  __shared__ long long pfix[kMaxQueryTok * kMaxProbe];
  __shared__ long long impf[kMaxQueryTok];  // imputed score of an unmatched token (0: off)
  __shared__ uint32_t pref[kMaxQueryTok + 1];
  __shared__ uint32_t lsz[kMaxQueryTok * kMaxProbe];
  __shared__ uint64_t lof[kMaxQueryTok * kMaxProbe];
  __shared__ uint32_t hist[2][256];
  __shared__ uint32_t s_ncand, s_sel, s_stok;     // CTA 0's copies are the cluster's
  __shared__ uint32_t s_digit, s_need, s_done, s_entries;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n_warp = blockDim.x >> 5;
  uint32_t cr = 0;
  if constexpr (CL > 1) asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(cr));
  const uint32_t b = blockIdx.x / CL;
  // fallback use: only the queries whose hash-table filter overflowed (the
  // flag is the same for every CTA of the cluster, read before any barrier;
  // it stays set until the next batch's hash filter clears it)
  if (only_if && only_if[b] == 0) return;
  // stamp epoch of this launch: a device counter (so that a replayed CUDA
  // graph sees a fresh epoch) plus the caller's offset
  const uint32_t epoch = (epoch_base ? *epoch_base : 0u) + epoch_add;
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);
  uint32_t *stamp = scr.stamp + (size_t)b * scr.n_item;
  uint8_t *rank = scr.rank + (size_t)b * scr.n_item * scr.rank_stride;
  uint64_t *key = scr.key + (size_t)b * scr.n_item;
  uint32_t *g_ncand = cl_ptr<CL>(&s_ncand, 0), *g_sel = cl_ptr<CL>(&s_sel, 0),
           *g_stok = cl_ptr<CL>(&s_stok, 0);
  const unsigned lt_mask = (1u << lane) - 1u;

  // probe scores (fixed point) and list sizes / offsets of every probe
  // (probe id 0xffffffff = no finite score)
  for (uint32_t i = tid; i < nq * nprobe; i += blockDim.x) {
    const uint32_t c = probe_id[tok0 * nprobe + i];
    pfix[i] = to_fixed(probe_s[tok0 * nprobe + i]);
    lsz[i] = c < ix.n_centroid ? ix.ivf_size[c] : 0u;
    lof[i] = c < ix.n_centroid ? ix.ivf_off[c] : 0ull;
  }
  for (uint32_t t = tid; t < nq; t += blockDim.x)
    impf[t] = impute ? to_fixed(probe_s[(tok0 + t) * nprobe + nprobe - 1]) : 0ll;
  if (tid == 0) { s_ncand = 0; s_sel = 0; s_stok = 0; s_entries = 0; }
  filter_sync<CL>();  // counters of CTA 0 initialised before any remote update

  // ---- phase A: scatter probed lists rank by rank ----
  const uint32_t gwarp = cr * n_warp + warp, gstride = CL * n_warp * 128;
  for (uint32_t j = 0; j < nprobe; j++) {
    if (warp == 0) {  // exclusive prefix of the nq list sizes of rank j
      const uint32_t s0 = (uint32_t)lane < nq ? lsz[lane * nprobe + j] : 0u;
      const uint32_t s1 = (uint32_t)lane + 32 < nq ? lsz[(lane + 32) * nprobe + j] : 0u;
      uint32_t i0 = s0, i1 = s1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v0 = __shfl_up_sync(kFull, i0, o), v1 = __shfl_up_sync(kFull, i1, o);
        if (lane >= o) { i0 += v0; i1 += v1; }
      }
      const uint32_t tot0 = __shfl_sync(kFull, i0, 31);
      if ((uint32_t)lane < nq) pref[lane] = i0 - s0;
      if ((uint32_t)lane + 32 < nq) pref[lane + 32] = tot0 + i1 - s1;
      if (lane == 31) {
        const uint32_t total = tot0 + i1;
        pref[nq] = total;
        s_entries += total;
      }
    }
    __syncthreads();
    const uint32_t total = pref[nq];
    // 4 entries per lane in flight: independent list-id and rank-byte loads
    for (uint32_t e0 = gwarp * 128; e0 < total; e0 += gstride) {
      uint32_t item[4], tt[4];
      uint8_t rv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t e = e0 + u * 32 + lane;
        tt[u] = 0xffffffffu;
        if (e < total) {
          const uint32_t t = find_seg(pref, (int)nq, e);
          tt[u] = t;
          item[u] = ix.ivf_ids[lof[t * nprobe + j] + (e - pref[t])];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (tt[u] != 0xffffffffu) rv[u] = rank[(size_t)item[u] * scr.rank_stride + tt[u]];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        bool fresh = false;
        if (tt[u] != 0xffffffffu && rv[u] == 0xff) {
          rank[(size_t)item[u] * scr.rank_stride + tt[u]] = (uint8_t)j;
          fresh = atomicExch(stamp + item[u], epoch) != epoch;
        }
        // warp-aggregated append to the cluster's candidate list
        const unsigned m = __ballot_sync(kFull, fresh);
        if (m) {
          uint32_t base = 0;
          if (lane == __ffs(m) - 1) base = atomicAdd(g_ncand, (uint32_t)__popc(m));
          base = __shfl_sync(kFull, base, __ffs(m) - 1);
          if (fresh) key[base + __popc(m & lt_mask)] = item[u];
        }
      }
    }
    filter_sync<CL>();
  }
  const uint32_t n_cand = *g_ncand;

  // ---- phase B: approximate score, restore rank rows (2 candidates in flight) ----
  const uint32_t cstride = CL * blockDim.x;
  for (uint32_t i0 = cr * blockDim.x + tid; i0 < n_cand; i0 += 2 * cstride) {
    long long ps_acc[2] = {0, 0};
    uint32_t item[2];
    uint8_t *row[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const uint32_t i = i0 + u * cstride;
      item[u] = i < n_cand ? (uint32_t)key[i] : 0u;
      row[u] = rank + (size_t)item[u] * scr.rank_stride;
    }
    for (uint32_t t0 = 0; t0 < nq; t0 += 16) {
      uint4 w[2];
#pragma unroll
      for (int u = 0; u < 2; u++)
        if (i0 + u * cstride < n_cand) w[u] = *reinterpret_cast<uint4 *>(row[u] + t0);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (i0 + u * cstride >= n_cand) continue;
        const uint8_t *bytes = reinterpret_cast<const uint8_t *>(&w[u]);
        long long s = ps_acc[u];
#pragma unroll
        for (int v = 0; v < 16; v++) {
          const uint32_t t = t0 + v;
          if (t < nq) s += bytes[v] != 0xff ? pfix[t * nprobe + bytes[v]] : impf[t];
        }
        ps_acc[u] = s;
        *reinterpret_cast<uint4 *>(row[u] + t0) = make_uint4(~0u, ~0u, ~0u, ~0u);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const uint32_t i = i0 + u * cstride;
      if (i < n_cand) key[i] = make_key(from_fixed(ps_acc[u]), item[u]);
    }
  }
  filter_sync<CL>();

  // ---- phases C/D: radix select + emit ----
  SelectSmem sm{hist, &s_digit, &s_need, &s_done};
  select_emit<CL>(ix, key, n_cand, probe_topk, b, cr, sm, g_sel, g_stok, short_id, short_approx);
  filter_sync<CL>();
  if (cr == 0 && tid == 0) {
    n_short_out[b] = min(s_sel, probe_topk);
    qstat[b * 3 + 0] = n_cand;
    qstat[b * 3 + 1] = s_entries;
    qstat[b * 3 + 2] = s_stok;
  }
}

// ---------------------------------------------------------------------
// Hash-table filter (main search path).  P = hash_parts(...) CTAs
// share a query; CTA p owns the docs [p * n_item / P, (p + 1) * n_item / P) and keeps one
// shared-memory hash-table slot per candidate doc of its range: doc id, the
// mask of query tokens that have visited it and the exact fixed-point sum of
// the first-visit probe scores.  The IVF lists are sorted by doc id, so the
// CTA's part of each probed list is the contiguous sub-list given by the
// index's partition table (ivf_part).  Warp w walks token w's sub-lists in
// probe-rank order (probes are sorted best-first), so the token's first
// visit of a doc carries the max over its probes; different tokens only meet
// in the order-free atomics (OR of the mask, integer add of the score).
// score = sum over tokens of those maxima, the same value the rank-table
// filter computes.  Each candidate's 64-bit (score, id) key goes to the
// query's key array, from which filter_select_kernel takes the shortlist.  A
// CTA whose range holds more than kHashFill candidates marks the query in
// scr.ovf and the rank-table filter redoes that query.
// ---------------------------------------------------------------------
constexpr uint32_t kHashLog = 13, kHashCap = 1u << kHashLog;  // slots per CTA
static_assert(kHashFill + 1024 <= kHashCap, "the fill limit must keep >= 1024 slots empty");
constexpr uint32_t kEmpty = 0xffffffffu;

__host__ __device__ constexpr size_t hash_smem_bytes(int mw) {
  return (size_t)kHashCap * (4 + 4 * mw + 8);
}

template <int MW>
__global__ void __launch_bounds__(kFilterThreads, 1)
filter_hash_kernel(DevIndex ix, const uint32_t *__restrict__ probe_id,
                   const float *__restrict__ probe_s, uint32_t nprobe,
                   const uint64_t *__restrict__ q_off, const uint64_t *__restrict__ cta_off,
                   uint32_t n_query, FilterScratch scr, uint32_t *__restrict__ qstat, int impute) {
  extern __shared__ __align__(16) uint8_t hsm[];
  uint32_t *tkey = reinterpret_cast<uint32_t *>(hsm);                      // [cap]
  uint32_t *tmask = tkey + kHashCap;                                       // [cap][MW]
  unsigned long long *tacc = reinterpret_cast<unsigned long long *>(tmask + kHashCap * MW);
  __shared__ long long pfix[kMaxQueryTok * kMaxProbe];
  __shared__ uint32_t lsz[kMaxQueryTok * kMaxProbe];   // this CTA's sub-list sizes
  __shared__ uint64_t lof[kMaxQueryTok * kMaxProbe];   // and offsets in ivf_ids
  __shared__ long long impf[kMaxQueryTok];  // imputed score of an unmatched token (0: off)
  __shared__ long long s_imp;               // sum of impf over the query's tokens
  __shared__ uint32_t s_fill, s_ovf, s_entries, s_b, s_kbase;
  __shared__ uint32_t s_wsum[32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n_warp = blockDim.x >> 5;
  // this CTA's query and doc range: cta_off[b] <= blockIdx.x < cta_off[b + 1]
  for (uint32_t i = tid; i < n_query; i += blockDim.x)
    if (cta_off[i] <= blockIdx.x && blockIdx.x < cta_off[i + 1]) s_b = i;
  __syncthreads();
  const uint32_t b = s_b;
  const uint32_t part = blockIdx.x - (uint32_t)cta_off[b];
  const uint32_t pstep = (uint32_t)kHashParts / (uint32_t)(cta_off[b + 1] - cta_off[b]);
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);

  for (uint32_t i = tid; i < kHashCap; i += blockDim.x) {
    tkey[i] = kEmpty;
    tacc[i] = 0ull;
#pragma unroll
    for (int w = 0; w < MW; w++) tmask[i * MW + w] = 0u;
  }
  if (tid == 0) { s_fill = 0; s_ovf = 0; s_entries = 0; }
  for (uint32_t t = tid; t < nq; t += blockDim.x)
    impf[t] = impute ? to_fixed(probe_s[(tok0 + t) * nprobe + nprobe - 1]) : 0ll;
  __syncthreads();
  if (tid == 0) {  // fixed order: the same integer in every CTA
    long long a = 0;
    for (uint32_t t = 0; t < nq; t++) a += impf[t];
    s_imp = a;
  }
  uint32_t ent = 0;
  for (uint32_t i = tid; i < nq * nprobe; i += blockDim.x) {
    const uint32_t c = probe_id[tok0 * nprobe + i];
    pfix[i] = to_fixed(probe_s[tok0 * nprobe + i]);
    uint32_t p0 = 0, p1 = 0;
    uint64_t o = 0;
    if (c < ix.n_centroid) {
      const uint32_t *pt = ix.ivf_part + (size_t)c * (kHashParts + 1) + part * pstep;
      p0 = pt[0];
      p1 = pt[pstep];
      o = ix.ivf_off[c];
      ent += ix.ivf_size[c];
    }
    lsz[i] = p1 - p0;
    lof[i] = o + p0;
  }
  if (part == 0) {
    ent = __reduce_add_sync(kFull, ent);
    if (lane == 0 && ent) atomicAdd(&s_entries, ent);
  }
  __syncthreads();

  for (uint32_t t = warp; t < nq; t += n_warp) {
    const uint32_t bit = 1u << (t & 31), word = t >> 5;
    for (uint32_t j = 0; j < nprobe; j++) {
      const uint32_t sz = lsz[t * nprobe + j];
      const uint32_t *ids = ix.ivf_ids + lof[t * nprobe + j];
      // first visit: the probe score replaces the token's imputed score
      const unsigned long long add = (unsigned long long)(pfix[t * nprobe + j] - impf[t]);
      // 4 entries per lane in flight (the loads are independent; the
      // entries of one probe carry the same score, so their order is free)
      for (uint32_t p0 = 0; p0 < sz; p0 += 128) {
        // a CTA past its fill limit stops: its query is redone by the
        // rank-table filter
        if (__any_sync(kFull, *reinterpret_cast<volatile uint32_t *>(&s_ovf) != 0u)) break;
        uint32_t its[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const uint32_t p = p0 + lane + 32u * u;
          its[u] = p < sz ? __ldg(ids + p) : kEmpty;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const uint32_t it = its[u];
          // find or insert `it` (linear probing; the walk is bounded by the
          // table size, and a CTA stops inserting once its fill count passes
          // the limit)
          uint32_t slot = kEmpty;
          bool inserted = false;
          if (it != kEmpty) {
            uint32_t h = (it * 2654435769u) >> (32 - kHashLog);
            for (uint32_t step = 0; step < kHashCap; step++) {
              const uint32_t k = *reinterpret_cast<volatile uint32_t *>(&tkey[h]);
              if (k == it) { slot = h; break; }
              if (k == kEmpty) {
                const uint32_t old = atomicCAS(&tkey[h], kEmpty, it);
                if (old == kEmpty) { slot = h; inserted = true; break; }
                if (old == it) { slot = h; break; }
              }
              h = (h + 1) & (kHashCap - 1);
            }
            if (slot == kEmpty) s_ovf = 1;  // the table is full
          }
          // the fill count (distinct docs inserted): one shared atomic per
          // warp and round instead of one per insert on a single address
          const unsigned ins = __ballot_sync(kFull, inserted);
          if (lane == 0 && ins) {
            const uint32_t n = (uint32_t)__popc(ins);
            if (atomicAdd(&s_fill, n) + n > kHashFill) s_ovf = 1;
          }
          if (slot == kEmpty) continue;
          const uint32_t old = atomicOr(&tmask[slot * MW + word], bit);
          if (!(old & bit)) atomicAdd(&tacc[slot], add);
        }
      }
      __syncwarp();  // rank j of token t before rank j + 1
    }
  }
  __syncthreads();

  // emit this CTA's candidates as (score, id) keys (at most kHashFill per CTA:
  // an overflowed CTA emits none, its query is redone by the rank-table
  // filter).  One global atomic per CTA reserves the CTA's key range: each
  // thread counts its slots (tid, tid + blockDim, ...), a block scan gives
  // its offset, and it writes its keys there.
  uint64_t *key = scr.hkey + (size_t)b * scr.key_stride;
  if (!s_ovf) {
    uint32_t mine = 0;
    for (uint32_t sl = tid; sl < kHashCap; sl += blockDim.x) mine += tkey[sl] != kEmpty ? 1u : 0u;
    uint32_t inc = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < n_warp ? s_wsum[lane] : 0u, wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, wi, o);
        if (lane >= o) wi += v;
      }
      if (lane < n_warp) s_wsum[lane] = wi - w;  // exclusive warp offsets
      if (lane == 31) s_kbase = wi ? atomicAdd(scr.qcnt + b, wi) : 0u;
    }
    __syncthreads();
    uint32_t pos = s_kbase + s_wsum[warp] + inc - mine;
    for (uint32_t sl = tid; sl < kHashCap; sl += blockDim.x) {
      const uint32_t k = tkey[sl];
      if (k != kEmpty) key[pos++] = make_key(from_fixed((long long)tacc[sl] + s_imp), k);
    }
  }
  if (tid == 0) {
    if (s_ovf) atomicOr(scr.ovf + b, 1u);
    if (part == 0) qstat[b * 3 + 1] = s_entries;
  }
}

__global__ void advance_epoch_kernel(uint32_t *epoch, uint32_t n) { *epoch += n; }

// ivf_part[c][p] = first position of list c whose doc id is >= p * n_item / P
// (p = 0..P): the doc-range sub-lists of the hash filter.
__global__ void ivf_part_kernel(const uint64_t *__restrict__ ivf_off,
                                const uint32_t *__restrict__ ivf_size,
                                const uint32_t *__restrict__ ivf_ids, uint32_t n_cent,
                                uint32_t n_item, uint32_t *__restrict__ out) {
  const size_t n = (size_t)n_cent * (kHashParts + 1);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c = (uint32_t)(i / (kHashParts + 1)), p = (uint32_t)(i % (kHashParts + 1));
    const uint32_t bound = (uint32_t)((uint64_t)p * n_item / kHashParts);
    const uint32_t *l = ivf_ids + ivf_off[c];
    uint32_t lo = 0, hi = ivf_size[c];
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (l[mid] < bound) lo = mid + 1; else hi = mid;
    }
    out[i] = lo;
  }
}

cudaError_t make_ivf_part(const DevIndex &ix, uint32_t *out, cudaStream_t st) {
  ivf_part_kernel<<<592, 256, 0, st>>>(ix.ivf_off, ix.ivf_size, ix.ivf_ids, ix.n_centroid,
                                       ix.n_item, out);
  return cudaGetLastError();
}

// Shortlist of every query from the keys filter_hash_kernel emitted; resets
// the query's key counter for the next batch.
__global__ void __launch_bounds__(kFilterThreads, 1)
filter_select_kernel(DevIndex ix, uint32_t probe_topk, FilterScratch scr,
                     uint32_t *__restrict__ short_id, float *__restrict__ short_approx,
                     uint32_t *__restrict__ n_short_out, uint32_t *__restrict__ qstat) {
  __shared__ uint32_t hist[2][256];
  __shared__ uint32_t s_sel, s_stok, s_digit, s_need, s_done;
  const uint32_t b = blockIdx.x;
  const uint32_t n_cand = scr.qcnt[b];
  if (threadIdx.x == 0) { s_sel = 0; s_stok = 0; }
  __syncthreads();
  SelectSmem sm{hist, &s_digit, &s_need, &s_done};
  select_emit<1>(ix, scr.hkey + (size_t)b * scr.key_stride, n_cand, probe_topk, b, 0, sm, &s_sel,
                 &s_stok, short_id, short_approx);
  __syncthreads();
  if (threadIdx.x == 0) {
    n_short_out[b] = min(s_sel, probe_topk);
    qstat[b * 3 + 0] = n_cand;
    qstat[b * 3 + 2] = s_stok;
    scr.qcnt[b] = 0;
  }
}

// ---------------------------------------------------------------------
// K3: decompress + exact MaxSim of up to kRkDocs shortlisted docs of one query.
//
// The docs' tokens, each doc padded to a multiple of 4 tokens, form a stream
// of 256-token tiles; a tile is consumed in 8 chunks of 16 dimensions.  Two
// CTAs of 256 threads per SM:
//  warps 4-7   decoders (one warpgroup): per chunk, each thread decodes 2
//              tokens (positions p and p + 128 of the tile) x 16 dims,
//              x = centroid + W[bucket] (one rounded FP32 add; W from a table
//              replicated across the 32 banks, read conflict-free), into
//              stage i % kRkStages of a shared-memory ring [16 dims][256];
//              the loads of chunk i + 1 are in flight while chunk i is
//              decoded, and the next tile's tokens are located a tile ahead;
//  warps 0-3   FMA (one warpgroup): thread (warp w, lane l) owns query tokens
//              16(w&1)..+16 of the pass and doc tokens 128(w>>1) + 4l..+4 of
//              the tile, so per dimension it reads 16 query values (4
//              broadcast LDS.128) and 4 doc values (one LDS.128) for 64 FMAs.
//              After the 8th chunk of a tile: max over the thread's valid
//              tokens (all of one doc, thanks to the padding), then per doc a
//              __reduce_max_sync over the lanes holding it, folded into
//              best[query token][doc] by atomicMax.
// Registers: the launch gives every thread 128; setmaxnreg lowers the FMA
// warpgroup to 120 and raises the decoders to 136.
// Queries of more than 32 tokens run in two passes (tokens 0-31, 32-63).
// Ring handoff: mbarriers full[s] (the 128 decoder threads arrive) and
// empty[s] (the 128 FMA threads arrive); every wait is bounded (wait_ns) and
// a timeout sets bit 32 of *err and stops the CTA without writing scores.
// Every dot product is the sequential __fmaf_rn chain over d = 0..127 from
// 0.0f, so the scores are bit-identical to the canonical arithmetic.
// ---------------------------------------------------------------------
constexpr int kRkDocs = 64;       // shortlisted docs per CTA
constexpr int kRkTile = 256;      // doc tokens per tile
constexpr int kRkChunk = 16;      // dimensions per ring stage
constexpr int kRkStages = 4;      // ring stages
constexpr int kRkQ = 32;          // query tokens per pass
constexpr int kRkThreads = 256;   // 4 FMA warps + 4 decoder warps (two CTAs per SM)
constexpr int kRkFma = 128;       // FMA threads
// registers per thread after the split (setmaxnreg): the launch gives every
// thread 128 (65,536 / 512 for the SM's two CTAs); the FMA warpgroup gives 8
// each back and the decoder warpgroup takes them, 128 x 120 + 128 x 136 =
// 256 x 128
constexpr int kRkRegLaunch = 128;
constexpr int kRkRegFma = 120;
constexpr int kRkRegDec = 136;
static_assert(kRkFma * kRkRegFma + (kRkThreads - kRkFma) * kRkRegDec == kRkThreads * kRkRegLaunch,
              "register split must equal the launch allocation");

// CTA-local barrier of the FMA warps only (named barrier 1, kRkFma threads)
__device__ __forceinline__ void fma_bar_sync() {
  asm volatile("bar.sync 1, %0;\n" ::"n"(kRkFma) : "memory");
}

__host__ __device__ constexpr size_t rk_smem_bytes(int n_bit) {
  return (size_t)kRkStages * kRkChunk * kRkTile * sizeof(float) +  // ring
         (size_t)kDim * kRkQ * sizeof(float) +                      // query tokens of the pass
         (size_t)(1 << n_bit) * 32 * sizeof(float) +                // replicated weights
         (size_t)kMaxQueryTok * kRkDocs * sizeof(int);              // best[q][doc]
}

template <int NBIT>
__global__ void __launch_bounds__(kRkThreads, 2)
rerank_kernel(DevIndex ix, const float *__restrict__ q, const uint64_t *__restrict__ q_off,
              const uint32_t *__restrict__ short_id, const uint32_t *__restrict__ n_short,
              uint32_t probe_topk, int semantics, float *__restrict__ exact,
              unsigned *__restrict__ err, uint64_t wait_ns) {
  constexpr int VPB = 8 / NBIT;             // values per residual byte
  constexpr int CB = kRkChunk * NBIT / 8;   // residual bytes per token and chunk
  constexpr int RW = (CB + 3) / 4;          // ... in 32-bit words
  constexpr uint32_t MASK = (1u << NBIT) - 1u;
  constexpr int NCH = kDim / kRkChunk;      // chunks per tile
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;                                       // [S][16][512]
  float *Qs = ring + kRkStages * kRkChunk * kRkTile;        // [128 dims][32 query tokens]
  float *wrep = Qs + kDim * kRkQ;                           // [2^NBIT][32]
  int *best = reinterpret_cast<int *>(wrep + (1 << NBIT) * 32);  // [64 query tokens][kRkDocs]
  __shared__ uint32_t d_len[kRkDocs], d_pp[kRkDocs + 1];
  __shared__ uint64_t d_off[kRkDocs];
  __shared__ uint64_t full[kRkStages], empty[kRkStages];
  __shared__ volatile int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t b = blockIdx.y;
  const uint32_t ns = n_short[b];
  const uint32_t d0 = blockIdx.x * kRkDocs;
  if (d0 >= ns) return;
  const uint32_t nd = min((uint32_t)kRkDocs, ns - d0);
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);

  if (tid < (int)nd) {
    const uint32_t it = short_id[(size_t)b * probe_topk + d0 + tid];
    d_len[tid] = ix.item_n_vec[it];
    d_off[tid] = ix.item_off[it];
  }
  if (tid == 0) {
    for (int s = 0; s < kRkStages; s++) {
      mbar_init(&full[s], kRkThreads - kRkFma);
      mbar_init(&empty[s], kRkFma);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
  }
  for (int i = tid; i < (1 << NBIT) * 32; i += kRkThreads) {
    // bucket v sits in the top NBIT bits of byte v << (8 - NBIT), position 0
    const uint32_t v = (uint32_t)i >> 5;
    wrep[i] = ix.lut[((v << (8 - NBIT)) & 0xffu) * VPB];
  }
  for (int i = tid; i < kMaxQueryTok * kRkDocs; i += kRkThreads) best[i] = f2si(-INFINITY);
  __syncthreads();
  if (warp == 0) {  // padded token offsets of the docs (warp scan)
    uint32_t carry = 0;
    if (lane == 0) d_pp[0] = 0;
    for (uint32_t base = 0; base < nd; base += 32) {
      uint32_t v = base + lane < nd ? (d_len[base + lane] + 3u) & ~3u : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
      }
      if (base + lane < nd) d_pp[base + lane + 1] = carry + v;
      carry += __shfl_sync(kFull, v, 31);
    }
  }
  __syncthreads();
  const uint32_t Tp = d_pp[nd];
  const uint32_t n_tiles = (Tp + kRkTile - 1) / kRkTile;
  const uint32_t n_pass = (nq + kRkQ - 1) / kRkQ;
  const uint32_t total = n_tiles * NCH;  // ring chunks per pass

  if (warp >= kRkFma / 32) {
    // ---------------- decoders (kRkRegDec registers) ----------------
    // thread pt decodes tile positions pt and pt + 256 of every chunk; the
    // loads of chunk i + 1 are in flight while chunk i is decoded, and the
    // tokens (codes, residual rows) of tile t + 1 are located during tile t
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kRkRegDec));
    const uint32_t pt = (uint32_t)(tid - kRkFma);
    uint32_t code[2], code_n[2];
    uint64_t vix[2], vix_n[2];
    // tile tl's tokens of this thread; past a doc's last token (padding) or
    // past the last doc: some valid token, whose values the FMA warps mask
    auto locate = [&](uint32_t tl, uint32_t (&cd)[2], uint64_t (&vx)[2]) {
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const uint32_t g = kRkTile * tl + (kRkTile / 2) * j + pt;
        uint64_t v = d_off[0];
        if (g < Tp) {
          const uint32_t d = find_seg(d_pp, (int)nd, g);
          v = d_off[d] + min(g - d_pp[d], d_len[d] - 1u);
        }
        vx[j] = v;
        cd[j] = __ldg(ix.vq_code + v);
      }
    };
    auto issue = [&](const uint32_t (&cd)[2], const uint64_t (&vx)[2], uint32_t c,
                     float4 (&cv)[2][4], uint32_t (&rw)[2][RW]) {
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const float4 *cp = reinterpret_cast<const float4 *>(ix.centroid + (size_t)cd[j] * kDim) + 4 * c;
#pragma unroll
        for (int u = 0; u < 4; u++) cv[j][u] = __ldg(cp + u);
        const uint8_t *rp = ix.residual + vx[j] * ix.bytes_per_vec + (size_t)c * CB;
        if constexpr (CB == 2) {
          rw[j][0] = __ldg(reinterpret_cast<const unsigned short *>(rp));
        } else if constexpr (CB == 4) {
          rw[j][0] = __ldg(reinterpret_cast<const uint32_t *>(rp));
        } else if constexpr (CB == 8) {
          const uint2 t = __ldg(reinterpret_cast<const uint2 *>(rp));
          rw[j][0] = t.x;
          rw[j][1] = t.y;
        } else {
          const uint4 t = __ldg(reinterpret_cast<const uint4 *>(rp));
          rw[j][0] = t.x;
          rw[j][1] = t.y;
          rw[j][2] = t.z;
          rw[j][3] = t.w;
        }
      }
    };
    bool ok = true;
    uint32_t base = 0;  // ring chunk counter at the start of the pass
    // decode chunk q of the pass (values in cv / rw) into its ring stage
    auto put = [&](uint32_t q, const float4 (&cv)[2][4], const uint32_t (&rw)[2][RW]) {
      const uint32_t gq = base + q;
      const uint32_t s = gq % kRkStages;
      if (gq >= (uint32_t)kRkStages &&
          !__all_sync(kFull, mbar_wait_sleep(&empty[s], ((gq / kRkStages) + 1) & 1, wait_ns))) {
        ok = false;
        return;
      }
      float *xs = ring + s * (kRkChunk * kRkTile) + pt;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const float cc[16] = {cv[j][0].x, cv[j][0].y, cv[j][0].z, cv[j][0].w,
                              cv[j][1].x, cv[j][1].y, cv[j][1].z, cv[j][1].w,
                              cv[j][2].x, cv[j][2].y, cv[j][2].z, cv[j][2].w,
                              cv[j][3].x, cv[j][3].y, cv[j][3].z, cv[j][3].w};
#pragma unroll
        for (int kk = 0; kk < kRkChunk; kk++) {
          // dim 16c + kk: byte kk / VPB of the chunk, most significant bits first
          const int gbit = 8 * (kk / VPB) + 8 - NBIT * (kk % VPB + 1);
          const uint32_t v = (rw[j][gbit >> 5] >> (gbit & 31)) & MASK;
          xs[kk * kRkTile + (kRkTile / 2) * j] = __fadd_rn(cc[kk], wrep[v * 32 + lane]);
        }
      }
      mbar_arrive(&full[s]);
      if (__any_sync(kFull, s_abort != 0)) ok = false;
    };
    // the loads of chunk q + 1 (the next tile's first chunk after chunk 7)
    auto prefetch = [&](uint32_t q, float4 (&cv)[2][4], uint32_t (&rw)[2][RW]) {
      if (q + 1 >= total) return;
      if ((q + 1) % NCH != 0) issue(code, vix, (q + 1) % NCH, cv, rw);
      else issue(code_n, vix_n, 0, cv, rw);
    };
    float4 cva[2][4], cvb[2][4];
    uint32_t rwa[2][RW], rwb[2][RW];
    for (uint32_t pass = 0; ok && pass < n_pass; pass++, base += total) {
      locate(0, code, vix);
      issue(code, vix, 0, cva, rwa);
      if (n_tiles > 1) locate(1, code_n, vix_n);
      for (uint32_t q = 0; ok && q < total; q += 2) {
        // even chunk q: values in a; a tile starts at every multiple of 8
        if (q % NCH == 0 && q > 0) {
          const uint32_t tl = q / NCH;
#pragma unroll
          for (int j = 0; j < 2; j++) {
            code[j] = code_n[j];
            vix[j] = vix_n[j];
          }
          if (tl + 1 < n_tiles) locate(tl + 1, code_n, vix_n);
        }
        prefetch(q, cvb, rwb);
        put(q, cva, rwa);
        if (!ok || q + 1 >= total) break;
        // odd chunk q + 1: values in b
        prefetch(q + 1, cva, rwa);
        put(q + 1, cvb, rwb);
      }
    }
    if (!ok && lane == 0) {
      atomicOr(err, 32u);
      s_abort = 1;
    }
  } else {
    // ---------------- FMA warps (kRkRegFma registers) ----------------
    // Every FMA warp executes the same sequence of named barriers (two per
    // pass and one at the end): a warp's own failure only skips its work.
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kRkRegFma));
    const uint32_t qg = (uint32_t)warp & 1u;
    const uint32_t tb = 128u * ((uint32_t)warp >> 1) + 4u * lane;
    uint32_t it = 0;  // ring chunk counter (continues across tiles and passes)
    bool ok = true;
    for (uint32_t pass = 0; pass < n_pass; pass++) {
      // query tokens 32 pass .. +32 -> Qs[dim][token] (zero past the last token)
      for (int i = tid; i < kDim / 4 * kRkQ; i += kRkFma) {
        const int j = i % kRkQ, k4 = i / kRkQ;
        const uint32_t t = kRkQ * pass + j;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (t < nq) v = __ldg(reinterpret_cast<const float4 *>(q + (tok0 + t) * kDim) + k4);
        Qs[(4 * k4 + 0) * kRkQ + j] = v.x;
        Qs[(4 * k4 + 1) * kRkQ + j] = v.y;
        Qs[(4 * k4 + 2) * kRkQ + j] = v.z;
        Qs[(4 * k4 + 3) * kRkQ + j] = v.w;
      }
      fma_bar_sync();
      for (uint32_t tl = 0; ok && tl < n_tiles; tl++) {
        const uint32_t g0 = kRkTile * tl + tb;
        int doc = -1;
        uint32_t nval = 0;
        if (g0 < Tp) {
          doc = (int)find_seg(d_pp, (int)nd, g0);
          nval = min(4u, d_len[doc] - (g0 - d_pp[doc]));
        }
        float acc[16][4];
#pragma unroll
        for (int i = 0; i < 16; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
        for (int c = 0; c < NCH; c++, it++) {
          const uint32_t s = it % kRkStages;
          if (!__all_sync(kFull, mbar_wait_sleep(&full[s], (it / kRkStages) & 1, wait_ns)) ||
              __any_sync(kFull, s_abort != 0)) {
            ok = false;
            break;
          }
          const float *xs = ring + s * (kRkChunk * kRkTile) + tb;
          const float *qs = Qs + (kRkChunk * c) * kRkQ + 16 * qg;
#pragma unroll
          for (int kk = 0; kk < kRkChunk; kk++) {
            const float4 x = *reinterpret_cast<const float4 *>(xs + kk * kRkTile);
            float a[16];
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const float4 t = *reinterpret_cast<const float4 *>(qs + kk * kRkQ + 4 * u);
              a[4 * u] = t.x;
              a[4 * u + 1] = t.y;
              a[4 * u + 2] = t.z;
              a[4 * u + 3] = t.w;
            }
#pragma unroll
            for (int i = 0; i < 16; i++) {
              acc[i][0] = __fmaf_rn(a[i], x.x, acc[i][0]);
              acc[i][1] = __fmaf_rn(a[i], x.y, acc[i][1]);
              acc[i][2] = __fmaf_rn(a[i], x.z, acc[i][2]);
              acc[i][3] = __fmaf_rn(a[i], x.w, acc[i][3]);
            }
          }
          mbar_arrive(&empty[s]);
        }
        if (!ok) {
          if (lane == 0) {
            atomicOr(err, 32u);
            s_abort = 1;
          }
          break;
        }
        // max over the thread's valid tokens (one doc), then over the lanes of that doc
        const unsigned grp = __match_any_sync(kFull, doc);
        const bool lead = lane == __ffs(grp) - 1;
#pragma unroll
        for (int i = 0; i < 16; i++) {
          int m = f2si(-INFINITY);
#pragma unroll
          for (int j = 0; j < 4; j++)
            if ((uint32_t)j < nval) m = max(m, f2si(acc[i][j]));
          m = __reduce_max_sync(grp, m);
          const uint32_t qt = kRkQ * pass + 16u * qg + i;
          if (doc >= 0 && lead && qt < nq) atomicMax(&best[qt * kRkDocs + doc], m);
        }
      }
      fma_bar_sync();  // Qs is reloaded by the next pass; best is complete after the last
    }
    if (tid < (int)nd && !s_abort) {  // FMA threads 0 .. nd - 1
      const bool clamp = semantics == 1 && d_len[tid] < ix.max_item_n_vec;
      float s = 0.0f;
      for (uint32_t t = 0; t < nq; t++) {
        float m = si2f(best[t * kRkDocs + tid]);
        if (clamp) m = fmaxf(m, 0.0f);
        s = __fadd_rn(s, m);
      }
      exact[(size_t)b * probe_topk + d0 + tid] = s;
    }
  }
}

// ---------------------------------------------------------------------
// K4: final top-k of the reranked shortlist (bitonic sort of 64-bit keys).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(512)
topk_kernel(const uint32_t *__restrict__ short_id, const float *__restrict__ exact,
            const uint32_t *__restrict__ n_short, uint32_t probe_topk,
            uint32_t n_pad, uint32_t topk, float *__restrict__ out_s,
            uint32_t *__restrict__ out_id, uint32_t *__restrict__ n_out) {
  extern __shared__ uint64_t keys[];
  const uint32_t b = blockIdx.x;
  const uint32_t n = n_short[b];
  if (n_out && threadIdx.x == 0) n_out[b] = min(n, topk);
  for (uint32_t i = threadIdx.x; i < n_pad; i += blockDim.x)
    keys[i] = i < n ? make_key(exact[(size_t)b * probe_topk + i], short_id[(size_t)b * probe_topk + i]) : 0ull;
  __syncthreads();
  for (uint32_t k = 2; k <= n_pad; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < n_pad; i += blockDim.x) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint64_t a = keys[i], c = keys[l];
          const bool desc = (i & k) == 0;
          if (desc ? (a < c) : (a > c)) { keys[i] = c; keys[l] = a; }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < topk; i += blockDim.x) {
    if (i < n) {
      out_s[(size_t)b * topk + i] = key_score(keys[i]);
      out_id[(size_t)b * topk + i] = key_id(keys[i]);
    } else {
      out_s[(size_t)b * topk + i] = -INFINITY;
      out_id[(size_t)b * topk + i] = 0xffffffffu;
    }
  }
}

// ---------------------------------------------------------------------
// K4 for k well below the list length: the same sorted top-k by a radix
// select of the k-th largest key in shared memory (8-bit digits, high to
// low, stopping once the boundary digit is unique), a compaction of the k
// keys at or above it (the keys are unique: exactly k), and a bitonic sort
// of those k only.  Same output as topk_kernel.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(512)
topk_select_kernel(const uint32_t *__restrict__ short_id, const float *__restrict__ exact,
                   const uint32_t *__restrict__ n_short, uint32_t probe_topk, uint32_t k_pad,
                   uint32_t topk, float *__restrict__ out_s, uint32_t *__restrict__ out_id,
                   uint32_t *__restrict__ n_out) {
  extern __shared__ uint64_t keys[];  // [probe_topk] keys, then [k_pad] selected
  uint64_t *sel = keys + probe_topk;
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_digit, s_need, s_done, s_cnt;
  const uint32_t b = blockIdx.x;
  const uint32_t n = min(n_short[b], probe_topk);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (n_out && tid == 0) n_out[b] = min(n, topk);
  for (uint32_t i = tid; i < n; i += blockDim.x)
    keys[i] = make_key(exact[(size_t)b * probe_topk + i], short_id[(size_t)b * probe_topk + i]);
  for (uint32_t i = tid; i < k_pad; i += blockDim.x) sel[i] = 0ull;
  if (tid == 0) s_cnt = 0;
  uint64_t prefix = 0, mask = 0;
  if (n > topk) {
    uint32_t need = topk;
    for (int pass = 0; pass < 8; pass++) {
      const int shift = 56 - 8 * pass;
      for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
      __syncthreads();
      for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
        const uint32_t i = i0 + tid;
        uint32_t dig = 256;
        if (i < n && (keys[i] & mask) == prefix) dig = (uint32_t)(keys[i] >> shift) & 0xffu;
        const unsigned grp = __match_any_sync(kFull, dig);
        if (dig < 256 && lane == __ffs(grp) - 1) atomicAdd(&hist[dig], (uint32_t)__popc(grp));
      }
      __syncthreads();
      if (warp == 0) {  // lane l owns bins 255-8l .. 248-8l (high to low)
        uint32_t cnt[8], sum = 0;
#pragma unroll
        for (int u = 0; u < 8; u++) {
          cnt[u] = hist[255 - 8 * lane - u];
          sum += cnt[u];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += v;
        }
        const uint32_t excl = incl - sum;
        if (excl < need && need <= incl) {
          uint32_t above = excl;
#pragma unroll
          for (int u = 0; u < 8; u++) {
            if (above < need && need <= above + cnt[u]) {
              s_digit = 255 - 8 * lane - u;
              s_need = need - above;
              s_done = (need - above == cnt[u]) ? 1u : 0u;
            }
            above += cnt[u];
          }
        }
      }
      __syncthreads();
      prefix |= (uint64_t)s_digit << shift;
      mask |= (uint64_t)0xff << shift;
      need = s_need;
      if (s_done) break;
    }
  }
  __syncthreads();
  // the top keys (all n when n <= topk), unordered, then sorted descending
  for (uint32_t i = tid; i < n; i += blockDim.x)
    if ((keys[i] & mask) >= prefix) sel[atomicAdd(&s_cnt, 1u)] = keys[i];
  __syncthreads();
  for (uint32_t kk = 2; kk <= k_pad; kk <<= 1) {
    for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
      for (uint32_t i = tid; i < k_pad; i += blockDim.x) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint64_t a = sel[i], c = sel[l];
          const bool desc = (i & kk) == 0;
          if (desc ? (a < c) : (a > c)) { sel[i] = c; sel[l] = a; }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = tid; i < topk; i += blockDim.x) {
    if (i < n) {
      out_s[(size_t)b * topk + i] = key_score(sel[i]);
      out_id[(size_t)b * topk + i] = key_id(sel[i]);
    } else {
      out_s[(size_t)b * topk + i] = -INFINITY;
      out_id[(size_t)b * topk + i] = 0xffffffffu;
    }
  }
}

// ---------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------
// The register split of rerank_kernel (setmaxnreg) hands the FMA warps' and
// decoders' shares out of the allocation the CTA was launched with; it is
// only valid when that allocation is kRkRegLaunch per thread (a smaller one
// would leave setmaxnreg.inc waiting), so the library refuses to run a build
// that compiled to another count.
template <typename K>
static cudaError_t check_rk_registers(K kernel) {
  cudaFuncAttributes a;
  const cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e != cudaSuccess) return e;
  return a.numRegs == kRkRegLaunch ? cudaSuccess : cudaErrorInvalidKernelImage;
}

cudaError_t configure_kernels() {
  cudaError_t e = cudaFuncSetAttribute(probe_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kProbeSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk_smem_bytes(1));
  if (e != cudaSuccess) return e;
  e = check_rk_registers(rerank_kernel<1>);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk_smem_bytes(2));
  if (e != cudaSuccess) return e;
  e = check_rk_registers(rerank_kernel<2>);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk_smem_bytes(4));
  if (e != cudaSuccess) return e;
  e = check_rk_registers(rerank_kernel<4>);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk_smem_bytes(8));
  if (e != cudaSuccess) return e;
  e = check_rk_registers(rerank_kernel<8>);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(filter_hash_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)hash_smem_bytes(1));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(filter_hash_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)hash_smem_bytes(2));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(topk_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)((kMaxShort + kMaxShort / 4) * sizeof(uint64_t)));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(kMaxShort * sizeof(uint64_t)));
}

int probe_splits(uint32_t n_tok, uint32_t n_cent_pad, int n_sm) {
  const uint32_t tok_tiles = (n_tok + kProbeTokTile - 1) / kProbeTokTile;
  const uint32_t cen_tiles = n_cent_pad / kProbeCenTile;
  uint32_t want = (uint32_t)(2 * n_sm + tok_tiles - 1) / tok_tiles;  // ~2 waves
  if (want < 1) want = 1;
  if (want > cen_tiles) want = cen_tiles;
  return (int)want;
}

cudaError_t launch_probe(const DevIndex &ix, const float *q, uint32_t n_tok,
                         uint32_t nprobe, int n_split, uint32_t *part_id,
                         float *part_s, uint32_t *out_id, float *out_s,
                         cudaStream_t st, int *n_launch) {
  const uint32_t cen_tiles = ix.n_centroid_pad / kProbeCenTile;
  const uint32_t per = (cen_tiles + n_split - 1) / n_split;
  const uint32_t splits = (cen_tiles + per - 1) / per;
  dim3 grid(splits, (n_tok + kProbeTokTile - 1) / kProbeTokTile);
  if (splits == 1) {
    probe_topk_kernel<<<grid, 256, kProbeSmem, st>>>(q, n_tok, ix.centroid_t, ix.n_centroid,
                                                    ix.n_centroid_pad, nprobe, per, out_id, out_s);
    *n_launch += 1;
    return cudaGetLastError();
  }
  probe_topk_kernel<<<grid, 256, kProbeSmem, st>>>(q, n_tok, ix.centroid_t, ix.n_centroid,
                                                  ix.n_centroid_pad, nprobe, per, part_id, part_s);
  probe_merge_kernel<<<(n_tok + 7) / 8, 256, 0, st>>>(part_id, part_s, splits, n_tok, nprobe,
                                                      out_id, out_s);
  *n_launch += 2;
  return cudaGetLastError();
}

cudaError_t launch_filter(const DevIndex &ix, const uint32_t *probe_id,
                          const float *probe_s, uint32_t nprobe,
                          const uint64_t *q_off, uint32_t n_query,
                          uint32_t probe_topk, const FilterScratch &scr,
                          uint32_t epoch, uint32_t *short_id,
                          float *short_approx, uint32_t *n_short,
                          uint32_t *qstat, cudaStream_t st, int *n_launch) {
  filter_kernel<1><<<n_query, kFilterThreads, 0, st>>>(ix, probe_id, probe_s, nprobe, q_off,
                                                       probe_topk, scr, nullptr, epoch, short_id,
                                                       short_approx, n_short, qstat, nullptr, 0);
  *n_launch += 1;
  return cudaGetLastError();
}

cudaError_t launch_filter_cluster(const DevIndex &ix, const uint32_t *probe_id,
                                  const float *probe_s, uint32_t nprobe,
                                  const uint64_t *q_off, uint32_t n_query,
                                  uint32_t probe_topk, const FilterScratch &scr,
                                  const uint32_t *epoch_base, uint32_t epoch_add,
                                  uint32_t *short_id, float *short_approx, uint32_t *n_short,
                                  uint32_t *qstat, cudaStream_t st, int *n_launch,
                                  uint32_t *only_if, int impute) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n_query * kFilterCluster, 1, 1);
  cfg.blockDim = dim3(kFilterThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kFilterCluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, filter_kernel<kFilterCluster>, ix, probe_id, probe_s,
                                     nprobe, q_off, probe_topk, scr, epoch_base, epoch_add,
                                     short_id, short_approx, n_short, qstat, only_if, impute);
  *n_launch += 1;
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_filter_hash(const DevIndex &ix, const uint32_t *probe_id,
                               const float *probe_s, uint32_t nprobe,
                               const uint64_t *q_off, const uint64_t *cta_off, uint32_t n_cta,
                               uint32_t n_query, uint32_t fb_slots,
                               uint32_t probe_topk, const FilterScratch &scr,
                               uint32_t *epoch, uint32_t *short_id,
                               float *short_approx, uint32_t *n_short,
                               uint32_t *qstat, cudaStream_t st, int *n_launch, int impute) {
  cudaError_t e = cudaMemsetAsync(scr.ovf, 0, (size_t)n_query * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  if (scr.rank_stride <= 32)
    filter_hash_kernel<1><<<n_cta, kFilterThreads, hash_smem_bytes(1), st>>>(
        ix, probe_id, probe_s, nprobe, q_off, cta_off, n_query, scr, qstat, impute);
  else
    filter_hash_kernel<2><<<n_cta, kFilterThreads, hash_smem_bytes(2), st>>>(
        ix, probe_id, probe_s, nprobe, q_off, cta_off, n_query, scr, qstat, impute);
  filter_select_kernel<<<n_query, kFilterThreads, 0, st>>>(ix, probe_topk, scr, short_id,
                                                          short_approx, n_short, qstat);
  *n_launch += 2;
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // queries whose candidates overflowed a hash table: rank-table filter, in
  // chunks of fb_slots queries over its fb_slots scratch slots; chunk c uses
  // stamp epoch *epoch + 1 + c, then the counter advances by the chunk count
  uint32_t c = 0;
  for (uint32_t q0 = 0; q0 < n_query; q0 += fb_slots, c++) {
    const uint32_t cnt = n_query - q0 < fb_slots ? n_query - q0 : fb_slots;
    e = launch_filter_cluster(ix, probe_id, probe_s, nprobe, q_off + q0, cnt, probe_topk, scr,
                              epoch, 1u + c, short_id + (size_t)q0 * probe_topk,
                              short_approx + (size_t)q0 * probe_topk, n_short + q0,
                              qstat + (size_t)q0 * 3, st, n_launch, scr.ovf + q0, impute);
    if (e != cudaSuccess) return e;
  }
  advance_epoch_kernel<<<1, 1, 0, st>>>(epoch, c);
  *n_launch += 1;
  return cudaGetLastError();
}

cudaError_t launch_rerank(const DevIndex &ix, const float *q, const uint64_t *q_off,
                          uint32_t n_query, const uint32_t *short_id,
                          const uint32_t *n_short, uint32_t probe_topk,
                          int semantics, float *exact, unsigned *err, cudaStream_t st,
                          int *n_launch, uint64_t wait_ns) {
  if (n_query == 0 || probe_topk == 0) return cudaSuccess;
  dim3 grid((probe_topk + kRkDocs - 1) / kRkDocs, n_query);
  const size_t sm = rk_smem_bytes((int)ix.n_bit);
#define MVR_RK(NB)                                                                              \
  rerank_kernel<NB><<<grid, kRkThreads, sm, st>>>(ix, q, q_off, short_id, n_short, probe_topk, \
                                                  semantics, exact, err, wait_ns)
  switch (ix.n_bit) {
    case 1: MVR_RK(1); break;
    case 2: MVR_RK(2); break;
    case 4: MVR_RK(4); break;
    case 8: MVR_RK(8); break;
    default: return cudaErrorInvalidValue;
  }
#undef MVR_RK
  *n_launch += 1;
  return cudaGetLastError();
}

cudaError_t launch_topk(const uint32_t *short_id, const float *exact,
                        const uint32_t *n_short, uint32_t n_query,
                        uint32_t probe_topk, uint32_t topk, float *out_s,
                        uint32_t *out_id, uint32_t *n_out, cudaStream_t st, int *n_launch) {
  uint32_t n_pad = 1;
  while (n_pad < probe_topk) n_pad <<= 1;
  uint32_t k_pad = 1;
  while (k_pad < topk) k_pad <<= 1;
  if (probe_topk >= 512 && 4 * topk <= probe_topk) {
    // select, then sort only the k best
    topk_select_kernel<<<n_query, 512, (probe_topk + k_pad) * sizeof(uint64_t), st>>>(
        short_id, exact, n_short, probe_topk, k_pad, topk, out_s, out_id, n_out);
  } else {
    topk_kernel<<<n_query, 512, n_pad * sizeof(uint64_t), st>>>(short_id, exact, n_short,
                                                              probe_topk, n_pad, topk, out_s,
                                                              out_id, n_out);
  }
  *n_launch += 1;
  return cudaGetLastError();
}

}  // namespace mvr
