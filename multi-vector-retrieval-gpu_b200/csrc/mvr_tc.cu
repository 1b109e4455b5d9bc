// mvr_tc.cu -- tensor-core (tcgen05, sm_100a) MaxSim for the mixed-precision
// search path.
//
// rerank_tc_kernel scores a query's shortlisted docs with BF16 operands and
// FP32 accumulation in TMEM: per 128-token tile the CTA decompresses doc tokens
// x = centroid + W[bucket] (BF16 centroid table + BF16 decode table, one BF16
// add) straight into a 128B-swizzled K-major shared-memory tile (operand A,
// M = 128 doc tokens), the query tokens sit in a second swizzled tile (operand
// B, N = 32 or 64), one elected thread issues 8 tcgen05.mma (K = 16 each) into
// a TMEM accumulator, and the epilogue reads D[token][query-token] back with
// tcgen05.ld and folds it into per-(query token, doc) maxima.  Two TMEM
// accumulators and two A tiles let the epilogue of tile i-1 overlap the MMA of
// tile i.  Scores are approximate (BF16 inputs); the search path re-scores the
// best of them with the exact FP32 kernel.
#include "mvr_common.cuh"
#include "mvr_tc.cuh"
#include "mvr_mbar.cuh"

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstring>

namespace mvr {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTcTile = 128;      // doc tokens per MMA tile (M)
constexpr int kTcDocs = 32;       // shortlisted docs per CTA
constexpr int kTcThreads = 256;

// K-major SWIZZLE_128B UMMA shared-memory descriptor: 8-row x 128 B atoms,
// SBO = 1024 B between 8-row groups, LBO unused (1), version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: BF16 A/B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// byte offset of element (row, k) in a [rows][64] BF16 K-block, 128B swizzle
__device__ __forceinline__ uint32_t sw128_off(uint32_t row, uint32_t chunk16) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk16 ^ (row & 7u)) << 4);
}


__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completing on the mbarrier's transaction count
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}


}  // namespace

// Decompress 8 dims (one 16-byte chunk of a BF16 row): centroid chunk +
// per-byte decode-table rows (VPB BF16 weights per residual byte).
template <int NBIT>
__device__ __forceinline__ uint4 decode_chunk(uint4 cen, const uint8_t *rb,
                                              const __nv_bfloat16 *lut, const uint32_t *nib,
                                              int lane) {
  constexpr int VPB = 8 / NBIT;
  uint32_t w[4];
  if constexpr (NBIT == 2) {         // 2 bytes = 4 nibbles -> 4 x (2 weights)
    // nib[(nibble * 32 + lane)]: bf16x2 of the nibble's two codes, one copy
    // per lane so that the 32 lanes read 32 different banks
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t byte = rb[u >> 1];
      const uint32_t nb = (u & 1) ? (byte & 0xfu) : (byte >> 4);
      w[u] = nib[nb * 32 + lane];
    }
  } else if constexpr (NBIT == 1) {  // 1 byte = 2 nibbles -> 2 x (4 weights)
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const uint32_t nb = u ? (rb[0] & 0xfu) : (rb[0] >> 4);
      const uint2 t = reinterpret_cast<const uint2 *>(nib)[nb * 32 + lane];
      w[2 * u] = t.x;
      w[2 * u + 1] = t.y;
    }
  } else if constexpr (VPB == 8) {   // (unused) 1 byte -> 8 weights
    const uint4 t = *reinterpret_cast<const uint4 *>(lut + rb[0] * 8);
    w[0] = t.x; w[1] = t.y; w[2] = t.z; w[3] = t.w;
  } else if constexpr (VPB == 4) {   // 2 bytes -> 2 x 4 weights
    const uint2 t0 = *reinterpret_cast<const uint2 *>(lut + rb[0] * 4);
    const uint2 t1 = *reinterpret_cast<const uint2 *>(lut + rb[1] * 4);
    w[0] = t0.x; w[1] = t0.y; w[2] = t1.x; w[3] = t1.y;
  } else if constexpr (VPB == 2) {   // 4 bytes -> 4 x 2 weights
#pragma unroll
    for (int u = 0; u < 4; u++) w[u] = *reinterpret_cast<const uint32_t *>(lut + rb[u] * 2);
  } else {                           // 8 bytes -> 8 x 1 weight
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t lo = *reinterpret_cast<const uint16_t *>(lut + rb[2 * u]);
      const uint32_t hi = *reinterpret_cast<const uint16_t *>(lut + rb[2 * u + 1]);
      w[u] = lo | (hi << 16);
    }
  }
  uint32_t c[4] = {cen.x, cen.y, cen.z, cen.w};
#pragma unroll
  for (int u = 0; u < 4; u++) {
    __nv_bfloat162 r = __hadd2(*reinterpret_cast<__nv_bfloat162 *>(&c[u]),
                               *reinterpret_cast<__nv_bfloat162 *>(&w[u]));
    c[u] = *reinterpret_cast<uint32_t *>(&r);
  }
  return make_uint4(c[0], c[1], c[2], c[3]);
}

// Dynamic shared memory of rerank_tc_kernel for a query-token tile of N rows.
__host__ __device__ constexpr size_t tc_smem_bytes(int nbit, uint32_t n) {
  return 1024 + 32768 /*A*/ + (size_t)n * 256 /*B*/ + 64 * kTcDocs * 4 /*best*/ +
         (nbit <= 2 ? 16 * 32 * 4 * (nbit == 1 ? 2 : 1) : 256 * (8 / nbit) * 2) /*decode table*/;
}

template <int NBIT>
__global__ void __launch_bounds__(kTcThreads, 4)
rerank_tc_kernel(DevIndex ix, const __nv_bfloat16 *__restrict__ cen_bf16,
                 const __nv_bfloat16 *__restrict__ lut_bf16, const float *__restrict__ q,
                 const uint64_t *__restrict__ q_off, const uint32_t *__restrict__ short_id,
                 const uint32_t *__restrict__ n_short, uint32_t probe_topk, int semantics,
                 uint32_t n_max, float *__restrict__ approx, unsigned *__restrict__ err) {
  constexpr int VPB = 8 / NBIT;
  constexpr int HALF_BYTES = 64 / VPB;  // residual bytes of 64 dims
  constexpr int NRW = HALF_BYTES / 8;   // uint2 words per half row
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *Ad = smem;                                          // [2 K-blocks][128 rows][128 B]
  uint8_t *Bq = smem + 32768;                                  // [2 K-blocks][n_max rows][128 B]
  int *best = reinterpret_cast<int *>(Bq + n_max * 256);       // [64][kTcDocs]
  uint32_t *nib = reinterpret_cast<uint32_t *>(best + 64 * kTcDocs);  // b<=2: [16][32](x2)
  __nv_bfloat16 *lut = reinterpret_cast<__nv_bfloat16 *>(nib);        // b>=4: [256][VPB]
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ uint32_t d_len[kTcDocs], d_pref[kTcDocs + 1];
  __shared__ uint64_t d_off[kTcDocs];
  __shared__ int tok_doc[2][kTcTile];
  __shared__ int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t b = blockIdx.y;
  const uint32_t ns = n_short[b];
  const uint32_t d0 = blockIdx.x * kTcDocs;
  if (d0 >= ns) return;  // uniform: before any TMEM / barrier use
  const uint32_t nd = min((uint32_t)kTcDocs, ns - d0);
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);
  const uint32_t N = nq <= 32 ? 32u : 64u;  // <= n_max (host sizes smem by the batch)
  const uint32_t idesc = idesc_bf16(kTcTile, (int)N);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(64u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
  }
  if (tid < (int)nd) {
    const uint32_t it = short_id[(size_t)b * probe_topk + d0 + tid];
    d_len[tid] = ix.item_n_vec[it];
    d_off[tid] = ix.item_off[it];
  }
  if constexpr (NBIT <= 2) {
    // nibble n is the top nibble of byte (n << 4): its codes' weights are the
    // first 4 / NBIT entries of that byte's decode-table row; one copy per
    // lane so the 32 lanes of a warp read 32 different banks
    for (int i = tid; i < 16 * 32; i += kTcThreads) {
      const int n = i >> 5, ln = i & 31;
      const uint16_t *row = reinterpret_cast<const uint16_t *>(lut_bf16) + (n << 4) * VPB;
      if constexpr (NBIT == 2) {
        nib[n * 32 + ln] = (uint32_t)row[0] | ((uint32_t)row[1] << 16);
      } else {
        reinterpret_cast<uint2 *>(nib)[n * 32 + ln] =
            make_uint2((uint32_t)row[0] | ((uint32_t)row[1] << 16), (uint32_t)row[2] | ((uint32_t)row[3] << 16));
      }
    }
  } else {
    for (int i = tid; i < 256 * VPB; i += kTcThreads) lut[i] = lut_bf16[i];
  }
  for (int i = tid; i < 64 * kTcDocs; i += kTcThreads) best[i] = f2si(-INFINITY);
  // query tokens -> B operand (BF16, swizzled, rows >= nq zero)
  for (int i = tid; i < (int)N * 16; i += kTcThreads) {
    const int row = i >> 4, ch = i & 15;  // 16 chunks of 8 dims
    uint4 v = make_uint4(0, 0, 0, 0);
    if ((uint32_t)row < nq) {
      const float4 *src = reinterpret_cast<const float4 *>(q + (tok0 + row) * kDim + ch * 8);
      const float4 a = __ldg(src), c = __ldg(src + 1);
      __nv_bfloat162 p0 = __floats2bfloat162_rn(a.x, a.y), p1 = __floats2bfloat162_rn(a.z, a.w);
      __nv_bfloat162 p2 = __floats2bfloat162_rn(c.x, c.y), p3 = __floats2bfloat162_rn(c.z, c.w);
      v.x = *reinterpret_cast<uint32_t *>(&p0);
      v.y = *reinterpret_cast<uint32_t *>(&p1);
      v.z = *reinterpret_cast<uint32_t *>(&p2);
      v.w = *reinterpret_cast<uint32_t *>(&p3);
    }
    *reinterpret_cast<uint4 *>(Bq + (ch >> 3) * (N * 128) + sw128_off(row, ch & 7)) = v;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t acc = 0;
    for (uint32_t i = 0; i < nd; i++) { d_pref[i] = acc; acc += d_len[i]; }
    d_pref[nd] = acc;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t n_tok = d_pref[nd];
  const uint32_t n_tiles = (n_tok + kTcTile - 1) / kTcTile;
  const uint32_t a_base = smem_u32(Ad), b_base = smem_u32(Bq);
  const uint32_t row = tid & (kTcTile - 1), half = tid >> 7;
  uint8_t *kb = Ad + half * 16384;

  // next tile's row data (doc, centroid id, residual bytes); the doc index
  // only moves forward as the tiles advance
  uint32_t di = 0;
  int p_doc = -1;
  uint32_t p_code = 0;
  uint2 p_res[NRW];
  auto prefetch = [&](uint32_t tile) {
    const uint32_t s = tile * kTcTile + row;
    p_doc = -1;
    if (tile < n_tiles && s < n_tok) {
      while (d_pref[di + 1] <= s) di++;
      const uint64_t v = d_off[di] + (s - d_pref[di]);
      p_doc = (int)di;
      p_code = __ldg(ix.vq_code + v);
      const uint2 *res = reinterpret_cast<const uint2 *>(ix.residual + v * ix.bytes_per_vec + half * HALF_BYTES);
#pragma unroll
      for (int u = 0; u < NRW; u++) p_res[u] = __ldg(res + u);
    }
  };

  auto epilogue = [&](uint32_t tile) {
    const bool ok = __all_sync(kFull, mbar_wait(&bar, tile & 1));
    if (!ok) {  // warp-uniform: record, skip, stop after the next barrier
      if (lane == 0) { atomicOr(err, 1u); s_abort = 1; }
      return;
    }
    tc_fence_after();
    const uint32_t r = 32 * (warp & 3) + lane;
    const int doc = tok_doc[tile & 1][r];
    const unsigned grp = __match_any_sync(kFull, doc);
    const bool leader = lane == __ffs(grp) - 1;
    for (uint32_t c0 = half * (N / 2); c0 < half * (N / 2) + N / 2; c0 += 16) {
      uint32_t v[16];
      tmem_ld16(tmem + ((32u * (warp & 3)) << 16) + c0, v);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int m = __reduce_max_sync(grp, f2si(__uint_as_float(v[j])));
        if (leader && doc >= 0 && c0 + j < nq) atomicMax(&best[(c0 + j) * kTcDocs + doc], m);
      }
    }
    tc_fence_before();
  };

  prefetch(0);
  for (uint32_t tile = 0; tile < n_tiles; tile++) {
    if (tile > 0) epilogue(tile - 1);  // MMA(tile-1) done: A reusable, D readable
    const int doc = p_doc;
    const uint32_t code = p_code;
    uint8_t rb[HALF_BYTES];
#pragma unroll
    for (int u = 0; u < NRW; u++) *reinterpret_cast<uint2 *>(rb + 8 * u) = p_res[u];
    if (half == 0) tok_doc[tile & 1][row] = doc;
    prefetch(tile + 1);
    if (doc >= 0) {
      const uint4 *cen = reinterpret_cast<const uint4 *>(cen_bf16 + (size_t)code * kDim + half * 64);
#pragma unroll
      for (int c = 0; c < 8; c++)
        *reinterpret_cast<uint4 *>(kb + sw128_off(row, c)) =
            decode_chunk<NBIT>(__ldg(cen + c), rb + c * (8 / VPB), lut, nib, lane);
    } else {
#pragma unroll
      for (int c = 0; c < 8; c++) *reinterpret_cast<uint4 *>(kb + sw128_off(row, c)) = make_uint4(0, 0, 0, 0);
    }
    fence_async_smem();
    __syncthreads();
    if (s_abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < 8; kk++) {
        const uint64_t ad = sw128_desc(a_base + (kk >> 2) * 16384 + (kk & 3) * 32);
        const uint64_t bd = sw128_desc(b_base + (kk >> 2) * (N * 128) + (kk & 3) * 32);
        mma_bf16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
      }
      mma_commit(&bar);
    }
  }
  if (!s_abort && n_tiles > 0) epilogue(n_tiles - 1);
  __syncthreads();

  if (tid < (int)nd && !s_abort) {
    const bool clamp = semantics == 1 && d_len[tid] < ix.max_item_n_vec;
    float s = 0.0f;
    for (uint32_t t = 0; t < nq; t++) {
      float m = si2f(best[t * kTcDocs + tid]);
      if (clamp) m = fmaxf(m, 0.0f);
      s += m;
    }
    approx[(size_t)b * probe_topk + d0 + tid] = s;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(64u));
  }
}

// ---------------------------------------------------------------------
// rerank_tmem_kernel: BF16 MaxSim for 1- and 2-bit residual codes with the
// doc-token operand in tensor memory.
//
// Per 128-token tile every thread decodes one half row (64 dims) in
// registers and writes it to TMEM with tcgen05.st; tcgen05.mma then reads A
// (M = 128 doc tokens, K = 128) from TMEM and B (the query tokens, N = 32 or
// 64) from a swizzled shared-memory tile, so the decoded tile never passes
// through shared memory.  Decode of one 32-bit residual word (4*VPB dims)
// needs no table lookups: the codes j of the four bytes are isolated with one
// shift and mask, turned into PRMT byte selectors with one IMAD
// (k -> k | (k+4) << 4 per byte), and two PRMTs pick the low / high bytes of
// the BF16 bucket weights held in two registers, giving bf16x2 words that a
// HADD2 adds to the centroid's.  That fixes the order of K inside each word's
// block of 4*VPB dims: position 4j + 2h + e holds dim VPB*(2h + e) + j.  The
// centroid rows (cen_perm) and the query tile are stored in the same order,
// so the contraction is unchanged.  Two A stages and three D stages in TMEM:
// iteration i issues tile i's loads, runs the epilogue of tile i-2 (its MMA
// was issued a whole iteration earlier, so the completion wait is short;
// tcgen05.ld, per-doc max with warp REDUX, shared-memory atomicMax), decodes
// tile i into A[i%2] and issues its MMA into D[i%3].  Every D stage starts
// at OFF, a power of two above |q.x| for every pair of the CTA (Cauchy-
// Schwarz with the query norms and the index's bound on |x|), so D holds
// positive floats whose bit patterns order like integers: the epilogue takes
// full-warp REDUX.MAX of the raw bits per doc group and re-arms the stage
// with OFF after reading it.
// ---------------------------------------------------------------------
constexpr int kTmTile = 128;
constexpr int kTmDocs = 64;       // shortlisted docs per CTA
constexpr int kTmThreads = 256;   // warp w: TMEM lane quadrant w & 3, half row w >> 2
// TMEM columns: A[2] x 64 + D[3] x N  (N = 32: 224 -> 256, 2 CTAs per SM;
// N = 64: 320 -> 512, one CTA per SM, enforced through the smem size)
__host__ __device__ constexpr uint32_t tm_cols(uint32_t n_max) { return n_max <= 32 ? 256u : 512u; }

template <int NBIT>
__host__ __device__ constexpr uint32_t tm_dim_of(uint32_t kappa) {
  constexpr uint32_t VPB = 8 / NBIT, WD = 4 * VPB;
  const uint32_t m = kappa / WD, r = kappa % WD;
  return m * WD + VPB * (r % 4) + r / 4;
}

__host__ __device__ constexpr size_t tm_smem_bytes(uint32_t n_max) {
  return n_max <= 32 ? 1024 + (size_t)n_max * 256 : 120 * 1024;  // dynamic part: B tile
}

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;\n" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

__device__ __forceinline__ uint32_t hadd2_u32(uint32_t a, uint32_t b) {
  __nv_bfloat162 r = __hadd2(*reinterpret_cast<__nv_bfloat162 *>(&a),
                             *reinterpret_cast<__nv_bfloat162 *>(&b));
  return *reinterpret_cast<uint32_t *>(&r);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}

// the same word into 16 consecutive TMEM columns of the warp's 32 lanes
__device__ __forceinline__ void tmem_fill16(uint32_t taddr, uint32_t x) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
      "%1,%1};\n" ::"r"(taddr), "r"(x)
      : "memory");
}

__device__ __forceinline__ void mma_bf16_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t b,
                                            uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}

// 16 output columns (bf16x2) of one half row from WPS residual words
// (WPS = 16 / (2 * VPB): 2 words for 2-bit, 1 for 1-bit) and 4 uint4 of the
// permuted centroid row.
template <int NBIT>
__device__ __forceinline__ void tm_decode16(const uint32_t *res, const uint4 *cen, uint32_t wlo,
                                            uint32_t whi, uint32_t (&out)[16]) {
  constexpr int VPB = 8 / NBIT;
  constexpr uint32_t MASK = NBIT == 2 ? 0x03030303u : 0x01010101u;
  constexpr int WPS = 16 / (2 * VPB);
#pragma unroll
  for (int wi = 0; wi < WPS; wi++) {
    const uint32_t w = res[wi];
#pragma unroll
    for (int j = 0; j < VPB; j++) {
      const uint32_t x = (w >> (8 - NBIT * (j + 1))) & MASK;
      const uint32_t t = x * 0x11u + 0x40404040u;
      out[wi * 2 * VPB + 2 * j] = prmt(wlo, whi, t);
      out[wi * 2 * VPB + 2 * j + 1] = prmt(wlo, whi, t >> 16);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
    out[4 * c + 0] = hadd2_u32(cen[c].x, out[4 * c + 0]);
    out[4 * c + 1] = hadd2_u32(cen[c].y, out[4 * c + 1]);
    out[4 * c + 2] = hadd2_u32(cen[c].z, out[4 * c + 2]);
    out[4 * c + 3] = hadd2_u32(cen[c].w, out[4 * c + 3]);
  }
}

// FP8 (e4m3) variant for 2-bit codes.  The 16 dims of one residual word
// expand with one PRMT per 4 dims: y1 = w & 0x33333333 puts the codes of dims
// 4i+3 and 4i+1 of byte i in nibbles 2i and 2i+1, y0 = (w >> 2) & 0x33333333
// those of dims 4i+2 and 4i; each nibble, used as a PRMT selector on the four
// FP8 bucket weights, yields the dim's weight.  K position 4p + e of the
// word's block (output word p = PRMT of y1, y1 >> 16, y0, y0 >> 16) holds
// dim kFp8Dim[4p + e].  The centroid part and the residual part are two A
// operands in TMEM accumulated into the same D (c + W[b] is never formed), so
// the centroid row goes from its loads to TMEM unchanged.  Query tokens are
// quantized with per-token power-of-two scales (their largest entry maps into
// [112, 224]), removed from the per-doc maxima at the end.
//
// 4-bit codes: the residual word's nibbles are PRMT selectors themselves
// (selector nibble e of a word holds the code of dim e ^ 1, the high nibble of
// each byte being its first dim), but 16 weights do not fit PRMT's 8-byte
// table.  Three PRMTs per 4 dims cover them: the magnitudes |W[0..7]| with
// the codes as selectors, |W[8..15]| with the codes ^ 8; a selector >= 8
// makes PRMT return the sign of the addressed byte replicated, 0x00 for a
// magnitude, so OR-ing the two picks the right one.  A third table holds the
// signs: byte j has bit 6 = sign of W[j], bit 7 = sign of W[8 + j], so with
// the codes as selectors bit 6 of the result is the sign of W[code] in both
// halves; shifted to bit 7 it completes the E4M3 byte.  K position kappa of
// an 8-dim word block holds dim kappa ^ 1.
template <int NBIT>
__host__ __device__ constexpr uint32_t fp8_dim_of(uint32_t kappa) {
  constexpr uint8_t kFp8Dim[16] = {3, 1, 7, 5, 11, 9, 15, 13, 2, 0, 6, 4, 10, 8, 14, 12};
  return NBIT == 4 ? kappa ^ 1u : (kappa & ~15u) + kFp8Dim[kappa & 15u];
}

// kind::f8f6f4 instruction descriptor: E4M3 A/B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_e4m3(int m, int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_e4m3_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t b,
                                            uint32_t idesc) {
  asm volatile("tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], [%1], %2, %3, 1;\n" ::"r"(tmem_d),
               "r"(tmem_a), "l"(b), "r"(idesc)
               : "memory");
}

// 16 A_r columns (4 FP8 weights each) of one 64-dim half row from its 4
// residual words; wtab: the 4 FP8 bucket weights in bytes 0..3.
__device__ __forceinline__ void fp8_decode16(const uint32_t *res, uint32_t wtab,
                                             uint32_t (&out)[16]) {
#pragma unroll
  for (int wi = 0; wi < 4; wi++) {
    const uint32_t y1 = res[wi] & 0x33333333u, y0 = (res[wi] >> 2) & 0x33333333u;
    out[4 * wi + 0] = prmt(wtab, 0u, y1);
    out[4 * wi + 1] = prmt(wtab, 0u, y1 >> 16);
    out[4 * wi + 2] = prmt(wtab, 0u, y0);
    out[4 * wi + 3] = prmt(wtab, 0u, y0 >> 16);
  }
}

// 4 E4M3 weights of the 4 codes in the low 16 bits of s (x = s ^ 0x8888)
__device__ __forceinline__ uint32_t fp8_pick4(uint32_t s, uint32_t x, const TmWeights &t) {
  const uint32_t a = prmt(t.w[0], t.w[1], s);  // |W[c]| for c < 8, else 0
  const uint32_t b = prmt(t.w[2], t.w[3], x);  // |W[c]| for c >= 8, else 0
  const uint32_t g = prmt(t.w[4], t.w[5], s);  // bit 6 of each byte: sign of W[c]
  return a | b | ((g << 1) & 0x80808080u);
}

// 16 A_r columns of one 64-dim half row from its 8 residual words (4-bit)
__device__ __forceinline__ void fp8_decode16_b4(const uint32_t *res, const TmWeights &t,
                                                uint32_t (&out)[16]) {
#pragma unroll
  for (int wi = 0; wi < 8; wi++) {
    const uint32_t s = res[wi], x = s ^ 0x88888888u;
    out[2 * wi] = fp8_pick4(s, x, t);
    out[2 * wi + 1] = fp8_pick4(s >> 16, x >> 16, t);
  }
}

template <int NBIT, bool FP8>
__global__ void __launch_bounds__(kTmThreads, 2)
rerank_tmem_kernel(DevIndex ix, const uint32_t *__restrict__ cen_perm, TmWeights tw,
                   const float *__restrict__ q, const uint64_t *__restrict__ q_off,
                   const uint32_t *__restrict__ short_id, const uint32_t *__restrict__ n_short,
                   uint32_t probe_topk, int semantics, uint32_t n_max, float x_bound,
                   float *__restrict__ approx, unsigned *__restrict__ err) {
  static_assert(FP8 ? (NBIT == 2 || NBIT == 4) : (NBIT == 1 || NBIT == 2),
                "BF16 decodes 1- and 2-bit codes, FP8 2- and 4-bit codes");
  constexpr int VPB = 8 / NBIT;
  constexpr int HW = 64 / (4 * VPB);  // residual words of a 64-dim half row (8, 4 or 2)
  constexpr int CW = FP8 ? 16 : 32;   // centroid words (TMEM columns) of a half row
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *Bq = smem;  // BF16: [2 K-blocks][n_max rows][128 B]; FP8: [n_max rows][128 B]
  __shared__ uint32_t best[kTmDocs * kMaxQueryTok];        // [doc][query token], bits of OFF + max
  __shared__ uint32_t s_qss;                               // max squared (scaled) token norm
  __shared__ float s_qinv[kMaxQueryTok];                   // FP8: 1 / query-token scale
  __shared__ __align__(16) uint32_t stage[kTmThreads / 32][16];  // per-warp epilogue staging
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_base_s;
  __shared__ uint32_t d_len[kTmDocs], d_pref[kTmDocs + 1];
  __shared__ uint64_t d_off[kTmDocs];
  __shared__ int tok_doc[3][kTmTile];
  __shared__ int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t b = blockIdx.y;
  const uint32_t ns = n_short[b];
  const uint32_t d0 = blockIdx.x * kTmDocs;
  if (d0 >= ns) return;  // uniform: before any TMEM / barrier use
  const uint32_t nd = min((uint32_t)kTmDocs, ns - d0);
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);
  const uint32_t N = nq <= 32 ? 32u : 64u;  // <= n_max (host sizes smem by the batch)
  const uint32_t idesc = FP8 ? idesc_e4m3(kTmTile, (int)N) : idesc_bf16(kTmTile, (int)N);
  const uint32_t n_cols = tm_cols(n_max);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(n_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
    s_qss = 0;
  }
  if (tid < (int)nd) {
    const uint32_t it = short_id[(size_t)b * probe_topk + d0 + tid];
    d_len[tid] = ix.item_n_vec[it];
    d_off[tid] = ix.item_off[it];
  }
  for (int i = tid; i < kMaxQueryTok * kTmDocs; i += kTmThreads) best[i] = 0u;
  __syncthreads();  // s_qss
  if constexpr (FP8) {
    // query tokens -> B operand (E4M3, scaled per token, permuted K order,
    // swizzled, rows >= nq zero); 8 lanes per row, 16 positions each
    for (int i = tid; i < (int)N * 8; i += kTmThreads) {  // N * 8 is a multiple of 256
      const int row = i >> 3, ch = i & 7;
      float x[16];
      float amax = 0.0f, ss = 0.0f;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        x[u] = (uint32_t)row < nq ? __ldg(q + (tok0 + row) * kDim + fp8_dim_of<NBIT>(16 * ch + u)) : 0.0f;
        amax = fmaxf(amax, fabsf(x[u]));
        ss = fmaf(x[u], x[u], ss);
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        amax = fmaxf(amax, __shfl_xor_sync(kFull, amax, o));
        ss += __shfl_xor_sync(kFull, ss, o);
      }
      // power-of-two scale: largest entry into [112, 224] (1 for an all-zero row)
      const float sc = amax > 0.0f ? exp2f(floorf(log2f(224.0f / amax))) : 1.0f;
      uint32_t v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const __nv_fp8x2_storage_t lo = __nv_cvt_float2_to_fp8x2(
            make_float2(x[4 * u] * sc, x[4 * u + 1] * sc), __NV_SATFINITE, __NV_E4M3);
        const __nv_fp8x2_storage_t hi = __nv_cvt_float2_to_fp8x2(
            make_float2(x[4 * u + 2] * sc, x[4 * u + 3] * sc), __NV_SATFINITE, __NV_E4M3);
        v[u] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
      *reinterpret_cast<uint4 *>(Bq + sw128_off(row, ch)) = make_uint4(v[0], v[1], v[2], v[3]);
      if ((lane & 7) == 0) {
        atomicMax(&s_qss, __float_as_uint(ss * sc * sc));
        if (row < kMaxQueryTok) s_qinv[row] = 1.0f / sc;
      }
    }
  } else
  // query tokens -> B operand (BF16, permuted K order, swizzled, rows >= nq
  // zero); the 16 lanes of a row also sum its squares (fixed shuffle order)
  for (int i = tid; i < (int)N * 16; i += kTmThreads) {  // N * 16 is a multiple of 256
    const int row = i >> 4, ch = i & 15;  // 16 chunks of 8 positions
    uint32_t v[4] = {0, 0, 0, 0};
    float ss = 0.0f;
    if ((uint32_t)row < nq) {
      const float *src = q + (tok0 + row) * kDim;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const float lo = __ldg(src + tm_dim_of<NBIT>(8 * ch + 2 * u));
        const float hi = __ldg(src + tm_dim_of<NBIT>(8 * ch + 2 * u + 1));
        ss = fmaf(lo, lo, fmaf(hi, hi, ss));
        __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
        v[u] = *reinterpret_cast<uint32_t *>(&p);
      }
    }
    *reinterpret_cast<uint4 *>(Bq + (ch >> 3) * (N * 128) + sw128_off(row, ch & 7)) =
        make_uint4(v[0], v[1], v[2], v[3]);
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) ss += __shfl_xor_sync(kFull, ss, o);
    if ((lane & 15) == 0) atomicMax(&s_qss, __float_as_uint(ss));
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t acc = 0;
    for (uint32_t i = 0; i < nd; i++) { d_pref[i] = acc; acc += d_len[i]; }
    d_pref[nd] = acc;
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t n_tok = d_pref[nd];
  // OFF: smallest power of two >= 1 above max |q| * |x| (margin for BF16 /
  // FP8 rounding; FP8: scaled query tokens)
  const float off = fmaxf(1.0f, exp2f(ceilf(log2f(sqrtf(__uint_as_float(s_qss)) * x_bound *
                                                  (FP8 ? 1.15f : 1.02f) + 1e-30f))));
  const uint32_t off_bits = __float_as_uint(off);
  const uint32_t n_tiles = (n_tok + kTmTile - 1) / kTmTile;
  const uint32_t b_base = smem_u32(Bq);
  const uint32_t qd = warp & 3, hf = warp >> 2;
  const uint32_t row = 32 * qd + lane;
  const uint32_t lane_off = (32u * qd) << 16;

  // per-thread row cursor: (doc, vector id) of this thread's row of a tile
  uint32_t di = 0;
  auto locate = [&](uint32_t tile, int &doc, uint64_t &v) {
    const uint32_t s = tile * kTmTile + row;
    doc = -1;
    v = 0;
    if (tile < n_tiles && s < n_tok) {
      while (d_pref[di + 1] <= s) di++;
      doc = (int)di;
      v = d_off[di] + (s - d_pref[di]);
    }
  };
  auto load_res = [&](uint64_t v, uint32_t (&r)[HW]) {
    const uint8_t *p = ix.residual + v * ix.bytes_per_vec + hf * (HW * 4);
    if constexpr (HW == 8) {
      const uint4 t0 = __ldg(reinterpret_cast<const uint4 *>(p));
      const uint4 t1 = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
      r[0] = t0.x; r[1] = t0.y; r[2] = t0.z; r[3] = t0.w;
      r[4] = t1.x; r[5] = t1.y; r[6] = t1.z; r[7] = t1.w;
    } else if constexpr (HW == 4) {
      const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p));
      r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
    } else {
      const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
      r[0] = t.x; r[1] = t.y;
    }
  };

  // every D stage starts at OFF (this warp's quadrant and column half)
  for (uint32_t st = 0; st < 3; st++)
    for (uint32_t c0 = hf * (N / 2); c0 < (hf + 1) * (N / 2); c0 += 16)
      tmem_fill16(tmem + lane_off + 128u + N * st + c0, off_bits);

  auto epilogue = [&](uint32_t tile) {
    const bool ok = __all_sync(kFull, mbar_wait(&bar[tile & 1], (tile >> 1) & 1));
    if (!ok) {  // warp-uniform: record, skip, stop after the next barrier
      if (lane == 0) { atomicOr(err, 4u); s_abort = 1; }
      return;
    }
    tc_fence_after();
    const int doc = tok_doc[tile % 3][row];
    const uint32_t dcol = tmem + lane_off + 128u + N * (tile % 3);
    for (uint32_t c0 = hf * (N / 2); c0 < (hf + 1) * (N / 2); c0 += 16) {
      uint32_t v[16];
      tmem_ld16(dcol + c0, v);
      tmem_fill16(dcol + c0, off_bits);  // re-arm the stage for tile + 3
      // doc groups of this warp's 32 rows, one uniform pass each: 16 full-warp
      // REDUX, the maxima staged in shared memory, one atomicMax by 16 lanes
      unsigned rem = __ballot_sync(kFull, doc >= 0);
      while (rem) {
        const int g = __shfl_sync(kFull, doc, __ffs(rem) - 1);
        const bool in = doc == g;
        rem &= ~__ballot_sync(kFull, in);
        uint32_t m[16];
#pragma unroll
        for (int j = 0; j < 16; j++) m[j] = __reduce_max_sync(kFull, in ? v[j] : 0u);
        if (lane == 0) {
          uint4 *dst = reinterpret_cast<uint4 *>(stage[warp]);
#pragma unroll
          for (int u = 0; u < 4; u++) dst[u] = make_uint4(m[4 * u], m[4 * u + 1], m[4 * u + 2], m[4 * u + 3]);
        }
        __syncwarp();
        if (lane < 16 && c0 + lane < nq) atomicMax(&best[g * kMaxQueryTok + c0 + lane], stage[warp][lane]);
        __syncwarp();
      }
    }
    tc_fence_before();
  };

  int doc_c;
  uint64_t v_c;
  uint32_t code_c = 0, res_c[HW];
  locate(0, doc_c, v_c);
  if (doc_c >= 0) {
    code_c = __ldg(ix.vq_code + v_c);
    load_res(v_c, res_c);
  }
  for (uint32_t tile = 0; tile < n_tiles; tile++) {
    const int st = tile & 1;
    // centroid half row of this tile (permuted BF16: 8 x 16 B; FP8: 4 x 16 B)
    uint4 cen[CW / 4];
    if (doc_c >= 0) {
      const uint4 *cp = reinterpret_cast<const uint4 *>(cen_perm + (size_t)code_c * (2 * CW) + hf * CW);
#pragma unroll
      for (int u = 0; u < CW / 4; u++) cen[u] = __ldg(cp + u);
    }
    // next tile's code and residual words
    int doc_n;
    uint64_t v_n;
    uint32_t code_n = 0, res_n[HW];
    locate(tile + 1, doc_n, v_n);
    if (doc_n >= 0) {
      code_n = __ldg(ix.vq_code + v_n);
      load_res(v_n, res_n);
    }
    if (tile > 1) epilogue(tile - 2);  // its MMA completed during the previous iteration
    if (hf == 0) tok_doc[tile % 3][row] = doc_c;
    if constexpr (FP8) {
      // A_c: columns 64 st + 16 hf (centroid, as loaded); A_r: + 32 (weights)
      const uint32_t acol = tmem + lane_off + 64u * st + 16u * hf;
      uint32_t out[16];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        out[4 * u] = doc_c >= 0 ? cen[u].x : 0u;
        out[4 * u + 1] = doc_c >= 0 ? cen[u].y : 0u;
        out[4 * u + 2] = doc_c >= 0 ? cen[u].z : 0u;
        out[4 * u + 3] = doc_c >= 0 ? cen[u].w : 0u;
      }
      tmem_st16(acol, out);
      if (doc_c >= 0) {
        if constexpr (NBIT == 4) fp8_decode16_b4(res_c, tw, out);
        else fp8_decode16(res_c, tw.w[0], out);
      } else {
#pragma unroll
        for (int u = 0; u < 16; u++) out[u] = 0u;
      }
      tmem_st16(acol + 32u, out);
    } else {
      const uint32_t acol = tmem + lane_off + 64u * st + 32u * hf;
#pragma unroll
      for (int part = 0; part < 2; part++) {
        uint32_t out[16];
        if (doc_c >= 0) {
          tm_decode16<NBIT>(res_c + part * (HW / 2), cen + part * 4, tw.w[0], tw.w[1], out);
        } else {
#pragma unroll
          for (int u = 0; u < 16; u++) out[u] = 0u;
        }
        tmem_st16(acol + 16u * part, out);
      }
    }
    asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (s_abort) break;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t dcol = tmem + 128u + N * (tile % 3);
      if constexpr (FP8) {
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {  // K = 32 per MMA; centroid part, then residual part
          const uint64_t bd = sw128_desc(b_base + kk * 32);
          mma_e4m3_ta(dcol, tmem + 64u * st + 8u * kk, bd, idesc);        // D starts at OFF
          mma_e4m3_ta(dcol, tmem + 64u * st + 32u + 8u * kk, bd, idesc);
        }
      } else {
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
          const uint64_t bd = sw128_desc(b_base + (kk >> 2) * (N * 128) + (kk & 3) * 32);
          mma_bf16_ta(dcol, tmem + 64u * st + 8u * kk, bd, idesc, 1u);  // D starts at OFF
        }
      }
      mma_commit(&bar[st]);
    }
    doc_c = doc_n;
    v_c = v_n;
    code_c = code_n;
#pragma unroll
    for (int u = 0; u < HW; u++) res_c[u] = res_n[u];
  }
  if (!s_abort && n_tiles > 1) epilogue(n_tiles - 2);
  if (!s_abort && n_tiles > 0) epilogue(n_tiles - 1);
  __syncthreads();

  if (tid < (int)nd && !s_abort) {
    const bool clamp = semantics == 1 && d_len[tid] < ix.max_item_n_vec;
    float s = 0.0f;
    for (uint32_t t = 0; t < nq; t++) {
      float m = __uint_as_float(best[tid * kMaxQueryTok + t]) - off;
      if constexpr (FP8) m *= s_qinv[t];
      if (clamp) m = fmaxf(m, 0.0f);
      s += m;
    }
    approx[(size_t)b * probe_topk + d0 + tid] = s;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(n_cols));
  }
}

// cen_perm[c][w] = bf16x2 of centroid c at K positions 2w, 2w+1 of the
// rerank_tmem_kernel order.
template <int NBIT>
__global__ void perm_centroid_kernel(const float *__restrict__ cen, uint32_t n_cent,
                                     uint32_t *__restrict__ out) {
  const size_t n = (size_t)n_cent * 64;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / 64;
    const uint32_t w = (uint32_t)(i % 64);
    const float *row = cen + c * kDim;
    __nv_bfloat162 p = __floats2bfloat162_rn(row[tm_dim_of<NBIT>(2 * w)], row[tm_dim_of<NBIT>(2 * w + 1)]);
    out[i] = *reinterpret_cast<uint32_t *>(&p);
  }
}

// ---------------------------------------------------------------------
// Centroid scoring on tensor cores.
//
// probe_tc_kernel: CTA = 128 query tokens (operand A, M = 128, BF16
// swizzled in smem) x a range of 64-centroid tiles (operand B, N = 64),
// warp-specialised.  Centroid tiles are stored pre-swizzled in HBM (cen_sw,
// 16 KB per tile, contiguous); one thread of warp 4 streams them by 1-D bulk
// copies (cp.async.bulk, mbarrier transaction count) into a 3-stage ring and
// issues 8 tcgen05.mma per tile into a double-buffered TMEM accumulator
// (2 x 64 columns); commits hand D to the epilogue and free the ring stage,
// and the epilogue releases D as soon as it has loaded it, so the MMAs of
// tile j + 1 run while tile j is scanned.  Epilogue (warps 0-3): thread =
// token row reads its 64 scores with tcgen05.ld (two 32-column chunks) and
// keeps the token's best kCand of the split sorted in registers.  Every
// mbarrier wait is bounded; a timeout sets bit 2 of *err and stops the CTA
// after its MMAs and copies have completed.  A chunk whose max beats the list's
// last score is staged in the thread's shared-memory row and only its
// qualifying columns are inserted (branch-free 16-slot insertion).  Candidate
// ids per token per split go to `cand`; probe_rescore_kernel recomputes their
// scores exactly (canonical FP32 fma chain) and selects the top nprobe.
// ---------------------------------------------------------------------
constexpr int kPtTok = 128;     // tokens per CTA (M) = epilogue threads
constexpr int kPtCen = 64;      // centroids per tile (N)
constexpr int kCand = 16;       // candidates kept per token per split
constexpr int kStage = 36;      // staging row stride in floats (16 B aligned, conflict-free STS.128)
constexpr uint32_t kPtTileBytes = kPtCen * 256;  // one swizzled BF16 centroid tile
constexpr int kPtStages = 3;    // centroid-tile ring stages
constexpr int kPtThreads = 160;  // 4 epilogue warps (one thread per token row) + copy / MMA warp
constexpr size_t kPtSmem = 1024 + 32768 /*A*/ + kPtStages * kPtTileBytes /*B ring*/ +
                           kPtTok * kStage * 4 /*stage*/;

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Insert (v, c) into a register list sorted by score descending, given v >
// s[kCand-1].  Centroids arrive in ascending id order, so an equal score
// already in the list has the smaller id and stays ahead (strict >).  The 16
// comparisons are independent and are collected as bits of one integer; each
// slot then takes its own value, its left neighbour's, or (v, c).  (Holding
// the comparisons as 16 separate bool values under the caller's v > s[15]
// guard was compiled into code that never wrote s[15] in some contexts with
// nvcc 12.9; the bit-mask form is checked by the probe parity tests and a
// per-token insert count.)
__device__ __forceinline__ void topk_insert(float (&s)[kCand], uint32_t (&d)[kCand], float v,
                                            uint32_t c) {
  uint32_t bm = 0;
#pragma unroll
  for (int k = 0; k < kCand; k++) bm |= (v > s[k] ? 1u : 0u) << k;
#pragma unroll
  for (int k = kCand - 1; k >= 1; k--) {
    const bool bk = (bm >> k) & 1u, bp = (bm >> (k - 1)) & 1u;
    const float sk = bp ? s[k - 1] : v;
    const uint32_t dk = bp ? d[k - 1] : c;
    s[k] = bk ? sk : s[k];
    d[k] = bk ? dk : d[k];
  }
  s[0] = (bm & 1u) ? v : s[0];
  d[0] = (bm & 1u) ? c : d[0];
}

__global__ void __launch_bounds__(kPtThreads, 2)
probe_tc_kernel(const float *__restrict__ q, uint32_t n_tok, const uint8_t *__restrict__ cen_sw,
                uint32_t n_cent, uint32_t tiles_per_split, uint32_t n_tiles,
                uint32_t *__restrict__ cand, unsigned *__restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *Aq = smem;                  // [2 K-blocks][128 rows][128 B]
  uint8_t *Bc = smem + 32768;          // [kPtStages][2 K-blocks][64 rows][128 B]
  float *stage_base = reinterpret_cast<float *>(Bc + kPtStages * kPtTileBytes);
  __shared__ uint64_t bfull[kPtStages], bfree[kPtStages], dfull[2], dfree[2], mdone;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t t0 = blockIdx.y * kPtTok;
  const uint32_t tile_begin = blockIdx.x * tiles_per_split;
  const uint32_t tile_end = min(n_tiles, tile_begin + tiles_per_split);
  if (tile_begin >= tile_end) return;
  const uint32_t n_local = tile_end - tile_begin;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < kPtStages; s++) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bfree[s], 1);
    }
    for (int d = 0; d < 2; d++) {
      mbar_init(&dfull[d], 1);
      mbar_init(&dfree[d], 4);
    }
    mbar_init(&mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
  }
  // query tokens -> A (BF16, swizzled; rows >= n_tok zero)
  for (int i = tid; i < kPtTok * 16; i += kPtThreads) {
    const int row = i >> 4, ch = i & 15;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (t0 + row < n_tok) {
      const float4 *src = reinterpret_cast<const float4 *>(q + (size_t)(t0 + row) * kDim + ch * 8);
      const float4 a = __ldg(src), c = __ldg(src + 1);
      __nv_bfloat162 p0 = __floats2bfloat162_rn(a.x, a.y), p1 = __floats2bfloat162_rn(a.z, a.w);
      __nv_bfloat162 p2 = __floats2bfloat162_rn(c.x, c.y), p3 = __floats2bfloat162_rn(c.z, c.w);
      v.x = *reinterpret_cast<uint32_t *>(&p0);
      v.y = *reinterpret_cast<uint32_t *>(&p1);
      v.z = *reinterpret_cast<uint32_t *>(&p2);
      v.w = *reinterpret_cast<uint32_t *>(&p3);
    }
    *reinterpret_cast<uint4 *>(Aq + (ch >> 3) * 16384 + sw128_off(row, ch & 7)) = v;
  }
  fence_async_smem();  // A (generic stores) before the MMAs read it
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  if (warp == 4) {
    // ---------------- copies and MMA issue (one thread) ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(kPtTok, kPtCen);
      const uint32_t a_base = smem_u32(Aq), b_base = smem_u32(Bc);
      uint32_t issued = 0;  // tiles whose copy was issued
      bool ok = true;
      // tile j -> ring stage j % kPtStages, once the MMA that read the
      // stage's previous tile has completed
      auto copy = [&](uint32_t j) -> bool {
        const uint32_t s = j % kPtStages;
        if (j >= (uint32_t)kPtStages &&
            !mbar_wait(&bfree[s], ((j / kPtStages) + 1) & 1, kWaitNs))
          return false;
        mbar_expect_tx(&bfull[s], kPtTileBytes);
        bulk_g2s(b_base + s * kPtTileBytes, cen_sw + (size_t)(tile_begin + j) * kPtTileBytes,
                 kPtTileBytes, &bfull[s]);
        issued = j + 1;
        return true;
      };
      for (uint32_t j = 0; j < n_local && j + 1 < (uint32_t)kPtStages && ok; j++) ok = copy(j);
      uint32_t j = 0;
      for (; ok && j < n_local; j++) {
        if (j + kPtStages - 1 < n_local && !copy(j + kPtStages - 1)) { ok = false; break; }
        const uint32_t s = j % kPtStages, d = j & 1;
        if (!mbar_wait(&bfull[s], (j / kPtStages) & 1, kWaitNs)) { ok = false; break; }
        if (j >= 2 && !mbar_wait(&dfree[d], ((j >> 1) + 1) & 1, kWaitNs)) { ok = false; break; }
        if (s_abort) { ok = false; break; }
        tc_fence_after();
        const uint32_t bt = b_base + s * kPtTileBytes;
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
          const uint64_t ad = sw128_desc(a_base + (kk >> 2) * 16384 + (kk & 3) * 32);
          const uint64_t bd = sw128_desc(bt + (kk >> 2) * (kPtTileBytes / 2) + (kk & 3) * 32);
          mma_bf16(tmem + d * kPtCen, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        mma_commit(&dfull[d]);
        mma_commit(&bfree[s]);
      }
      if (!ok) {
        atomicOr(err, 2u);
        s_abort = 1;
      }
      mma_commit(&mdone);  // every MMA of this CTA has completed once this phase does
      mbar_wait(&mdone, 0);
      // the copies still in flight land before the CTA may exit
      for (uint32_t i = issued > (uint32_t)kPtStages ? issued - kPtStages : 0; i < issued; i++)
        mbar_wait(&bfull[i % kPtStages], (i / kPtStages) & 1);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: thread = token row ----------------
    float *stage = stage_base + tid * kStage;
    float ts[kCand];     // this thread's token: best kCand scores of the split so far
    uint32_t td[kCand];  // and their centroid ids
#pragma unroll
    for (int k = 0; k < kCand; k++) { ts[k] = -INFINITY; td[k] = 0xffffffffu; }
    for (uint32_t j = 0; j < n_local; j++) {
      const uint32_t d = j & 1;
      if (!__all_sync(kFull, mbar_wait(&dfull[d], (j >> 1) & 1, kWaitNs))) {
        if (lane == 0) {
          atomicOr(err, 2u);
          s_abort = 1;
        }
        break;
      }
      tc_fence_after();
      uint32_t r0[32], r1[32];
      tmem_ld32(tmem + ((32u * warp) << 16) + d * kPtCen, r0);
      tmem_ld32(tmem + ((32u * warp) << 16) + d * kPtCen + 32, r1);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&dfree[d]);
#pragma unroll
      for (int part = 0; part < 2; part++) {
        const uint32_t(&r)[32] = part ? r1 : r0;
        float mx = __uint_as_float(r[0]);
#pragma unroll
        for (int i = 1; i < 32; i++) mx = fmaxf(mx, __uint_as_float(r[i]));
        const float thr = ts[kCand - 1];
        if (__any_sync(kFull, mx > thr)) {
          const uint32_t cbase = (tile_begin + j) * kPtCen + part * 32;
          const uint32_t valid = cbase >= n_cent        ? 0u
                                 : n_cent - cbase >= 32 ? 0xffffffffu
                                                        : (1u << (n_cent - cbase)) - 1u;
          uint32_t m4[4] = {0, 0, 0, 0};
#pragma unroll
          for (int i = 0; i < 32; i++) m4[i >> 3] |= (__uint_as_float(r[i]) > thr ? 1u : 0u) << i;
          uint32_t m = ((m4[0] | m4[1]) | (m4[2] | m4[3])) & valid;
          if (m) {
#pragma unroll
            for (int i = 0; i < 8; i++)
              reinterpret_cast<uint4 *>(stage)[i] =
                  make_uint4(r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
            while (m) {
              const int i = __ffs(m) - 1;
              m &= m - 1;
              const float v = stage[i];
              if (v > ts[kCand - 1]) topk_insert(ts, td, v, cbase + i);
            }
          }
          __syncwarp();
        }
      }
      if (__any_sync(kFull, s_abort != 0)) break;
    }
    // this split's candidates of this token: [token][split][kCand], best first
    if (t0 + tid < n_tok && !s_abort) {
      uint4 *dst = reinterpret_cast<uint4 *>(cand + ((size_t)(t0 + tid) * gridDim.x + blockIdx.x) * kCand);
#pragma unroll
      for (int i = 0; i < kCand / 4; i++)
        dst[i] = make_uint4(td[4 * i], td[4 * i + 1], td[4 * i + 2], td[4 * i + 3]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128u));
  }
}

// One warp per token: exact FP32 scores (sequential fma over d, + 1.0f) of
// the token's BF16 candidates, top nprobe by (score desc, id asc).
__global__ void __launch_bounds__(256)
probe_rescore_kernel(const float *__restrict__ q, uint32_t n_tok, const float *__restrict__ cen,
                     uint32_t n_cent, const uint32_t *__restrict__ cand, uint32_t n_cand,
                     uint32_t nprobe, uint32_t *__restrict__ out_id, float *__restrict__ out_s) {
  __shared__ float qs[8][kDim];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t t = blockIdx.x * 8 + w;
  if (t >= n_tok) return;
  for (int d = lane; d < kDim; d += 32) qs[w][d] = q[(size_t)t * kDim + d];
  __syncwarp();
  const int np = (int)nprobe;
  float ls = -INFINITY, thr_s = -INFINITY;
  uint32_t lid = 0xffffffffu, thr_id = 0xffffffffu;
  const uint32_t *cl = cand + (size_t)t * n_cand;
  for (uint32_t c0 = 0; c0 < n_cand; c0 += 32) {
    const uint32_t i = c0 + lane;
    uint32_t c = i < n_cand ? cl[i] : 0xffffffffu;
    float s = -INFINITY;
    if (c < n_cent) {
      const float4 *row = reinterpret_cast<const float4 *>(cen + (size_t)c * kDim);
      float acc = 0.0f;
#pragma unroll 8
      for (int d4 = 0; d4 < kDim / 4; d4++) {
        const float4 x = __ldg(row + d4);
        acc = __fmaf_rn(qs[w][4 * d4 + 0], x.x, acc);
        acc = __fmaf_rn(qs[w][4 * d4 + 1], x.y, acc);
        acc = __fmaf_rn(qs[w][4 * d4 + 2], x.z, acc);
        acc = __fmaf_rn(qs[w][4 * d4 + 3], x.w, acc);
      }
      s = __fadd_rn(acc, 1.0f);
    } else {
      c = 0xffffffffu;
    }
    unsigned m = __ballot_sync(kFull, c != 0xffffffffu && better(s, c, thr_s, thr_id));
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const float ns = __shfl_sync(kFull, s, src);
      const uint32_t nid = __shfl_sync(kFull, c, src);
      if (better(ns, nid, thr_s, thr_id)) {
        const bool ahead = lane < np && better(ls, lid, ns, nid);
        const int pos = __popc(__ballot_sync(kFull, ahead));
        const float up_s = __shfl_up_sync(kFull, ls, 1);
        const uint32_t up_id = __shfl_up_sync(kFull, lid, 1);
        if (lane > pos) { ls = up_s; lid = up_id; }
        else if (lane == pos) { ls = ns; lid = nid; }
        thr_s = __shfl_sync(kFull, ls, np - 1);
        thr_id = __shfl_sync(kFull, lid, np - 1);
      }
    }
  }
  if (lane < np) {
    out_id[(size_t)t * nprobe + lane] = lid;
    out_s[(size_t)t * nprobe + lane] = ls;
  }
}

// cen_sw[tile][kb][row][128 B] = swizzled BF16 centroid rows of 64-centroid
// tiles (rows >= C zero)
__global__ void swizzle_centroid_kernel(const float *__restrict__ cen, uint32_t n_cent,
                                        uint32_t n_tiles, uint8_t *__restrict__ out) {
  const size_t n_chunks = (size_t)n_tiles * kPtCen * 16;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_chunks;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t tile = (uint32_t)(i / (kPtCen * 16));
    const uint32_t row = (uint32_t)((i / 16) % kPtCen), ch = (uint32_t)(i % 16);
    const uint32_t c = tile * kPtCen + row;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (c < n_cent) {
      const float *src = cen + (size_t)c * kDim + ch * 8;
      __nv_bfloat162 p0 = __floats2bfloat162_rn(src[0], src[1]), p1 = __floats2bfloat162_rn(src[2], src[3]);
      __nv_bfloat162 p2 = __floats2bfloat162_rn(src[4], src[5]), p3 = __floats2bfloat162_rn(src[6], src[7]);
      v.x = *reinterpret_cast<uint32_t *>(&p0);
      v.y = *reinterpret_cast<uint32_t *>(&p1);
      v.z = *reinterpret_cast<uint32_t *>(&p2);
      v.w = *reinterpret_cast<uint32_t *>(&p3);
    }
    *reinterpret_cast<uint4 *>(out + (size_t)tile * kPtTileBytes + (ch >> 3) * (kPtTileBytes / 2) +
                               sw128_off(row, ch & 7)) = v;
  }
}

cudaError_t make_centroid_tiles(const float *cen, uint32_t n_cent, uint32_t n_tiles, void *out,
                                cudaStream_t st) {
  swizzle_centroid_kernel<<<592, 256, 0, st>>>(cen, n_cent, n_tiles, reinterpret_cast<uint8_t *>(out));
  return cudaGetLastError();
}

uint32_t probe_tc_cand_per_token(uint32_t n_tok, uint32_t n_cent, int n_sm, uint32_t *splits) {
  const uint32_t n_tiles = (n_cent + kPtCen - 1) / kPtCen;
  const uint32_t tok_tiles = (n_tok + kPtTok - 1) / kPtTok;
  uint32_t s = (2u * (uint32_t)n_sm + tok_tiles - 1) / tok_tiles;  // ~1 wave of 2 CTAs/SM
  s = std::max(1u, std::min(s, n_tiles));
  const uint32_t per = (n_tiles + s - 1) / s;
  *splits = (n_tiles + per - 1) / per;
  return *splits * kCand;
}

cudaError_t launch_probe_tc(const float *q, uint32_t n_tok, const void *cen_sw, const float *cen,
                            uint32_t n_cent, uint32_t nprobe, uint32_t splits, uint32_t *cand,
                            uint32_t *out_id, float *out_s, unsigned *err, cudaStream_t st,
                            int *n_launch) {
  const uint32_t n_tiles = (n_cent + kPtCen - 1) / kPtCen;
  const uint32_t per = (n_tiles + splits - 1) / splits;
  dim3 grid(splits, (n_tok + kPtTok - 1) / kPtTok);
  probe_tc_kernel<<<grid, kPtThreads, kPtSmem, st>>>(q, n_tok, reinterpret_cast<const uint8_t *>(cen_sw),
                                                 n_cent, per, n_tiles, cand, err);
  probe_rescore_kernel<<<(n_tok + 7) / 8, 256, 0, st>>>(q, n_tok, cen, n_cent, cand,
                                                       splits * kCand, nprobe, out_id, out_s);
  *n_launch += 2;
  return cudaGetLastError();
}

// BF16 tables: centroid rows and the byte -> per-value weight table.
// ---------------------------------------------------------------------
// rerank_ws_kernel<NBIT, NMAX, FEAT, DOCS>: the FP8 (E4M3) MaxSim of the
// mixed-precision path for 2- and 4-bit codes, warp-specialised.
//
// The CTA takes DOCS docs of a query's shortlist; their tokens, doc after
// doc, are the rows of its MMA tiles (128 rows per tile; rows past the last
// token are zero).  Roles of the 320 threads:
//  warp 0     producer: per tile, one 1-D bulk copy (cp.async.bulk, completion
//             by mbarrier transaction count) of the residual bytes of every
//             doc segment the tile covers, into stage i % kWsStages of a
//             shared-memory ring;
//  warps 2-5  decoders, one thread per row: the row's vq code (loaded from
//             HBM three tiles ahead), its E4M3 centroid row from L2 (one tile
//             ahead), a tcgen05.st of that row (A_c), the residual bytes from
//             the ring (read in a bank-conflict-free order) expanded by PRMT
//             into E4M3 bucket weights (as rerank_tmem_kernel's FP8 decode),
//             a tcgen05.st of those (A_r);
//  warp 1     MMA: one thread issues per tile a bias MMA that writes OFF into
//             every element of the tile's D stage (a constant A_e of 16.0 in
//             TMEM times a B_e tile of OFF / 512, 32 products summed exactly),
//             then 4 K-steps x 2 tcgen05.mma (kind::f8f6f4, M = 128,
//             N = NMAX, K = 32): A_c and A_r from TMEM, the query tile B from
//             shared memory; commits release the A stage and hand D over;
//  warps 6-9  epilogue, one warp per 32 rows: tcgen05.ld of its rows, the D
//             stage released at once, then for each doc its rows belong to
//             one full-warp REDUX.MAX per query-token column (rows of other
//             docs masked to 0), folded into the per-(doc, query token) maxima
//             by shared-memory atomicMax.
// D starts at OFF, a power of two above |q.x| for every pair of the CTA
// (Cauchy-Schwarz with the query-token norms and the index's bound on |x|),
// so every D value is a positive float ordered like its bit pattern.  With
// FEAT the kernel computes the learned pruner's features instead: the
// centroid part only (no producer, residual decode or residual MMA), and
// per doc the maxima themselves (per query token the best centroid score
// over the doc's tokens) plus log(doc length).  Every pipeline mbarrier wait
// is bounded (wait_ns, 1 s by default); on a timeout the CTA records the
// error and every role stops; the producer then waits (1 s bound) for its
// bulk copies still in flight and the MMA thread for its MMAs before TMEM
// is freed.
// ---------------------------------------------------------------------
constexpr int kWsDocs = 256;         // shortlisted docs per CTA (default; 32, 64, 128 or 256)
constexpr int kWsStages = 4;         // shared-memory ring stages (residual bytes of one tile)
constexpr int kWsDStages = 3;        // D stages in TMEM
constexpr int kWsThreads = 320;

__host__ __device__ constexpr int ws_astages(int nmax) { return nmax <= 32 ? 2 : 4; }
__host__ __device__ constexpr uint32_t ws_cols(int nmax) { return nmax <= 32 ? 256u : 512u; }
__host__ __device__ constexpr uint32_t ws_stage_bytes(int nbit) { return 128u * (128u * nbit / 8u); }
// dynamic shared memory: 1 KB alignment slack + query tile + bias tile + ring;
// the wide (NMAX = 64) variant asks for more than half an SM's shared memory
// so that one CTA holds the SM's 512 TMEM columns alone
__host__ __device__ constexpr size_t ws_smem_bytes(int nbit, int nmax) {
  return nmax <= 32 ? 1024 + 2 * (size_t)nmax * 128 + kWsStages * (size_t)ws_stage_bytes(nbit)
                    : 120 * 1024;
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
      "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
      "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}
// the same word into 8 consecutive TMEM columns of the warp's 32 lanes
__device__ __forceinline__ void tmem_fill8(uint32_t taddr, uint32_t x) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1};\n" ::"r"(
                   taddr),
               "r"(x)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void mma_e4m3_acc(uint32_t tmem_d, uint32_t tmem_a, uint64_t b,
                                             uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], [%1], %2, %3, p;\n}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}

template <int NBIT, int NMAX, bool FEAT = false, int DOCS = kWsDocs>
__global__ void __launch_bounds__(kWsThreads, NMAX <= 32 ? 2 : 1)
rerank_ws_kernel(DevIndex ix, const uint8_t *__restrict__ cen8, TmWeights tw,
                 const float *__restrict__ q, const uint64_t *__restrict__ q_off,
                 const uint32_t *__restrict__ short_id, const uint32_t *__restrict__ n_short,
                 uint32_t probe_topk, int semantics, float x_bound, float *__restrict__ approx,
                 unsigned *__restrict__ err, uint64_t wait_ns) {
  static_assert(NBIT == 2 || NBIT == 4, "FP8 decode of 2- and 4-bit codes");
  static_assert(NMAX == 32 || NMAX == 64, "query tiles of 32 or 64 rows");
  static_assert(!FEAT || NMAX == 32, "pruner features: queries of up to 32 tokens");
  static_assert(DOCS == 32 || DOCS == 64 || DOCS == 128 || (DOCS == 256 && NMAX == 32),
                "docs per CTA (256: the 32-column variant only, whose maxima fit static smem)");
  constexpr int S = kWsStages, SA = ws_astages(NMAX), SD = kWsDStages;
  constexpr uint32_t BPV = 128u * NBIT / 8u;       // residual bytes per token
  constexpr uint32_t STAGE = ws_stage_bytes(NBIT);
  constexpr uint32_t COLS = ws_cols(NMAX);
  constexpr uint32_t DCOL0 = 64u * SA;              // D stages after the A stages
  constexpr uint32_t ECOL = DCOL0 + NMAX * SD;      // bias operand A_e (8 columns)
  static_assert(ECOL + 8 <= COLS, "TMEM columns");
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *Bq = smem;                     // [NMAX rows][128 B] E4M3, SW128, K-major
  uint8_t *Be = smem + NMAX * 128;        // bias B operand, same layout
  uint8_t *ring = smem + 2 * NMAX * 128;  // [S][128 rows][BPV] residual bytes
  __shared__ uint32_t best[DOCS * NMAX];  // [doc][query token]: bits of OFF + max
  __shared__ uint32_t s_qss, tmem_base_s;
  __shared__ float s_qinv[NMAX];
  __shared__ uint64_t full[S], sfree[S], afull[SA], afree[SA], dfull[SD], dempty[SD], mdone;
  __shared__ uint32_t d_len[DOCS], d_pref[DOCS + 1];
  __shared__ uint64_t d_off[DOCS];
  __shared__ volatile int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t b = blockIdx.y;
  const uint32_t ns = n_short[b];
  const uint32_t d0 = blockIdx.x * DOCS;
  const uint64_t tok0 = q_off[b];
  const uint32_t nq = (uint32_t)(q_off[b + 1] - tok0);
  // uniform exits before any TMEM or barrier use: no docs here, or the query
  // belongs to the other width's launch
  if (d0 >= ns || (nq > 32) != (NMAX > 32)) return;
  const uint32_t nd = min((uint32_t)DOCS, ns - d0);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < S; s++) { mbar_init(&full[s], 1); mbar_init(&sfree[s], 4); }
    for (int s = 0; s < SA; s++) { mbar_init(&afull[s], 4); mbar_init(&afree[s], 1); }
    for (int s = 0; s < SD; s++) { mbar_init(&dfull[s], 1); mbar_init(&dempty[s], 4); }
    mbar_init(&mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
    s_qss = 0;
  }
  if (tid < (int)nd) {
    const uint32_t it = short_id[(size_t)b * probe_topk + d0 + tid];
    d_len[tid] = ix.item_n_vec[it];
    d_off[tid] = ix.item_off[it];
  }
  for (int i = tid; i < DOCS * NMAX; i += kWsThreads) best[i] = 0u;
  __syncthreads();
  if (warp == 0) {  // token offsets of the docs within the CTA (warp scan)
    uint32_t carry = 0;
    if (lane == 0) d_pref[0] = 0;
    for (uint32_t base = 0; base < nd; base += 32) {
      uint32_t v = base + lane < nd ? d_len[base + lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
      }
      if (base + lane < nd) d_pref[base + lane + 1] = carry + v;
      carry += __shfl_sync(kFull, v, 31);
    }
  }
  // query tokens -> B (E4M3, per-token power-of-two scales, FP8 K order,
  // swizzled, rows >= nq zero): 8 lanes per row, 16 positions each
  for (int i = tid; i < NMAX * 8; i += kWsThreads) {
    const int row = i >> 3, ch = i & 7;
    float x[16];
    float amax = 0.0f, ss = 0.0f;
#pragma unroll
    for (int u = 0; u < 16; u++) {
      x[u] = (uint32_t)row < nq ? __ldg(q + (tok0 + row) * kDim + fp8_dim_of<NBIT>(16 * ch + u))
                                : 0.0f;
      amax = fmaxf(amax, fabsf(x[u]));
      ss = fmaf(x[u], x[u], ss);
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      amax = fmaxf(amax, __shfl_xor_sync(kFull, amax, o));
      ss += __shfl_xor_sync(kFull, ss, o);
    }
    const float sc = amax > 0.0f ? exp2f(floorf(log2f(224.0f / amax))) : 1.0f;
    uint32_t v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const __nv_fp8x2_storage_t lo = __nv_cvt_float2_to_fp8x2(
          make_float2(x[4 * u] * sc, x[4 * u + 1] * sc), __NV_SATFINITE, __NV_E4M3);
      const __nv_fp8x2_storage_t hi = __nv_cvt_float2_to_fp8x2(
          make_float2(x[4 * u + 2] * sc, x[4 * u + 3] * sc), __NV_SATFINITE, __NV_E4M3);
      v[u] = (uint32_t)lo | ((uint32_t)hi << 16);
    }
    *reinterpret_cast<uint4 *>(Bq + sw128_off(row, ch)) = make_uint4(v[0], v[1], v[2], v[3]);
    if ((lane & 7) == 0) {
      atomicMax(&s_qss, __float_as_uint(ss * sc * sc));
      s_qinv[row] = 1.0f / sc;
    }
  }
  __syncthreads();
  const uint32_t tmem = tmem_base_s;
  const uint32_t T = d_pref[nd];                 // rows (tokens) of the CTA
  const uint32_t n_tiles = (T + 127u) / 128u;
  const float off = fmaxf(1.0f, exp2f(ceilf(log2f(sqrtf(__uint_as_float(s_qss)) * x_bound * 1.15f +
                                                  1e-30f))));
  // bias operands: OFF = 2^e = 32 * A_e * B_e with A_e = 2^a (a in [4, 8],
  // every row and K position of A_e) and B_e = 2^(e - 5 - a) >= 2^-9 in K
  // positions 0..31 of every row of the bias tile (the rest 0): both exact in
  // E4M3, the 32 products sum to OFF exactly, for OFF up to 2^21
  const int e_off = (int)log2f(off);
  const int a_exp = min(8, e_off + 4);
  if (e_off > 21) {  // norms beyond the bias's range: report, do not guess
    if (tid == 0) atomicOr(err, 16u);
  }
  for (int i = tid; i < NMAX * 8; i += kWsThreads) {
    const int row = i >> 3, ch = i & 7;
    const uint32_t e = ch < 2 ? (uint32_t)__nv_cvt_float_to_fp8(exp2f((float)(e_off - 5 - a_exp)),
                                                                __NV_SATFINITE, __NV_E4M3) *
                                    0x01010101u
                              : 0u;
    *reinterpret_cast<uint4 *>(Be + sw128_off(row, ch)) = make_uint4(e, e, e, e);
  }
  const uint32_t qd = warp & 3;  // TMEM lane quadrant of this warp
  const uint32_t lane_off = (32u * qd) << 16;
  if (warp >= 2 && warp < 6) {  // A_e = 2^a: E4M3 exponent field a + 7, mantissa 0
    tmem_fill8(tmem + lane_off + ECOL, (uint32_t)((a_exp + 7) << 3) * 0x01010101u);
    tmem_wait_st();
  }
  fence_async_smem();  // B and bias tiles (generic stores) before the MMAs read them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp == 0) {
    // ---------------- producer: residual bytes of each tile's doc segments ----------------
    if constexpr (!FEAT) {
      const uint32_t ring_u32 = smem_u32(ring);
      uint32_t dfirst = 0, issued = 0;
      bool ok = true;
      for (uint32_t i = 0; i < n_tiles; i++) {
        const uint32_t s = i % S;
        if (i >= (uint32_t)S &&
            !__all_sync(kFull, mbar_wait(&sfree[s], ((i / S) + 1) & 1, wait_ns))) {
          ok = false;
          break;
        }
        const uint32_t R0 = 128u * i, R1 = min(R0 + 128u, T);
        if (lane == 0) mbar_expect_tx(&full[s], (R1 - R0) * BPV);
        __syncwarp();
        for (uint32_t d = dfirst + lane; d < nd && d_pref[d] < R1; d += 32) {
          const uint32_t rs = max(d_pref[d], R0), re = min(d_pref[d + 1], R1);
          if (re > rs)
            bulk_g2s(ring_u32 + s * STAGE + (rs - R0) * BPV,
                     ix.residual + (d_off[d] + (rs - d_pref[d])) * BPV, (re - rs) * BPV, &full[s]);
        }
        while (dfirst < nd && d_pref[dfirst + 1] <= R1) dfirst++;
        issued = i + 1;
        if (__any_sync(kFull, s_abort != 0)) {
          ok = false;
          break;
        }
      }
      if (!ok && lane == 0) {
        atomicOr(err, 4u);
        s_abort = 1;
      }
      // the copies still in flight land before the CTA may exit (after a
      // normal run the decoders have seen every one of them land; after an
      // abort of another role some may still be on their way)
      for (uint32_t i = issued > (uint32_t)S ? issued - S : 0; i < issued; i++)
        mbar_wait(&full[i % S], (i / S) & 1);
    }
  } else if (warp == 1) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_e4m3(128, NMAX);
      const uint32_t b_base = smem_u32(Bq);
      const uint64_t be_desc = sw128_desc(smem_u32(Be));
      uint32_t i = 0;
      for (; i < n_tiles; i++) {
        const uint32_t sa = i % SA, sd = i % SD;
        if (!mbar_wait(&afull[sa], (i / SA) & 1, wait_ns)) break;
        if (i >= (uint32_t)SD && !mbar_wait(&dempty[sd], ((i / SD) + 1) & 1, wait_ns)) break;
        tc_fence_after();
        const uint32_t dcol = tmem + DCOL0 + NMAX * sd;
        mma_e4m3_acc(dcol, tmem + ECOL, be_desc, idesc, 0u);  // D = OFF
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {  // K = 32 per MMA: centroid part, residual part
          const uint64_t bd = sw128_desc(b_base + kk * 32);
          mma_e4m3_acc(dcol, tmem + 64u * sa + 8u * kk, bd, idesc, 1u);
          if constexpr (!FEAT) mma_e4m3_acc(dcol, tmem + 64u * sa + 32u + 8u * kk, bd, idesc, 1u);
        }
        mma_commit(&dfull[sd]);
        mma_commit(&afree[sa]);
        if (s_abort) {
          i++;
          break;
        }
      }
      if (i < n_tiles || s_abort) {
        atomicOr(err, 4u);
        s_abort = 1;
      }
      mma_commit(&mdone);  // every MMA of this CTA has completed once this phase does
      mbar_wait(&mdone, 0);
    }
    __syncwarp();
  } else if (warp < 6) {
    // ---------------- decoders: one thread per row ----------------
    const uint32_t r = 32u * qd + lane;  // row of each tile
    uint32_t dcur = 0;                    // doc of the row whose code is loaded next (monotone)
    auto code_of = [&](uint32_t tile) -> uint32_t {
      const uint32_t g = 128u * tile + r;
      if (tile >= n_tiles || g >= T) return ix.n_centroid;  // the zero row
      while (d_pref[dcur + 1] <= g) dcur++;
      return __ldg(ix.vq_code + d_off[dcur] + (g - d_pref[dcur]));
    };
    uint32_t cen[32];
    auto load_cen = [&](uint32_t code) {
      const uint4 *cp = reinterpret_cast<const uint4 *>(cen8 + (size_t)code * kDim);
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint4 t = __ldg(cp + u);
        cen[4 * u] = t.x;
        cen[4 * u + 1] = t.y;
        cen[4 * u + 2] = t.z;
        cen[4 * u + 3] = t.w;
      }
    };
    // codes three tiles ahead, centroid rows one tile ahead
    const uint32_t c0 = code_of(0);
    uint32_t c1 = code_of(1), c2 = code_of(2);
    load_cen(c0);
    // chunk rotation of the residual reads: rows are BPV bytes apart, so a
    // wavefront's 8 lanes (rows) start in 4 (2-bit) or 2 (4-bit) bank groups
    const uint32_t rot = NBIT == 2 ? ((uint32_t)lane >> 2) & 1u : ((uint32_t)lane >> 1) & 3u;
    bool ok = true;
    for (uint32_t i = 0; ok && i < n_tiles; i++) {
      const uint32_t s = i % S, sa = i % SA;
      if (i >= (uint32_t)SA &&
          !__all_sync(kFull, mbar_wait(&afree[sa], ((i / SA) + 1) & 1, wait_ns))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t acol = tmem + lane_off + 64u * sa;
      tmem_st32(acol, cen);  // A_c: the centroid row as loaded
      tmem_wait_st();
      if (i + 1 < n_tiles) load_cen(c1);
      c1 = c2;
      c2 = code_of(i + 3);
      if constexpr (!FEAT) {
        if (!__all_sync(kFull, mbar_wait(&full[s], (i / S) & 1, wait_ns))) ok = false;
        // A_r: this row's residual words decoded into E4M3 bucket weights
        // (rows past the last token decode stale ring bytes; the epilogue
        // skips them).  The 16-byte chunks of a row are read in an order that
        // depends on the lane, so that the 8 lanes of each shared-memory
        // wavefront hit 8 different groups of 4 banks
        uint32_t res[BPV / 4];
        const uint4 *rp = reinterpret_cast<const uint4 *>(ring + s * STAGE + r * BPV);
        uint4 t[BPV / 16];
#pragma unroll
        for (int u = 0; u < (int)(BPV / 16); u++) t[u] = rp[u ^ rot];
        // undo the rotation: chunk u sits in t[u ^ rot], one swap stage per bit of rot
#pragma unroll
        for (int bit = 1; bit < (int)(BPV / 16); bit <<= 1) {
          if (rot & bit) {
#pragma unroll
            for (int u = 0; u < (int)(BPV / 16); u++)
              if (!(u & bit)) {
                const uint4 x = t[u];
                t[u] = t[u | bit];
                t[u | bit] = x;
              }
          }
        }
#pragma unroll
        for (int u = 0; u < (int)(BPV / 16); u++) {
          res[4 * u] = t[u].x;
          res[4 * u + 1] = t[u].y;
          res[4 * u + 2] = t[u].z;
          res[4 * u + 3] = t[u].w;
        }
        uint32_t out[16];
        if constexpr (NBIT == 4) {
          fp8_decode16_b4(res, tw, out);
          tmem_st16(acol + 32u, out);
          fp8_decode16_b4(res + 8, tw, out);
          tmem_st16(acol + 48u, out);
        } else {
          fp8_decode16(res, tw.w[0], out);
          tmem_st16(acol + 32u, out);
          fp8_decode16(res + 4, tw.w[0], out);
          tmem_st16(acol + 48u, out);
        }
        tmem_wait_st();
      } else {
        (void)rot;
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&afull[sa]);
        if constexpr (!FEAT) mbar_arrive(&sfree[s]);
      }
      if (__any_sync(kFull, s_abort != 0)) ok = false;
    }
    if (!__all_sync(kFull, ok) && lane == 0) {
      atomicOr(err, 4u);
      s_abort = 1;
    }
  } else {
    // ---------------- epilogue: one warp per 32 rows ----------------
    const uint32_t r = 32u * qd + lane;
    uint32_t dcur = 0;
    bool ok = true;
    for (uint32_t i = 0; i < n_tiles; i++) {
      const uint32_t sd = i % SD;
      if (!__all_sync(kFull, mbar_wait(&dfull[sd], (i / SD) & 1, wait_ns))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t dcol = tmem + lane_off + DCOL0 + NMAX * sd;
      uint32_t v0[32];
      tmem_ld32(dcol, v0);
      uint32_t v1[NMAX > 32 ? 32 : 1];
      if constexpr (NMAX > 32) tmem_ld32(dcol + 32u, v1);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&dempty[sd]);
      const uint32_t g = 128u * i + r;
      int doc = -1;
      if (g < T) {
        while (d_pref[dcur + 1] <= g) dcur++;
        doc = (int)dcur;
      }
      // per doc of these rows: REDUX over its rows of every column
      unsigned rem = __ballot_sync(kFull, doc >= 0);
      while (rem) {
        const int gd = __shfl_sync(kFull, doc, __ffs(rem) - 1);
        const bool in = doc == gd;
        const unsigned mem = __ballot_sync(kFull, in);
        rem &= ~mem;
        uint32_t m0 = 0u;
        if (mem == kFull) {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const uint32_t m = __reduce_max_sync(kFull, v0[j]);
            m0 = lane == j ? m : m0;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const uint32_t m = __reduce_max_sync(kFull, in ? v0[j] : 0u);
            m0 = lane == j ? m : m0;
          }
        }
        if ((uint32_t)lane < nq) atomicMax(&best[gd * NMAX + lane], m0);
        if constexpr (NMAX > 32) {
          uint32_t m1 = 0u;
          if (mem == kFull) {
#pragma unroll
            for (int j = 0; j < 32; j++) {
              const uint32_t m = __reduce_max_sync(kFull, v1[j]);
              m1 = lane == j ? m : m1;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 32; j++) {
              const uint32_t m = __reduce_max_sync(kFull, in ? v1[j] : 0u);
              m1 = lane == j ? m : m1;
            }
          }
          if ((uint32_t)lane + 32u < nq) atomicMax(&best[gd * NMAX + 32 + lane], m1);
        }
      }
      if (__any_sync(kFull, s_abort != 0)) {
        ok = false;
        break;
      }
    }
    if (!ok && lane == 0) {
      atomicOr(err, 4u);
      s_abort = 1;
    }
  }
  __syncthreads();

  if constexpr (FEAT) {
    // pruner features: approx is [queries][probe_topk][33]: per query token
    // the doc's best centroid score (0 past the query's last token), then
    // log(doc length)
    for (int i = tid; i < (int)nd * 33 && !s_abort; i += kWsThreads) {
      const int d = i / 33, t = i % 33;
      float f = 0.0f;
      if (t == 32) f = logf((float)d_len[d]);
      else if ((uint32_t)t < nq) f = (__uint_as_float(best[d * NMAX + t]) - off) * s_qinv[t];
      approx[((size_t)b * probe_topk + d0 + d) * 33 + t] = f;
    }
  } else if (tid < (int)nd && !s_abort) {
    const bool clamp = semantics == 1 && d_len[tid] < ix.max_item_n_vec;
    float s = 0.0f;
    for (uint32_t t = 0; t < nq; t++) {
      float m = (__uint_as_float(best[tid * NMAX + t]) - off) * s_qinv[t];
      if (clamp) m = fmaxf(m, 0.0f);
      s += m;
    }
    approx[(size_t)b * probe_topk + d0 + tid] = s;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(COLS));
  }
}

// ---------------------------------------------------------------------
// prune_mlp_kernel: the learned pruner's MLP (33 -> 256 -> 256 -> 1, GELU)
// on the tensor cores, over the features of every shortlisted doc of a
// batch.  Persistent: each CTA loads the BF16 weights once (pre-swizzled
// K-major tiles, 1-D bulk copies: W1 [256 x 64] 32 KB, W2 [256 x 256]
// 128 KB) and loops over tiles of 128 (query, doc) rows.  Per tile: the
// threads write the rows' features as BF16 into a swizzled A tile (K = 33,
// zero-padded to 64); one thread issues 4 tcgen05.mma (kind::f16, M = 128,
// N = 256, K = 16) into a 256-column TMEM accumulator; the 8 warps read it
// back (warp w: lane quadrant w & 3, columns 128 (w >> 2) ..), add b1, apply
// GELU and write H1 as BF16 into a second swizzled A tile [128 x 256]
// (aliasing the feature tile); 16 more MMAs compute H1 W2^T into the same
// columns; the epilogue adds b2, applies GELU, multiplies by w3 and sums
// each row (the two column halves combined through shared memory).  GELU is
// the tanh form with the hardware tanh approximation.
// ---------------------------------------------------------------------
constexpr int kMlpThreads = 256;
constexpr uint32_t kMlpW1Bytes = 256u * 128u, kMlpW2Bytes = 4u * 256u * 128u;
constexpr uint32_t kMlpHBytes = 4u * 128u * 128u;
constexpr size_t kMlpSmem = 1024 + kMlpW1Bytes + kMlpW2Bytes + kMlpHBytes;  // 225 KB

__device__ __forceinline__ float gelu_fast(float x) {
  float t;
  asm("tanh.approx.f32 %0, %1;\n" : "=f"(t) : "f"(0.7978845608f * fmaf(0.044715f * x * x, x, x)));
  return 0.5f * x * (1.0f + t);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&p);
}

__global__ void __launch_bounds__(kMlpThreads, 1)
prune_mlp_kernel(const float *__restrict__ feat, const uint32_t *__restrict__ n_short,
                 uint32_t n_query, uint32_t probe_topk, const uint8_t *__restrict__ wts,
                 const float *__restrict__ vecs, float *__restrict__ pred,
                 unsigned *__restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *W1s = smem, *W2s = smem + kMlpW1Bytes, *H = W2s + kMlpW2Bytes;
  __shared__ uint64_t bar_load, bar_mma;
  __shared__ uint32_t tmem_base_s;
  __shared__ float red[128];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t n_rows = n_query * probe_topk;
  const uint32_t n_tiles = (n_rows + 127u) / 128u;
  if (blockIdx.x >= n_tiles) return;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(&bar_load, 1);
    mbar_init(&bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(&bar_load, kMlpW1Bytes + kMlpW2Bytes);
    for (uint32_t o = 0; o < kMlpW1Bytes + kMlpW2Bytes; o += 16384u)
      bulk_g2s(smem_u32(W1s) + o, wts + o, 16384u, &bar_load);
  }
  bool ok = mbar_wait(&bar_load, 0);
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t qd = warp & 3, hh = warp >> 2;
  const uint32_t lane_off = (32u * qd) << 16;
  const uint32_t row = 32u * qd + lane;  // this thread's row of the tile (epilogues)
  const float *b1 = vecs, *b2 = vecs + 256, *w3 = vecs + 512;
  const float b3 = vecs[768];
  const uint32_t idesc = idesc_bf16(128, 256);
  uint32_t phase = 0;
  for (uint32_t t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
    // features -> BF16 A tile (two threads per row, 4 of the 8 chunks each)
    {
      const uint32_t r = tid >> 1, half = tid & 1;
      const uint32_t gr = t * 128u + r;
      const uint32_t bq = gr / probe_topk, d = gr % probe_topk;
      const bool valid = gr < n_rows && d < n_short[bq];
      const float *f = feat + (size_t)gr * 33;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint32_t ch = half * 4 + c;
        uint32_t v[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const uint32_t k = ch * 8 + 2 * e;
          const float a = valid && k < 33 ? __ldg(f + k) : 0.0f;
          const float bb = valid && k + 1 < 33 ? __ldg(f + k + 1) : 0.0f;
          v[e] = pack_bf16(a, bb);
        }
        *reinterpret_cast<uint4 *>(H + sw128_off(r, ch)) = make_uint4(v[0], v[1], v[2], v[3]);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
#pragma unroll
      for (int ks = 0; ks < 4; ks++)
        mma_bf16(tmem, sw128_desc(smem_u32(H) + 32 * ks), sw128_desc(smem_u32(W1s) + 32 * ks),
                 idesc, ks > 0 ? 1u : 0u);
      mma_commit(&bar_mma);
    }
    if (!__syncthreads_and(mbar_wait(&bar_mma, phase & 1))) { ok = false; break; }
    phase++;
    tc_fence_after();
    // H1 = GELU(X W1^T + b1) -> BF16 A tile of layer 2 (over the feature tile)
    for (uint32_t c0 = 0; c0 < 128; c0 += 32) {
      const uint32_t col0 = 128u * hh + c0;
      uint32_t v[32];
      tmem_ld32(tmem + lane_off + col0, v);
#pragma unroll
      for (int g = 0; g < 4; g++) {  // 4 chunks of 8 columns
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const uint32_t c = col0 + 8 * g + 2 * e;
          const float a = gelu_fast(__uint_as_float(v[8 * g + 2 * e]) + __ldg(b1 + c));
          const float bb = gelu_fast(__uint_as_float(v[8 * g + 2 * e + 1]) + __ldg(b1 + c + 1));
          w[e] = pack_bf16(a, bb);
        }
        const uint32_t col = col0 + 8 * g;
        *reinterpret_cast<uint4 *>(H + (col >> 6) * 16384u + sw128_off(row, (col & 63) >> 3)) =
            make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
#pragma unroll
      for (int kb = 0; kb < 4; kb++)
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
          mma_bf16(tmem, sw128_desc(smem_u32(H) + kb * 16384u + 32 * ks),
                   sw128_desc(smem_u32(W2s) + kb * 32768u + 32 * ks), idesc,
                   (kb | ks) ? 1u : 0u);
      mma_commit(&bar_mma);
    }
    if (!__syncthreads_and(mbar_wait(&bar_mma, phase & 1))) { ok = false; break; }
    phase++;
    tc_fence_after();
    // y = GELU(H1 W2^T + b2) . w3 + b3
    float part = 0.0f;
    for (uint32_t c0 = 0; c0 < 128; c0 += 32) {
      const uint32_t col0 = 128u * hh + c0;
      uint32_t v[32];
      tmem_ld32(tmem + lane_off + col0, v);
#pragma unroll
      for (int j = 0; j < 32; j++)
        part = fmaf(gelu_fast(__uint_as_float(v[j]) + __ldg(b2 + col0 + j)), __ldg(w3 + col0 + j),
                    part);
    }
    if (hh == 1) red[row] = part;
    tc_fence_before();
    __syncthreads();
    if (hh == 0) {
      const uint32_t gr = t * 128u + row;
      if (gr < n_rows) pred[gr] = part + red[row] + b3;
    }
  }
  if (!ok && tid == 0) atomicOr(err, 8u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(256u));
  }
}

// BF16 weight tiles of the MLP kernel from the float parameter vector
// (layout of mvr_prune.cuh): W1 [256 rows][K 64] (K >= 33 zero), then W2 as
// 4 K-blocks of [256 rows][64], all K-major with the 128-byte swizzle; vecs:
// b1, b2, w3 (256 each), b3.
__global__ void prune_prep_kernel(const float *__restrict__ p, uint8_t *__restrict__ wts,
                                  float *__restrict__ vecs) {
  const uint32_t n1 = 256u * 64u, n2 = 4u * 256u * 64u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2 + 769u;
       i += gridDim.x * blockDim.x) {
    if (i < n1) {
      const uint32_t r = i / 64, k = i % 64;
      const float w = k < 33 ? p[r * 33 + k] : 0.0f;
      *reinterpret_cast<__nv_bfloat16 *>(wts + sw128_off(r, k >> 3) + 2 * (k & 7)) =
          __float2bfloat16_rn(w);
    } else if (i < n1 + n2) {
      const uint32_t j = i - n1, kb = j / (256u * 64u), r = (j / 64) % 256u, k = j % 64;
      const float w = p[256u * 33u + 256u + r * 256u + kb * 64u + k];
      *reinterpret_cast<__nv_bfloat16 *>(wts + kMlpW1Bytes + kb * 32768u + sw128_off(r, k >> 3) +
                                         2 * (k & 7)) = __float2bfloat16_rn(w);
    } else {
      const uint32_t j = i - n1 - n2;  // b1 (256), b2 (256), w3 (256), b3
      const uint32_t src = j < 256 ? 256u * 33u + j
                         : j < 512 ? 256u * 33u + 256u + 65536u + (j - 256u)
                         : j < 768 ? 256u * 33u + 256u + 65536u + 256u + (j - 512u)
                                   : 256u * 33u + 256u + 65536u + 512u;
      vecs[j] = j >= 512 && j < 768 ? __bfloat162float(__float2bfloat16_rn(p[src])) : p[src];
    }
  }
}

// Per query (one warp): the docs the rerank takes after the pruner -- the
// `keep` best predictions (kept_id, sorted best first, stride keep) when the
// shortlist is longer than keep and the prediction of its R-th best doc
// leads the keep-th best by at least margin; otherwise the whole shortlist
// (a fallback, counted in *n_fallback).  fin_id / n_fin: stride probe_topk.
// qstat[b * 3 + 2] becomes the chosen docs' token count.
__global__ void prune_choose_kernel(const DevIndex ix, const uint32_t *__restrict__ short_id,
                                    const uint32_t *__restrict__ n_short,
                                    const uint32_t *__restrict__ kept_id,
                                    const float *__restrict__ kept_s, uint32_t n_query,
                                    uint32_t probe_topk, uint32_t keep, uint32_t R, float margin,
                                    uint32_t *__restrict__ fin_id, uint32_t *__restrict__ n_fin,
                                    uint32_t *__restrict__ qstat,
                                    unsigned long long *__restrict__ n_fallback) {
  const uint32_t b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= n_query) return;
  const uint32_t ns = n_short[b];
  bool prune = ns > keep;
  if (prune) {
    const float *ks = kept_s + (size_t)b * keep;
    prune = ks[min(R, keep) - 1] - ks[keep - 1] >= margin;
    if (!prune && lane == 0) atomicAdd(n_fallback, 1ull);
  }
  const uint32_t n = prune ? keep : ns;
  const uint32_t *src = prune ? kept_id + (size_t)b * keep : short_id + (size_t)b * probe_topk;
  uint32_t tok = 0;
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t d = src[i];
    fin_id[(size_t)b * probe_topk + i] = d;
    tok += ix.item_n_vec[d];
  }
  tok = __reduce_add_sync(kFull, tok);
  if (lane == 0) {
    n_fin[b] = n;
    qstat[b * 3 + 2] = tok;
  }
}

__global__ void to_bf16_kernel(const float *__restrict__ in, size_t n, __nv_bfloat16 *__restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

cudaError_t make_bf16(const float *in, size_t n, void *out, cudaStream_t st) {
  to_bf16_kernel<<<592, 256, 0, st>>>(in, n, reinterpret_cast<__nv_bfloat16 *>(out));
  return cudaGetLastError();
}

cudaError_t configure_tc_kernels() {
  cudaError_t e;
  e = cudaFuncSetAttribute(rerank_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes(1, 64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes(2, 64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes(4, 64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(probe_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPtSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tmem_kernel<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tm_smem_bytes(64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tmem_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tm_smem_bytes(64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tmem_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tm_smem_bytes(64));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tmem_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tm_smem_bytes(64));
  if (e != cudaSuccess) return e;
#define MVR_WS_ATTR(NB, NM, F, D)                                                                \
  e = cudaFuncSetAttribute(rerank_ws_kernel<NB, NM, F, D>,                                       \
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws_smem_bytes(NB, NM)); \
  if (e != cudaSuccess) return e;
  MVR_WS_ATTR(2, 32, false, 32) MVR_WS_ATTR(2, 32, false, 64) MVR_WS_ATTR(2, 32, false, 128)
  MVR_WS_ATTR(2, 32, false, 256) MVR_WS_ATTR(4, 32, false, 256)
  MVR_WS_ATTR(2, 64, false, 32) MVR_WS_ATTR(2, 64, false, 64) MVR_WS_ATTR(2, 64, false, 128)
  MVR_WS_ATTR(4, 32, false, 32) MVR_WS_ATTR(4, 32, false, 64) MVR_WS_ATTR(4, 32, false, 128)
  MVR_WS_ATTR(4, 64, false, 32) MVR_WS_ATTR(4, 64, false, 64) MVR_WS_ATTR(4, 64, false, 128)
  // the pruner's feature launch: the default docs per CTA
  MVR_WS_ATTR(2, 32, true, kWsDocs) MVR_WS_ATTR(4, 32, true, kWsDocs)
#undef MVR_WS_ATTR
  e = cudaFuncSetAttribute(prune_mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMlpSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(rerank_tc_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes(8, 64));
}

cudaError_t launch_rerank_tc(const DevIndex &ix, const void *cen_bf16, const void *lut_bf16,
                             const float *q, const uint64_t *q_off, uint32_t n_query,
                             const uint32_t *short_id, const uint32_t *n_short,
                             uint32_t probe_topk, int semantics, uint32_t nq_max, float *approx,
                             unsigned *err, cudaStream_t st, int *n_launch) {
  dim3 grid((probe_topk + kTcDocs - 1) / kTcDocs, n_query);
  const uint32_t n_max = nq_max <= 32 ? 32u : 64u;
  const size_t sm = tc_smem_bytes((int)ix.n_bit, n_max);
  const __nv_bfloat16 *c = reinterpret_cast<const __nv_bfloat16 *>(cen_bf16);
  const __nv_bfloat16 *l = reinterpret_cast<const __nv_bfloat16 *>(lut_bf16);
  switch (ix.n_bit) {
    case 1: rerank_tc_kernel<1><<<grid, kTcThreads, sm, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, n_max, approx, err); break;
    case 2: rerank_tc_kernel<2><<<grid, kTcThreads, sm, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, n_max, approx, err); break;
    case 4: rerank_tc_kernel<4><<<grid, kTcThreads, sm, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, n_max, approx, err); break;
    case 8: rerank_tc_kernel<8><<<grid, kTcThreads, sm, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, n_max, approx, err); break;
    default: return cudaErrorInvalidValue;
  }
  *n_launch += 1;
  return cudaGetLastError();
}

bool tmem_rerank_supported(uint32_t n_bit) { return n_bit == 1 || n_bit == 2; }
bool fp8_rerank_supported(uint32_t n_bit) { return n_bit == 2 || n_bit == 4; }

TmWeights make_tm_weights(uint32_t n_bit, const float *weight, bool fp8) {
  TmWeights t{};
  auto e4m3 = [](float v) { return (uint32_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3); };
  if (fp8 && n_bit == 4) {
    for (uint32_t k = 0; k < 16; k++) {
      const uint32_t e = e4m3(weight[k]);
      const uint32_t j = k & 7u, sh = 8u * (j & 3u);
      t.w[(k >> 3) * 2 + (j >> 2)] |= (e & 0x7fu) << sh;          // magnitude tables
      t.w[4 + (j >> 2)] |= ((e >> 7) << (k < 8 ? 6u : 7u)) << sh;  // sign table
    }
  } else if (fp8) {
    for (uint32_t k = 0; k < (1u << n_bit); k++) t.w[0] |= e4m3(weight[k]) << (8 * k);
  } else {
    for (uint32_t k = 0; k < (1u << n_bit) && k < 4; k++) {
      const __nv_bfloat16 b = __float2bfloat16_rn(weight[k]);
      const uint16_t wb = *reinterpret_cast<const uint16_t *>(&b);
      t.w[0] |= (uint32_t)(wb & 0xffu) << (8 * k);
      t.w[1] |= (uint32_t)(wb >> 8) << (8 * k);
    }
  }
  return t;
}

// cen8[c][k] = E4M3 of centroid c at K position k of the FP8 rerank order
template <int NBIT>
__global__ void perm_centroid_fp8_kernel(const float *__restrict__ cen, uint32_t n_cent,
                                         uint8_t *__restrict__ out) {
  const size_t n = (size_t)n_cent * kDim;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / kDim;
    out[i] = __nv_cvt_float_to_fp8(cen[c * kDim + fp8_dim_of<NBIT>((uint32_t)(i % kDim))],
                                   __NV_SATFINITE, __NV_E4M3);
  }
}

cudaError_t make_centroid_fp8(const float *cen, uint32_t n_cent, uint32_t n_bit, void *out,
                              cudaStream_t st) {
  uint8_t *o = reinterpret_cast<uint8_t *>(out);
  if (n_bit == 2) perm_centroid_fp8_kernel<2><<<592, 256, 0, st>>>(cen, n_cent, o);
  else if (n_bit == 4) perm_centroid_fp8_kernel<4><<<592, 256, 0, st>>>(cen, n_cent, o);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

__global__ void centroid_norm_max_kernel(const float *__restrict__ cen, uint32_t n_cent,
                                         unsigned *__restrict__ out) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cent; c += gridDim.x * blockDim.x) {
    const float4 *row = reinterpret_cast<const float4 *>(cen + (size_t)c * kDim);
    float ss = 0.0f;
    for (int i = 0; i < kDim / 4; i++) {
      const float4 v = row[i];
      ss = fmaf(v.x, v.x, fmaf(v.y, v.y, fmaf(v.z, v.z, fmaf(v.w, v.w, ss))));
    }
    atomicMax(out, __float_as_uint(sqrtf(ss)));
  }
}

cudaError_t max_centroid_norm(const float *cen, uint32_t n_cent, unsigned *d_tmp, float *out,
                              cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_tmp, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  centroid_norm_max_kernel<<<296, 256, 0, st>>>(cen, n_cent, d_tmp);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  unsigned bits = 0;
  e = cudaMemcpyAsync(&bits, d_tmp, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);
  std::memcpy(out, &bits, 4);
  return e;
}

cudaError_t make_centroid_perm(const float *cen, uint32_t n_cent, uint32_t n_bit, void *out,
                               cudaStream_t st) {
  uint32_t *o = reinterpret_cast<uint32_t *>(out);
  if (n_bit == 2) perm_centroid_kernel<2><<<592, 256, 0, st>>>(cen, n_cent, o);
  else if (n_bit == 1) perm_centroid_kernel<1><<<592, 256, 0, st>>>(cen, n_cent, o);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_rerank_tmem(const DevIndex &ix, const void *cen_perm, const TmWeights &tw,
                               const float *q, const uint64_t *q_off, uint32_t n_query,
                               const uint32_t *short_id, const uint32_t *n_short,
                               uint32_t probe_topk, int semantics, uint32_t nq_max, float x_bound,
                               float *approx, unsigned *err, cudaStream_t st, int *n_launch,
                               bool fp8) {
  if (fp8 ? !fp8_rerank_supported(ix.n_bit) : !tmem_rerank_supported(ix.n_bit))
    return cudaErrorInvalidValue;
  dim3 grid((probe_topk + kTmDocs - 1) / kTmDocs, n_query);
  const uint32_t n_max = nq_max <= 32 ? 32u : 64u;
  const size_t sm = tm_smem_bytes(n_max);
  const uint32_t *c = reinterpret_cast<const uint32_t *>(cen_perm);
#define MVR_TM_LAUNCH(NB, F8)                                                                   \
  rerank_tmem_kernel<NB, F8><<<grid, kTmThreads, sm, st>>>(ix, c, tw, q, q_off, short_id, n_short, \
                                                           probe_topk, semantics, n_max, x_bound, \
                                                           approx, err)
  if (fp8 && ix.n_bit == 4) MVR_TM_LAUNCH(4, true);
  else if (fp8) MVR_TM_LAUNCH(2, true);
  else if (ix.n_bit == 2) MVR_TM_LAUNCH(2, false);
  else MVR_TM_LAUNCH(1, false);
#undef MVR_TM_LAUNCH
  *n_launch += 1;
  return cudaGetLastError();
}

bool ws_docs_supported(uint32_t docs) {
  return docs == 32 || docs == 64 || docs == 128 || docs == 256;
}

template <int NB, int NM, int DOCS>
static void ws_launch(const DevIndex &ix, const uint8_t *c, const TmWeights &tw, const float *q,
                      const uint64_t *q_off, uint32_t n_query, const uint32_t *short_id,
                      const uint32_t *n_short, uint32_t probe_topk, int semantics, float x_bound,
                      float *approx, unsigned *err, cudaStream_t st, uint64_t wait_ns) {
  const dim3 grid((probe_topk + DOCS - 1) / DOCS, n_query);
  rerank_ws_kernel<NB, NM, false, DOCS><<<grid, kWsThreads, ws_smem_bytes(NB, NM), st>>>(
      ix, c, tw, q, q_off, short_id, n_short, probe_topk, semantics, x_bound, approx, err,
      wait_ns);
}

template <int NB, int NM>
static void ws_launch_docs(uint32_t docs, const DevIndex &ix, const uint8_t *c,
                           const TmWeights &tw, const float *q, const uint64_t *q_off,
                           uint32_t n_query, const uint32_t *short_id, const uint32_t *n_short,
                           uint32_t probe_topk, int semantics, float x_bound, float *approx,
                           unsigned *err, cudaStream_t st, uint64_t wait_ns) {
  if (docs == 32)
    ws_launch<NB, NM, 32>(ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk, semantics,
                          x_bound, approx, err, st, wait_ns);
  else if (docs == 256 && NM == 32)  // the 64-column variant's maxima would not fit: 128 there
    ws_launch<NB, NM, NM == 32 ? 256 : 128>(ix, c, tw, q, q_off, n_query, short_id, n_short,
                                            probe_topk, semantics, x_bound, approx, err, st,
                                            wait_ns);
  else if (docs >= 128)
    ws_launch<NB, NM, 128>(ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk, semantics,
                           x_bound, approx, err, st, wait_ns);
  else
    ws_launch<NB, NM, 64>(ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk, semantics,
                          x_bound, approx, err, st, wait_ns);
}

cudaError_t launch_rerank_ws(const DevIndex &ix, const void *cen8, const TmWeights &tw,
                             const float *q, const uint64_t *q_off, uint32_t n_query,
                             const uint32_t *short_id, const uint32_t *n_short,
                             uint32_t probe_topk, int semantics, uint32_t nq_max, float x_bound,
                             float *approx, unsigned *err, cudaStream_t st, int *n_launch,
                             uint64_t wait_ns, uint32_t docs) {
  if (!fp8_rerank_supported(ix.n_bit) || !ws_docs_supported(docs)) return cudaErrorInvalidValue;
  const uint8_t *c = reinterpret_cast<const uint8_t *>(cen8);
  // queries of up to 32 tokens run in the 32-column variant (two CTAs per
  // SM), longer ones in the 64-column variant (one CTA per SM); each launch
  // skips the other's queries
  if (ix.n_bit == 4)
    ws_launch_docs<4, 32>(docs, ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk,
                          semantics, x_bound, approx, err, st, wait_ns);
  else
    ws_launch_docs<2, 32>(docs, ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk,
                          semantics, x_bound, approx, err, st, wait_ns);
  *n_launch += 1;
  if (nq_max > 32) {
    if (ix.n_bit == 4)
      ws_launch_docs<4, 64>(docs, ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk,
                            semantics, x_bound, approx, err, st, wait_ns);
    else
      ws_launch_docs<2, 64>(docs, ix, c, tw, q, q_off, n_query, short_id, n_short, probe_topk,
                            semantics, x_bound, approx, err, st, wait_ns);
    *n_launch += 1;
  }
  return cudaGetLastError();
}

cudaError_t launch_prune_features(const DevIndex &ix, const void *cen8, const float *q,
                                  const uint64_t *q_off, uint32_t n_query,
                                  const uint32_t *short_id, const uint32_t *n_short,
                                  uint32_t probe_topk, float x_bound, float *feat, unsigned *err,
                                  cudaStream_t st, int *n_launch, uint64_t wait_ns) {
  if (!fp8_rerank_supported(ix.n_bit)) return cudaErrorInvalidValue;
  const dim3 grid((probe_topk + kWsDocs - 1) / kWsDocs, n_query);
  const uint8_t *c = reinterpret_cast<const uint8_t *>(cen8);
  const TmWeights none{};
  if (ix.n_bit == 4)
    rerank_ws_kernel<4, 32, true><<<grid, kWsThreads, ws_smem_bytes(4, 32), st>>>(
        ix, c, none, q, q_off, short_id, n_short, probe_topk, 0, x_bound, feat, err, wait_ns);
  else
    rerank_ws_kernel<2, 32, true><<<grid, kWsThreads, ws_smem_bytes(2, 32), st>>>(
        ix, c, none, q, q_off, short_id, n_short, probe_topk, 0, x_bound, feat, err, wait_ns);
  *n_launch += 1;
  return cudaGetLastError();
}

cudaError_t launch_prune_choose(const DevIndex &ix, const uint32_t *short_id,
                                const uint32_t *n_short, const uint32_t *kept_id,
                                const float *kept_s, uint32_t n_query, uint32_t probe_topk,
                                uint32_t keep, uint32_t R, float margin, uint32_t *fin_id,
                                uint32_t *n_fin, uint32_t *qstat,
                                unsigned long long *n_fallback, cudaStream_t st, int *n_launch) {
  prune_choose_kernel<<<(n_query + 7) / 8, 256, 0, st>>>(ix, short_id, n_short, kept_id, kept_s,
                                                         n_query, probe_topk, keep, R, margin,
                                                         fin_id, n_fin, qstat, n_fallback);
  *n_launch += 1;
  return cudaGetLastError();
}

size_t prune_weight_bytes() { return kMlpW1Bytes + kMlpW2Bytes; }

cudaError_t prune_prepare(const float *params, uint8_t *wts, float *vecs, cudaStream_t st) {
  prune_prep_kernel<<<592, 256, 0, st>>>(params, wts, vecs);
  return cudaGetLastError();
}

cudaError_t launch_prune_mlp(const float *feat, const uint32_t *n_short, uint32_t n_query,
                             uint32_t probe_topk, const uint8_t *wts, const float *vecs,
                             float *pred, unsigned *err, int n_sm, cudaStream_t st,
                             int *n_launch) {
  const uint32_t tiles = (n_query * probe_topk + 127u) / 128u;
  const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)n_sm);
  if (grid == 0) return cudaSuccess;
  prune_mlp_kernel<<<grid, kMlpThreads, kMlpSmem, st>>>(feat, n_short, n_query, probe_topk, wts,
                                                         vecs, pred, err);
  *n_launch += 1;
  return cudaGetLastError();
}

}  // namespace mvr
