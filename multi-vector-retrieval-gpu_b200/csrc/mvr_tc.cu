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

#include <cuda_bf16.h>

namespace mvr {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTcTile = 128;      // doc tokens per MMA tile (M)
constexpr int kTcDocs = 32;       // shortlisted docs per CTA
constexpr int kTcThreads = 256;
constexpr uint32_t kWaitLimit = 1u << 26;  // bounded mbarrier polls (~1 s)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

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

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait on an mbarrier phase; returns false after kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
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

__device__ __forceinline__ uint32_t find_doc(const uint32_t *pref, int n, uint32_t e) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return (uint32_t)lo;
}

}  // namespace

// smem layout (dynamic, 1024-aligned inside): A[2] 2 x 32 KB, B 16 KB,
// lut (bf16) <= 4 KB, best [64][kTcDocs] ints 8 KB
constexpr size_t kTcSmem = 1024 + 2 * 32768 + 16384 + 4096 + 64 * kTcDocs * 4;

template <int NBIT>
__global__ void __launch_bounds__(kTcThreads, 1)
rerank_tc_kernel(DevIndex ix, const __nv_bfloat16 *__restrict__ cen_bf16,
                 const __nv_bfloat16 *__restrict__ lut_bf16, const float *__restrict__ q,
                 const uint64_t *__restrict__ q_off, const uint32_t *__restrict__ short_id,
                 const uint32_t *__restrict__ n_short, uint32_t probe_topk, int semantics,
                 float *__restrict__ approx, unsigned *__restrict__ err) {
  constexpr int VPB = 8 / NBIT;
  constexpr int HALF_BYTES = 64 / VPB;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *A0 = smem;              // [2][2 K-blocks][128 rows][128 B]
  uint8_t *Bq = smem + 2 * 32768;  // [2 K-blocks][64 rows][128 B]
  __nv_bfloat16 *lut = reinterpret_cast<__nv_bfloat16 *>(Bq + 16384);  // [256][VPB]
  int *best = reinterpret_cast<int *>(Bq + 16384 + 4096);             // [64][kTcDocs]
  __shared__ uint64_t bars[2];
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
  const uint32_t N = nq <= 32 ? 32u : 64u;
  const uint32_t idesc = idesc_bf16(kTcTile, (int)N);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
  }
  if (tid < (int)nd) {
    const uint32_t it = short_id[(size_t)b * probe_topk + d0 + tid];
    d_len[tid] = ix.item_n_vec[it];
    d_off[tid] = ix.item_off[it];
  }
  for (int i = tid; i < 256 * VPB; i += kTcThreads) lut[i] = lut_bf16[i];
  for (int i = tid; i < 64 * kTcDocs; i += kTcThreads) best[i] = f2si(-INFINITY);
  // query tokens -> B operand (BF16, swizzled, rows >= nq zero)
  for (int i = tid; i < 64 * 16; i += kTcThreads) {
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
    if ((uint32_t)row < N)
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
  const uint32_t a_base = smem_u32(A0), b_base = smem_u32(Bq);

  auto epilogue = [&](uint32_t tile) {
    const int buf = tile & 1;
    const bool ok = __all_sync(kFull, mbar_wait(&bars[buf], (tile >> 1) & 1));
    if (!ok) {  // warp-uniform: record, skip this tile, stop after the next barrier
      if (lane == 0) { atomicOr(err, 1u); s_abort = 1; }
      return;
    }
    tc_fence_after();
    const uint32_t row = 32 * (warp & 3) + lane;
    const int doc = tok_doc[buf][row];
    const unsigned grp = __match_any_sync(kFull, doc);
    const bool leader = lane == __ffs(grp) - 1;
    for (uint32_t c0 = (warp >> 2) * (N / 2); c0 < (warp >> 2) * (N / 2) + N / 2; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + ((32u * (warp & 3)) << 16) + buf * N + c0, r);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int m = __reduce_max_sync(grp, f2si(__uint_as_float(r[j])));
        if (leader && doc >= 0 && c0 + j < nq) atomicMax(&best[(c0 + j) * kTcDocs + doc], m);
      }
    }
    tc_fence_before();
  };

  for (uint32_t tile = 0; tile < n_tiles; tile++) {
    const int buf = tile & 1;
    uint8_t *Ab = A0 + buf * 32768;
    // -- decompress 128 tokens to BF16: thread = (row tid&127, half tid>>7) --
    {
      const uint32_t row = tid & (kTcTile - 1), half = tid >> 7;
      const uint32_t s = tile * kTcTile + row;
      uint8_t *kb = Ab + half * 16384;
      if (s < n_tok) {
        const uint32_t di = find_doc(d_pref, (int)nd, s);
        const uint64_t v = d_off[di] + (s - d_pref[di]);
        if (half == 0) tok_doc[buf][row] = (int)di;
        const uint4 *cen = reinterpret_cast<const uint4 *>(cen_bf16 + (size_t)ix.vq_code[v] * kDim + half * 64);
        const uint8_t *res = ix.residual + v * ix.bytes_per_vec + half * HALF_BYTES;
        uint8_t rb[HALF_BYTES];
#pragma unroll
        for (int u = 0; u < HALF_BYTES / 8; u++)
          *reinterpret_cast<uint2 *>(rb + 8 * u) = __ldg(reinterpret_cast<const uint2 *>(res) + u);
#pragma unroll
        for (int c = 0; c < 8; c++) {  // 8 dims per 16-byte chunk
          uint4 cv = __ldg(cen + c);
          __nv_bfloat162 *cp = reinterpret_cast<__nv_bfloat162 *>(&cv);
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int d = c * 8 + 2 * u;
            const __nv_bfloat16 w0 = lut[(uint32_t)rb[d / VPB] * VPB + (d % VPB)];
            const __nv_bfloat16 w1 = lut[(uint32_t)rb[(d + 1) / VPB] * VPB + ((d + 1) % VPB)];
            cp[u] = __hadd2(cp[u], __halves2bfloat162(w0, w1));
          }
          *reinterpret_cast<uint4 *>(kb + sw128_off(row, c)) = cv;
        }
      } else {
        if (half == 0) tok_doc[buf][row] = -1;
#pragma unroll
        for (int c = 0; c < 8; c++) *reinterpret_cast<uint4 *>(kb + sw128_off(row, c)) = make_uint4(0, 0, 0, 0);
      }
    }
    fence_async_smem();
    __syncthreads();
    if (s_abort) break;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_tile = a_base + buf * 32768;
#pragma unroll
      for (int kk = 0; kk < 8; kk++) {
        const uint64_t ad = sw128_desc(a_tile + (kk >> 2) * 16384 + (kk & 3) * 32);
        const uint64_t bd = sw128_desc(b_base + (kk >> 2) * (N * 128) + (kk & 3) * 32);
        mma_bf16(tmem + buf * N, ad, bd, idesc, kk > 0 ? 1u : 0u);
      }
      mma_commit(&bars[buf]);
    }
    if (tile > 0) epilogue(tile - 1);
    __syncthreads();
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128u));
  }
}

// BF16 tables: centroid rows and the byte -> per-value weight table.
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
  e = cudaFuncSetAttribute(rerank_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rerank_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(rerank_tc_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
}

cudaError_t launch_rerank_tc(const DevIndex &ix, const void *cen_bf16, const void *lut_bf16,
                             const float *q, const uint64_t *q_off, uint32_t n_query,
                             const uint32_t *short_id, const uint32_t *n_short,
                             uint32_t probe_topk, int semantics, float *approx, unsigned *err,
                             cudaStream_t st, int *n_launch) {
  dim3 grid((probe_topk + kTcDocs - 1) / kTcDocs, n_query);
  const __nv_bfloat16 *c = reinterpret_cast<const __nv_bfloat16 *>(cen_bf16);
  const __nv_bfloat16 *l = reinterpret_cast<const __nv_bfloat16 *>(lut_bf16);
  switch (ix.n_bit) {
    case 1: rerank_tc_kernel<1><<<grid, kTcThreads, kTcSmem, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, approx, err); break;
    case 2: rerank_tc_kernel<2><<<grid, kTcThreads, kTcSmem, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, approx, err); break;
    case 4: rerank_tc_kernel<4><<<grid, kTcThreads, kTcSmem, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, approx, err); break;
    case 8: rerank_tc_kernel<8><<<grid, kTcThreads, kTcSmem, st>>>(ix, c, l, q, q_off, short_id, n_short, probe_topk, semantics, approx, err); break;
    default: return cudaErrorInvalidValue;
  }
  *n_launch += 1;
  return cudaGetLastError();
}

}  // namespace mvr
