// mvr_common.cuh -- device-side types and helpers shared by the search
// kernels of libmvr (B200, sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mvr {

constexpr int kDim = 128;          // token embedding width (ColBERTv2)
constexpr int kMaxQueryTok = 64;   // query tokens per query
constexpr int kMaxProbe = 32;      // nprobe upper bound
constexpr int kMaxShort = 8192;    // probe_topk upper bound
constexpr int kMaxTopk = 1024;
constexpr int kHashParts = 64;     // doc ranges of the hash filter's partition table (max CTAs per query)

// Index arrays resident in HBM (one copy per loaded index).
struct DevIndex {
  uint32_t n_item, n_centroid, n_centroid_pad, n_bit, bytes_per_vec;
  uint32_t max_item_n_vec;
  uint64_t n_vec, n_ele_ivf;
  const float *centroid;      // [C][128] row-major
  const float *centroid_t;    // [128][C_pad] (columns >= C are zero)
  const uint32_t *vq_code;    // [n_vec]
  const uint8_t *residual;    // [n_vec][bytes_per_vec]
  const uint32_t *item_n_vec; // [n_item]
  const uint64_t *item_off;   // [n_item]
  const uint64_t *ivf_off;    // [C]
  const uint32_t *ivf_size;   // [C]
  const uint32_t *ivf_ids;    // [n_ele_ivf]
  const float *lut;           // [256][8/n_bit] byte -> per-value weight
  const uint32_t *ivf_part;   // [C][kHashParts + 1] doc-range sub-list starts
};

// (score desc, id asc) total order used by every top-k on the path.
__host__ __device__ __forceinline__ bool better(float s1, uint32_t i1, float s2,
                                                uint32_t i2) {
  return s1 > s2 || (s1 == s2 && i1 < i2);
}

// float -> uint32 whose unsigned order equals the float order.
__host__ __device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  __builtin_memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
#ifdef __CUDA_ARCH__
  f = __uint_as_float(u);
#else
  __builtin_memcpy(&f, &u, 4);
#endif
  return f;
}
// 64-bit key: larger key == better (score desc, id asc).
__host__ __device__ __forceinline__ uint64_t make_key(float s, uint32_t id) {
  return ((uint64_t)f2ord(s) << 32) | (uint64_t)(~id);
}
__host__ __device__ __forceinline__ float key_score(uint64_t k) {
  return ord2f((uint32_t)(k >> 32));
}
__host__ __device__ __forceinline__ uint32_t key_id(uint64_t k) {
  return ~(uint32_t)k;
}

// float <-> signed int whose signed order equals the float order (for
// shared-memory atomicMax / __reduce_max_sync on scores).
__device__ __forceinline__ int f2si(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float si2f(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

}  // namespace mvr
