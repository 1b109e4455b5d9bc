// mvr_aux.cu -- index-side kernels of libmvr: centroid transpose for the
// probe kernel, standalone decode (decompression / bucket unpack with the
// rerank decoder's bit layout) and the index-build kernels (residual packing,
// FP64 k-means accumulation).
#include "mvr_aux.cuh"

#include <cstring>
#include <vector>

namespace mvr {

// ct[k][c] = centroid[c][k] for c < C, 0 for C <= c < C_pad.
__global__ void transpose_centroid_kernel(const float *__restrict__ cen, uint32_t n_cent,
                                          uint32_t n_cent_pad, float *__restrict__ ct) {
  __shared__ float tile[32][33];
  const uint32_t c0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const uint32_t c = c0 + r, k = k0 + tx;
    tile[r][tx] = (c < n_cent) ? cen[(size_t)c * kDim + k] : 0.0f;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const uint32_t k = k0 + r, c = c0 + tx;
    if (c < n_cent_pad) ct[(size_t)k * n_cent_pad + c] = tile[tx][r];
  }
}

cudaError_t launch_transpose_centroid(const float *cen, uint32_t n_cent, uint32_t n_cent_pad,
                                      float *ct, cudaStream_t st) {
  dim3 grid(n_cent_pad / 32, kDim / 32), block(32, 8);
  transpose_centroid_kernel<<<grid, block, 0, st>>>(cen, n_cent, n_cent_pad, ct);
  return cudaGetLastError();
}

// value i of a packed byte (MSB-first): (byte >> (8 - b*(i+1))) & (2^b - 1)
__device__ __forceinline__ uint32_t bucket_of(const uint8_t *res, uint32_t d, uint32_t n_bit) {
  const uint32_t vpb = 8u / n_bit;
  const uint32_t byte = res[d / vpb];
  const uint32_t i = d % vpb;
  return (byte >> (8u - n_bit * (i + 1u))) & ((1u << n_bit) - 1u);
}

__global__ void decompress_kernel(DevIndex ix, const uint64_t *__restrict__ vec_id, uint64_t n,
                                  float *__restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kDim) return;
  const uint64_t t = i / kDim;
  const uint32_t d = (uint32_t)(i % kDim);
  const uint64_t v = vec_id[t];
  const uint8_t *res = ix.residual + v * ix.bytes_per_vec;
  const uint32_t vpb = 8u / ix.n_bit;
  const float w = ix.lut[(uint32_t)res[d / vpb] * vpb + d % vpb];
  out[i] = __fadd_rn(ix.centroid[(size_t)ix.vq_code[v] * kDim + d], w);
}

__global__ void unpack_kernel(DevIndex ix, const uint64_t *__restrict__ vec_id, uint64_t n,
                              uint8_t *__restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kDim) return;
  const uint64_t t = i / kDim;
  const uint32_t d = (uint32_t)(i % kDim);
  out[i] = (uint8_t)bucket_of(ix.residual + vec_id[t] * ix.bytes_per_vec, d, ix.n_bit);
}

cudaError_t launch_decompress(const DevIndex &ix, const uint64_t *vec_id, uint64_t n, float *out,
                              cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const uint64_t tot = n * kDim;
  decompress_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(ix, vec_id, n, out);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const DevIndex &ix, const uint64_t *vec_id, uint64_t n, uint8_t *out,
                          cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const uint64_t tot = n * kDim;
  unpack_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(ix, vec_id, n, out);
  return cudaGetLastError();
}

// One thread per packed byte: bucket = #cutoffs <= (vec - centroid) for each
// of its 8/n_bit values, packed MSB-first (compressSQCode semantics).
__global__ void pack_residual_kernel(const float *__restrict__ vec, uint64_t n_vec,
                                     const float *__restrict__ cen, const uint32_t *__restrict__ code,
                                     Cutoffs cut, uint32_t n_bit, uint8_t *__restrict__ out) {
  const uint32_t vpb = 8u / n_bit;
  const uint32_t bpv = kDim / vpb;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_vec * bpv) return;
  const uint64_t v = i / bpv;
  const uint32_t p = (uint32_t)(i % bpv);
  const float *x = vec + v * kDim;
  const float *c = cen + (size_t)code[v] * kDim;
  const uint32_t n_cut = (1u << n_bit) - 1u;
  uint32_t byte = 0;
  for (uint32_t u = 0; u < vpb; u++) {
    const uint32_t d = p * vpb + u;
    const float e = __fsub_rn(x[d], c[d]);
    uint32_t bk = n_cut;
    for (uint32_t k = 0; k < n_cut; k++)
      if (cut.v[k] > e) { bk = k; break; }
    byte = (byte << n_bit) | bk;
  }
  out[i] = (uint8_t)byte;
}

cudaError_t launch_pack_residual(const float *vec, uint64_t n_vec, const float *cen,
                                 const uint32_t *code, const Cutoffs &cut, uint32_t n_bit,
                                 uint8_t *out, cudaStream_t st) {
  const uint64_t tot = n_vec * (kDim / (8u / n_bit));
  if (tot == 0) return cudaSuccess;
  pack_residual_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(vec, n_vec, cen, code, cut, n_bit, out);
  return cudaGetLastError();
}

// sum[code[i]][d] += vec[i][d] in FP64; count[code[i]] += 1.  One warp per
// token, 4 dims per lane.
__global__ void kmeans_accumulate_kernel(const float *__restrict__ vec, uint64_t n_vec,
                                         const uint32_t *__restrict__ code, double *__restrict__ sum,
                                         unsigned long long *__restrict__ count) {
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n_vec) return;
  const uint32_t c = code[w];
  const float4 x = reinterpret_cast<const float4 *>(vec + w * kDim)[lane];
  double *s = sum + (size_t)c * kDim + lane * 4;
  atomicAdd(s + 0, (double)x.x);
  atomicAdd(s + 1, (double)x.y);
  atomicAdd(s + 2, (double)x.z);
  atomicAdd(s + 3, (double)x.w);
  if (lane == 0) atomicAdd(count + c, 1ull);
}

cudaError_t launch_kmeans_accumulate(const float *vec, uint64_t n_vec, const uint32_t *code,
                                     double *sum, uint64_t *count, cudaStream_t st) {
  if (n_vec == 0) return cudaSuccess;
  const uint64_t threads = n_vec * 32;
  kmeans_accumulate_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      vec, n_vec, code, sum, reinterpret_cast<unsigned long long *>(count));
  return cudaGetLastError();
}

// Order statistics of the residual errors e = vec[i][d] - centroid[code[i]][d]
// (one rounded FP32 subtraction, as the codec computes them), without
// materialising them: e is mapped to a 32-bit key whose unsigned order is
// the float order; pass 1 counts the keys' high 16 bits, pass 2 the low 16
// bits of the keys inside the high-half bins that hold a wanted rank.
__device__ __forceinline__ uint32_t order_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void residual_hist_hi_kernel(const float *__restrict__ vec, uint64_t n_vec,
                                        const float *__restrict__ cen,
                                        const uint32_t *__restrict__ code,
                                        unsigned long long *__restrict__ hist) {
  const uint64_t n = n_vec * kDim;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = i / kDim;
    const uint32_t d = (uint32_t)(i % kDim);
    const float e = __fsub_rn(vec[i], cen[(size_t)code[v] * kDim + d]);
    atomicAdd(hist + (order_key(e) >> 16), 1ull);
  }
}

// slot_of[hi] = index of the wanted high half hi among the pass-2 histograms
// (-1: none); hist2[slot][lo]
__global__ void residual_hist_lo_kernel(const float *__restrict__ vec, uint64_t n_vec,
                                        const float *__restrict__ cen,
                                        const uint32_t *__restrict__ code,
                                        const int *__restrict__ slot_of,
                                        unsigned long long *__restrict__ hist2) {
  const uint64_t n = n_vec * kDim;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = i / kDim;
    const uint32_t d = (uint32_t)(i % kDim);
    const uint32_t k = order_key(__fsub_rn(vec[i], cen[(size_t)code[v] * kDim + d]));
    const int sl = slot_of[k >> 16];
    if (sl >= 0) atomicAdd(hist2 + (size_t)sl * 65536u + (k & 0xffffu), 1ull);
  }
}

cudaError_t residual_select(const float *vec, uint64_t n_vec, const float *cen,
                            const uint32_t *code, const uint64_t *rank, uint32_t n_rank,
                            float *out, cudaStream_t st) {
  if (n_rank == 0) return cudaSuccess;
  const uint64_t n = n_vec * kDim;
  for (uint32_t r = 0; r < n_rank; r++)
    if (rank[r] >= n) return cudaErrorInvalidValue;
  unsigned long long *hist = nullptr, *hist2 = nullptr;
  int *slot_of = nullptr;
  cudaError_t e = cudaMalloc(&hist, 65536 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&slot_of, 65536 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&hist2, (size_t)n_rank * 65536 * sizeof(unsigned long long));
  std::vector<unsigned long long> h(65536), h2;
  std::vector<uint32_t> hi_of(n_rank);
  std::vector<uint64_t> below(n_rank);  // keys in lower high-half bins
  std::vector<int> slot(65536, -1);
  std::vector<uint32_t> wanted;  // distinct high halves, in slot order
  const unsigned grid = 148u * 8u;
  if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, 65536 * sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    residual_hist_hi_kernel<<<grid, 256, 0, st>>>(vec, n_vec, cen, code, hist);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), hist, 65536 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    for (uint32_t r = 0; r < n_rank; r++) {
      uint64_t acc = 0;
      uint32_t b = 0;
      while (acc + h[b] <= rank[r]) acc += h[b++];
      hi_of[r] = b;
      below[r] = acc;
      if (slot[b] < 0) {
        slot[b] = (int)wanted.size();
        wanted.push_back(b);
      }
    }
    e = cudaMemcpyAsync(slot_of, slot.data(), 65536 * sizeof(int), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess)
    e = cudaMemsetAsync(hist2, 0, wanted.size() * 65536 * sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    residual_hist_lo_kernel<<<grid, 256, 0, st>>>(vec, n_vec, cen, code, slot_of, hist2);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    h2.resize(wanted.size() * 65536);
    e = cudaMemcpyAsync(h2.data(), hist2, h2.size() * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    for (uint32_t r = 0; r < n_rank; r++) {
      const unsigned long long *g = h2.data() + (size_t)slot[hi_of[r]] * 65536;
      uint64_t acc = below[r];
      uint32_t lo = 0;
      while (acc + g[lo] <= rank[r]) acc += g[lo++];
      const uint32_t k = (hi_of[r] << 16) | lo;
      const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
      float f;
      std::memcpy(&f, &u, 4);
      out[r] = f;
    }
  }
  cudaFree(hist);
  cudaFree(slot_of);
  cudaFree(hist2);
  return e;
}

}  // namespace mvr
