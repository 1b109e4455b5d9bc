// mvr_prune.cu -- training of the learned candidate pruner's MLP
// (33 -> 256 -> 256 -> 1, GELU) on CUDA cores: FP32 activations and
// accumulation with the weights rounded to BF16 as the inference kernel
// applies them, mean-squared-error loss, backward pass and Adam, all
// hand-written kernels.  The pruner has no counterpart in the reference.
#include "mvr_prune.cuh"

#include <cuda_bf16.h>

namespace mvr {

namespace {

constexpr int kGT = 64;      // GEMM output tile (rows and columns)
constexpr int kGK = 16;      // GEMM K step
constexpr int kGThreads = 256;

__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608f * (1.0f + 0.134145f * x * x);
}

// C[M][N] = op(A) op(B) (+ bias[N] when bias is set), row-major storage:
// op(A) is [M][K] (A stored [M][K], or [K][M] when TA), op(B) is [K][N]
// (B stored [K][N], or [N][K] when TB).  64 x 64 output tiles, K in steps
// of 16 through shared memory, 4 x 4 outputs per thread; out-of-range
// elements read as 0.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kGThreads)
gemm_kernel(const float *__restrict__ A, const float *__restrict__ B, float *__restrict__ C,
            const float *__restrict__ bias, int M, int N, int K) {
  __shared__ float As[kGK][kGT + 4];
  __shared__ float Bs[kGK][kGT + 4];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  const int tr = tid / 16, tc = tid % 16;  // 16 x 16 threads, 4 x 4 outputs each
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kGK) {
    for (int i = tid; i < kGK * kGT; i += kGThreads) {
      const int kk = i / kGT, mm = i % kGT;
      const int m = m0 + mm, k = k0 + kk;
      float a = 0.0f;
      if (m < M && k < K) a = TA ? A[(size_t)k * M + m] : A[(size_t)m * K + k];
      As[kk][mm] = a;
      const int n = n0 + mm;
      float b = 0.0f;
      if (n < N && k < K) b = TB ? B[(size_t)n * K + k] : B[(size_t)k * N + n];
      Bs[kk][mm] = b;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        a[u] = As[kk][tr * 4 + u];
        b[u] = Bs[kk][tc * 4 + u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int m = m0 + tr * 4 + u;
    if (m >= M) continue;
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int n = n0 + tc * 4 + v;
      if (n < N) C[(size_t)m * N + n] = acc[u][v] + (bias ? bias[n] : 0.0f);
    }
  }
}

template <bool TA, bool TB>
cudaError_t gemm(const float *A, const float *B, float *C, const float *bias, int M, int N, int K,
                 cudaStream_t st) {
  const dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT);
  gemm_kernel<TA, TB><<<grid, kGThreads, 0, st>>>(A, B, C, bias, M, N, K);
  return cudaGetLastError();
}

__global__ void round_bf16_kernel(const float *__restrict__ in, float *__restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = bf16r(in[i]);
}

// h = GELU(z), rounded to BF16 (the next layer's operand precision)
__global__ void gelu_fwd_kernel(const float *__restrict__ z, float *__restrict__ h, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    h[i] = bf16r(gelu(z[i]));
}

// yhat[r] = h2[r] . w3 + b3; with y: loss += 0.5 (yhat - y)^2 / n and
// dy = (yhat - y) / n
__global__ void head_kernel(const float *__restrict__ h2, const float *__restrict__ w3,
                            const float *__restrict__ b3, const float *__restrict__ y,
                            uint32_t n, float *__restrict__ yhat, float *__restrict__ dy,
                            float *__restrict__ loss) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const float *row = h2 + (size_t)warp * kHid;
  float s = 0.0f;
  for (int j = lane; j < kHid; j += 32) s = fmaf(row[j], w3[j], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const float v = s + b3[0];
    yhat[warp] = v;
    if (y) {
      const float e = v - y[warp];
      dy[warp] = e / (float)n;
      atomicAdd(loss, 0.5f * e * e / (float)n);
    }
  }
}

// dz = (dh, or dy (x) w3 when dh is null) * GELU'(z)
__global__ void gelu_bwd_kernel(const float *__restrict__ z, const float *__restrict__ dh,
                                const float *__restrict__ dy, const float *__restrict__ w3,
                                float *__restrict__ dz, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float g = dh ? dh[i] : dy[i / kHid] * w3[i % kHid];
    dz[i] = g * gelu_grad(z[i]);
  }
}

// out[c] += sum over rows r of m[r][c] (times wvec[r] when wvec is set)
__global__ void colsum_kernel(const float *__restrict__ m, const float *__restrict__ wvec,
                              uint32_t rows, uint32_t cols, float *__restrict__ out) {
  const uint32_t c = threadIdx.x;  // blockDim.x == cols (<= 1024)
  float s = 0.0f;
  for (uint32_t r = blockIdx.x; r < rows; r += gridDim.x)
    s += m[(size_t)r * cols + c] * (wvec ? wvec[r] : 1.0f);
  atomicAdd(out + c, s);
}

__global__ void sum_kernel(const float *__restrict__ v, uint32_t n, float *__restrict__ out) {
  float s = 0.0f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void adam_kernel(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ g, uint32_t n, float lr, float c1,
                            float c2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  }
}

struct MlpWork {
  float *z1, *h1, *z2, *h2, *yhat, *dy, *pr, *grad;
  MlpWork(float *w, uint32_t n) {
    z1 = w;
    h1 = z1 + (size_t)n * kHid;
    z2 = h1 + (size_t)n * kHid;
    h2 = z2 + (size_t)n * kHid;
    yhat = h2 + (size_t)n * kHid;
    dy = yhat + n;
    pr = dy + n + ((16 - (n * 2) % 16) % 16);
    grad = pr + kNumParams;
  }
};

cudaError_t forward(const float *x, uint32_t n, const float *params, const MlpWork &w,
                    const float *y, float *loss, cudaStream_t st) {
  round_bf16_kernel<<<148, 256, 0, st>>>(params, w.pr, kNumParams);
  cudaError_t e;
  if ((e = gemm<false, true>(x, w.pr + kOffW1, w.z1, params + kOffB1, n, kHid, kFeat, st)))
    return e;
  gelu_fwd_kernel<<<592, 256, 0, st>>>(w.z1, w.h1, (size_t)n * kHid);
  if ((e = gemm<false, true>(w.h1, w.pr + kOffW2, w.z2, params + kOffB2, n, kHid, kHid, st)))
    return e;
  gelu_fwd_kernel<<<592, 256, 0, st>>>(w.z2, w.h2, (size_t)n * kHid);
  head_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(w.h2, w.pr + kOffW3, params + kOffB3, y, n,
                                                    w.yhat, w.dy, loss);
  return cudaGetLastError();
}

}  // namespace

cudaError_t mlp_forward_ref(const float *x, uint32_t n, const float *params, float *work,
                            float *out, cudaStream_t st) {
  MlpWork w(work, n);
  cudaError_t e = forward(x, n, params, w, nullptr, nullptr, st);
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(out, w.yhat, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

cudaError_t mlp_train_step(const float *x, const float *y, uint32_t n, float *params,
                           float *adam_m, float *adam_v, float *work, float lr, uint32_t step,
                           float *loss_out, cudaStream_t st) {
  if (n == 0 || step == 0) return cudaErrorInvalidValue;
  MlpWork w(work, n);
  float *loss = w.grad + kNumParams;  // one float past the gradient
  cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(float), st);
  if (e != cudaSuccess) return e;
  if ((e = forward(x, n, params, w, y, loss, st))) return e;
  if (loss_out && (e = cudaMemcpyAsync(loss_out, loss, sizeof(float), cudaMemcpyDeviceToDevice, st)))
    return e;
  if ((e = cudaMemsetAsync(w.grad, 0, kNumParams * sizeof(float), st))) return e;
  const size_t nh = (size_t)n * kHid;
  // head: db3 = sum dy, dw3 = h2^T dy
  sum_kernel<<<64, 256, 0, st>>>(w.dy, n, w.grad + kOffB3);
  colsum_kernel<<<256, kHid, 0, st>>>(w.h2, w.dy, n, kHid, w.grad + kOffW3);
  // layer 2: dz2 = (dy w3^T) * GELU'(z2) (into h2, no longer needed)
  float *dz2 = w.h2;
  gelu_bwd_kernel<<<592, 256, 0, st>>>(w.z2, nullptr, w.dy, w.pr + kOffW3, dz2, nh);
  if ((e = gemm<true, false>(dz2, w.h1, w.grad + kOffW2, nullptr, kHid, kHid, n, st))) return e;
  colsum_kernel<<<256, kHid, 0, st>>>(dz2, nullptr, n, kHid, w.grad + kOffB2);
  // layer 1: dh1 = dz2 W2 (into z2), dz1 = dh1 * GELU'(z1) (into h1)
  float *dh1 = w.z2, *dz1 = w.h1;
  if ((e = gemm<false, false>(dz2, w.pr + kOffW2, dh1, nullptr, n, kHid, kHid, st))) return e;
  gelu_bwd_kernel<<<592, 256, 0, st>>>(w.z1, dh1, nullptr, nullptr, dz1, nh);
  if ((e = gemm<true, false>(dz1, x, w.grad + kOffW1, nullptr, kHid, kFeat, n, st))) return e;
  colsum_kernel<<<256, kHid, 0, st>>>(dz1, nullptr, n, kHid, w.grad + kOffB1);
  const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
  adam_kernel<<<148, 256, 0, st>>>(params, adam_m, adam_v, w.grad, kNumParams, lr, c1, c2);
  return cudaGetLastError();
}

}  // namespace mvr
