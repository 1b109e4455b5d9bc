// ref_gpu.cu -- runs the reference's own GPU search kernels, compiled
// unmodified from its headers where they lie (oracle/Makefile, target
// `ref`), on small cases, so that the oracle and the CUDA path can be
// pinned to reference output for the search stages.  Test infrastructure
// only (tests/golden/make_ref_gpu_golden.py calls it on a GPU and freezes
// what it returns as fixtures); nothing in the product links it.
//
// Reference code that runs here (src/include/...):
//   alg/igp_gpu_pp/DataStructPP.hpp   ItemVecInfoPP / VQInfoPP / IVFInfoPP /
//                                     SQInfoPP: device uploads and the
//                                     byte -> weights decode table
//   alg/MatrixMulCUBLAS.hpp:33-61     MatrixMultiply (cuBLAS SGEMM)
//   alg/igp_gpu_pp/FilterPP.hpp:19-142  gather_ivf_data, find_candidate_item,
//                                     max_qvec_doc_score
//   alg/igp_gpu_pp/RerankPP.hpp:16-161  gather_vq_data,
//                                     decompressAndAddResidual, reduceMax
// The host orchestration between those kernels (thrust sort / unique /
// lower_bound / exclusive_scan / transform / copy_if, launch shapes, the
// residual gather of RerankPP::transmitSQCode) is restated from
// FilterPP::filter (FilterPP.hpp:267-361) and RerankPP::compute
// (RerankPP.hpp:368-441), whose classes hold RAFT handles and so are not
// instantiated.  RAFT's select_k and row reduce are not run: the probe
// selection is a (score desc, id asc) sort here, and the sums over query
// tokens are left to the caller.  RAFT's float atomicMax is replaced by the
// project-written compare-and-swap loop in ref_stub/raft/util.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include <cublas_v2.h>
#include "spdlog/spdlog.h"
#include "include/util/CUDAUtil.hpp"
#include "include/alg/MatrixMulCUBLAS.hpp"
#include "include/alg/igp_gpu_pp/DataStructPP.hpp"
#include "include/alg/igp_gpu_pp/FilterPP.hpp"
#include "include/alg/igp_gpu_pp/RerankPP.hpp"

using namespace VectorSetSearch;

namespace {

// returns a nonzero status instead of exiting, for the checks made here
#define RG_TRY(call)                                                        \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      fprintf(stderr, "ref_gpu: %s at %s:%d\n", cudaGetErrorString(e_),    \
              __FILE__, __LINE__);                                          \
      return 2;                                                             \
    }                                                                       \
  } while (0)

template <class T>
struct DevBuf {
  T *p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, (n ? n : 1) * sizeof(T)); }
};

}  // namespace

extern "C" {

// S[q][c] = dot(query q, centroid c) + 1: MatrixMultiply as
// GenerateVQScoreCandidatePP::generateCandidate calls it
// (GenerateVQScoreCandidatePP.hpp:134-146), then the +1 pass.
int ref_centroid_scores(const float *query, uint32_t nq, const float *centroid,
                        uint32_t n_centroid, uint32_t dim, float *out) {
  if (!nq || !n_centroid || !dim) return 1;
  DevBuf<float> q, c, s;
  RG_TRY(q.alloc((size_t)nq * dim));
  RG_TRY(c.alloc((size_t)n_centroid * dim));
  RG_TRY(s.alloc((size_t)nq * n_centroid));
  RG_TRY(cudaMemcpy(q.p, query, (size_t)nq * dim * 4, cudaMemcpyHostToDevice));
  RG_TRY(cudaMemcpy(c.p, centroid, (size_t)n_centroid * dim * 4, cudaMemcpyHostToDevice));
  cublasHandle_t h;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return 3;
  MatrixMultiply(h, q.p, c.p, nq, n_centroid, dim, s.p);
  RG_TRY(cudaDeviceSynchronize());
  cublasDestroy(h);
  float *sp = s.p;
  thrust::for_each(thrust::device, sp, sp + (size_t)nq * n_centroid,
                   [] __device__(float &x) { x += 1.0f; });
  RG_TRY(cudaDeviceSynchronize());
  RG_TRY(cudaMemcpy(out, s.p, (size_t)nq * n_centroid * 4, cudaMemcpyDeviceToHost));
  return 0;
}

// The PP candidate filter for one query from its probe lists
// (probe_id / probe_score [nq * nprobe], token-major): the candidate docs in
// ascending id order (out_cand [n_item], count in *out_n_cand) and, for each
// candidate c and query token t, the max over t's probes whose IVF list holds
// c of the probe score, 0 if none (out_qmax [n_item * nq], row c of the
// candidate order) -- qvec_max_score_l_gpu_ of FilterPP::filter.
int ref_filter(uint32_t n_item, uint32_t n_centroid, const uint64_t *ivf_off,
               const uint32_t *ivf_size, const uint32_t *ivf_ids, uint64_t n_ele,
               const uint32_t *probe_id, const float *probe_score, uint32_t nq,
               uint32_t nprobe, uint32_t *out_cand, uint32_t *out_n_cand, float *out_qmax) {
  if (!n_item || !n_centroid || !nq || !nprobe) return 1;
  const uint32_t n_probe = nq * nprobe;
  for (uint32_t i = 0; i < n_probe; i++)
    if (probe_id[i] >= n_centroid) return 1;
  std::vector<size_t> off(ivf_off, ivf_off + n_centroid);
  for (uint32_t c = 0; c < n_centroid; c++)
    if (off[c] + ivf_size[c] > n_ele) return 1;
  for (uint64_t e = 0; e < n_ele; e++)
    if (ivf_ids[e] >= n_item) return 1;
  IVFInfoPP ivf(n_centroid, n_ele, off.data(), ivf_size, ivf_ids);
  const uint32_t max_ele = ivf.max_n_ele_ivf_;
  // find_candidate_item / max_qvec_doc_score run ceil(max_ele / 32) threads
  // per block: 1..1024 for lists of 1..32768 entries
  if (max_ele == 0 || max_ele > 32768) return 1;

  DevBuf<uint32_t> fid, uniq, f2u, u_n, u_items, need, cand_cache, item2cand, seq, cand;
  DevBuf<float> fsc, qmax;
  RG_TRY(fid.alloc(n_probe));
  RG_TRY(fsc.alloc(n_probe));
  RG_TRY(uniq.alloc(n_probe));
  RG_TRY(f2u.alloc(n_probe));
  RG_TRY(u_n.alloc(n_probe));
  RG_TRY(u_items.alloc((size_t)n_probe * max_ele));
  RG_TRY(need.alloc(n_item));
  RG_TRY(cand_cache.alloc(n_item));
  RG_TRY(item2cand.alloc(n_item));
  RG_TRY(seq.alloc(n_item));
  RG_TRY(cand.alloc(n_item));
  RG_TRY(qmax.alloc((size_t)n_item * nq));
  RG_TRY(cudaMemcpy(fid.p, probe_id, n_probe * 4, cudaMemcpyHostToDevice));
  RG_TRY(cudaMemcpy(fsc.p, probe_score, n_probe * 4, cudaMemcpyHostToDevice));
  // FilterPP::reset (FilterPP.hpp:255-264)
  RG_TRY(cudaMemset(qmax.p, 0, (size_t)n_item * nq * 4));
  RG_TRY(cudaMemset(need.p, 0, (size_t)n_item * 4));
  thrust::sequence(thrust::device, seq.p, seq.p + n_item, 0u);

  // unique probed centroids and the probe -> unique map (FilterPP.hpp:281-290)
  RG_TRY(cudaMemcpy(uniq.p, fid.p, n_probe * 4, cudaMemcpyDeviceToDevice));
  thrust::sort(thrust::device, uniq.p, uniq.p + n_probe);
  uint32_t *uend = thrust::unique(thrust::device, uniq.p, uniq.p + n_probe);
  const uint32_t n_unique = (uint32_t)(uend - uniq.p);
  thrust::lower_bound(thrust::device, uniq.p, uniq.p + n_unique, fid.p, fid.p + n_probe, f2u.p);
  gather_ivf_data<<<n_unique, 256>>>(uniq.p, ivf.ivf_offset_l_gpu_, ivf.ivf_size_l_gpu_,
                                    ivf.ivf_gpu_, n_unique, max_ele, u_items.p, u_n.p);
  RG_TRY(cudaGetLastError());
  const uint32_t ivf_n_thread = (max_ele + 31) / 32;
  find_candidate_item<<<n_unique, ivf_n_thread>>>(u_n.p, u_items.p, max_ele, n_unique,
                                                  ivf_n_thread, need.p);
  RG_TRY(cudaGetLastError());
  // item -> (candidate rank + 1), 0 for non-candidates (FilterPP.hpp:318-336)
  thrust::exclusive_scan(thrust::device, need.p, need.p + n_item, cand_cache.p);
  thrust::transform(thrust::device, need.p, need.p + n_item, cand_cache.p, item2cand.p,
                    [] __device__(uint32_t flag, uint32_t prefix) -> uint32_t {
                      return flag ? prefix + 1 : 0;
                    });
  max_qvec_doc_score<<<n_probe, ivf_n_thread>>>(fid.p, fsc.p, uniq.p, f2u.p, u_n.p, u_items.p,
                                                item2cand.p, max_ele, nq, nprobe, ivf_n_thread,
                                                qmax.p);
  RG_TRY(cudaGetLastError());
  // ascending candidate list (FilterPP.hpp:348-359)
  uint32_t *need_p = need.p;
  uint32_t *cend = thrust::copy_if(thrust::device, seq.p, seq.p + n_item, cand.p,
                                   [need_p] __device__(uint32_t i) { return need_p[i] == 1u; });
  RG_TRY(cudaDeviceSynchronize());
  const uint32_t n_cand = (uint32_t)(cend - cand.p);
  *out_n_cand = n_cand;
  RG_TRY(cudaMemcpy(out_cand, cand.p, (size_t)n_cand * 4, cudaMemcpyDeviceToHost));
  RG_TRY(cudaMemcpy(out_qmax, qmax.p, (size_t)n_cand * nq * 4, cudaMemcpyDeviceToHost));
  ivf.FinishCompute();
  return 0;
}

// The PP rerank of one query's shortlist (short_id [P], doc ids): the
// decompressed doc tokens in shortlist order (out_vec [sum of their lengths
// * dim], nullable) and, for each query token t and shortlisted doc c, the
// max over c's tokens of the cuBLAS dot q_t . x (out_max [nq * P], row t) --
// max_score_l_gpu_ of RerankPP::compute.  nq * P must be a multiple of 256
// (reduceMax's blocks of 256 then have no idle threads).
int ref_rerank(uint32_t n_item, const uint32_t *item_n_vec, const uint64_t *item_off,
               uint64_t n_vec, const float *centroid, uint32_t n_centroid, uint32_t dim,
               const uint32_t *vq_code, const uint8_t *residual, const float *weight,
               uint32_t n_bit, const float *query, uint32_t nq, const uint32_t *short_id,
               uint32_t P, float *out_vec, float *out_max) {
  if (!n_item || !nq || !P || !dim || ((uint64_t)nq * P) % 256 != 0) return 1;
  if (n_bit != 1 && n_bit != 2 && n_bit != 4 && n_bit != 8) return 1;
  for (uint32_t i = 0; i < P; i++)
    if (short_id[i] >= n_item) return 1;
  for (uint64_t v = 0; v < n_vec; v++)
    if (vq_code[v] >= n_centroid) return 1;
  const uint32_t vpb = 8 / n_bit, bpv = dim / vpb;
  std::vector<size_t> off(item_off, item_off + n_item);
  uint32_t max_len = 0;
  for (uint32_t i = 0; i < n_item; i++) max_len = std::max(max_len, item_n_vec[i]);
  ItemVecInfoPP items(n_item, max_len, 0, dim, n_vec, item_n_vec, off.data());
  VQInfoPP vq(n_centroid, dim, n_vec, centroid, vq_code);
  SQInfoPP sq(n_vec, dim, n_bit, vpb, bpv, 1u << n_bit, weight, residual);

  // residual bytes of the shortlist, stacked in shortlist order
  // (RerankPP::transmitSQCode, RerankPP.hpp:289-365)
  std::vector<uint32_t> len(P);
  uint64_t n_rr = 0;
  for (uint32_t i = 0; i < P; i++) { len[i] = item_n_vec[short_id[i]]; n_rr += len[i]; }
  if (n_rr == 0 || n_rr >= (1ull << 31)) return 1;
  std::vector<uint8_t> stacked(n_rr * bpv);
  uint64_t pos = 0;
  for (uint32_t i = 0; i < P; i++) {
    memcpy(stacked.data() + pos * bpv, residual + off[short_id[i]] * bpv, (size_t)len[i] * bpv);
    pos += len[i];
  }
  const uint32_t n_rerank_vec = (uint32_t)n_rr;

  DevBuf<uint32_t> ids, glen, goff, gcode;
  DevBuf<uint8_t> sqc;
  DevBuf<float> q, vec, table, mx;
  RG_TRY(ids.alloc(P));
  RG_TRY(glen.alloc(P));
  RG_TRY(goff.alloc(P));
  RG_TRY(gcode.alloc(n_rerank_vec));
  RG_TRY(sqc.alloc((size_t)n_rerank_vec * bpv));
  RG_TRY(q.alloc((size_t)nq * dim));
  RG_TRY(vec.alloc((size_t)n_rerank_vec * dim));
  RG_TRY(table.alloc((size_t)nq * n_rerank_vec));
  RG_TRY(mx.alloc((size_t)nq * P));
  RG_TRY(cudaMemcpy(ids.p, short_id, P * 4, cudaMemcpyHostToDevice));
  RG_TRY(cudaMemcpy(glen.p, len.data(), P * 4, cudaMemcpyHostToDevice));
  RG_TRY(cudaMemcpy(sqc.p, stacked.data(), stacked.size(), cudaMemcpyHostToDevice));
  RG_TRY(cudaMemcpy(q.p, query, (size_t)nq * dim * 4, cudaMemcpyHostToDevice));
  RG_TRY(cudaMemset(vec.p, 0, (size_t)n_rerank_vec * dim * 4));
  RG_TRY(cudaMemset(table.p, 0, (size_t)nq * n_rerank_vec * 4));

  // RerankPP::compute (RerankPP.hpp:368-441): offsets, code gather,
  // decompression, the query x token GEMM, max over each doc's tokens
  thrust::exclusive_scan(thrust::device, glen.p, glen.p + P, goff.p);
  gather_vq_data<<<P, 16>>>(ids.p, items.item_n_vec_l_gpu_, items.item_n_vec_offset_l_gpu_,
                            vq.vq_code_l_gpu_, glen.p, goff.p, P, gcode.p);
  RG_TRY(cudaGetLastError());
  const uint32_t per_vec = 16, block = 1024;
  const uint32_t grid = (uint32_t)(((uint64_t)n_rerank_vec * per_vec + block - 1) / block);
  decompressAndAddResidual<<<grid, block, SQInfoPP::pack_code_range_ * vpb * sizeof(float)>>>(
      gcode.p, sqc.p, vq.centroid_l_gpu_, sq.pack_code2weight_l_gpu_, n_rerank_vec, per_vec, dim,
      bpv, SQInfoPP::pack_code_range_, vpb, vec.p);
  RG_TRY(cudaGetLastError());
  cublasHandle_t h;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return 3;
  MatrixMultiply(h, q.p, vec.p, nq, n_rerank_vec, dim, table.p);
  RG_TRY(cudaDeviceSynchronize());
  cublasDestroy(h);
  const uint64_t tasks = (uint64_t)nq * P;
  reduceMax<<<(uint32_t)(tasks / 256), 256, 256 * sizeof(float)>>>(table.p, glen.p, goff.p, nq, P,
                                                                   n_rerank_vec, 1, mx.p);
  RG_TRY(cudaGetLastError());
  RG_TRY(cudaDeviceSynchronize());
  if (out_vec)
    RG_TRY(cudaMemcpy(out_vec, vec.p, (size_t)n_rerank_vec * dim * 4, cudaMemcpyDeviceToHost));
  RG_TRY(cudaMemcpy(out_max, mx.p, (size_t)nq * P * 4, cudaMemcpyDeviceToHost));
  sq.FinishCompute();
  cudaFree(sq.pack_code2weight_l_gpu_);
  vq.FinishCompute();
  cudaFree(items.item_n_vec_l_gpu_);
  cudaFree(items.item_n_vec_offset_l_gpu_);
  return 0;
}

}  // extern "C"
