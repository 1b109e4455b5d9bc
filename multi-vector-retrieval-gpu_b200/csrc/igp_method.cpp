// igp_method.cpp -- see igp_method.hpp.
#include "igp_method.hpp"

#include <algorithm>
#include <stdexcept>

#include "mvr.h"

namespace mvr::Method {

IndexBase::IndexBase(const std::string &item_n_vec_l_fname, int device)
    : item_n_vec_l_fname_(item_n_vec_l_fname), device_(device) {}

IndexBase::~IndexBase() {
  if (h_) mvr_index_free(h_);
}

bool IndexBase::buildIndex(const std::string &centroid_l_fname, const std::string &vq_code_l_fname,
                           const std::string &ivf_index_fname, const std::string &weight_l_fname,
                           const std::string &residual_code_l_fname, uint32_t n_centroid,
                           uint32_t n_bit) {
  if (h_) {
    mvr_index_free(h_);
    h_ = nullptr;
  }
  const int rc = mvr_index_load_files(item_n_vec_l_fname_.c_str(), centroid_l_fname.c_str(),
                                      vq_code_l_fname.c_str(), ivf_index_fname.c_str(),
                                      weight_l_fname.c_str(), residual_code_l_fname.c_str(),
                                      n_centroid, n_bit, device_, &h_);
  if (rc != MVR_OK) {
    err_ = mvr_last_error();
    h_ = nullptr;
    return false;
  }
  return true;
}

void IndexBase::run(const float *query_l, uint32_t n_query, uint32_t query_n_vec, uint32_t topk,
                    uint32_t nprobe, uint32_t probe_topk, uint32_t flags,
                    std::vector<float> &score, std::vector<uint32_t> &id,
                    std::vector<double> &qtime, std::vector<double> *stage, double *wall_s) {
  if (!h_) throw std::runtime_error("search before a successful buildIndex");
  if (probe_topk < topk)
    throw std::invalid_argument(
        "the number of refined topk is smaller than the number of returned topk");
  // warm-up on the first min(n_query, 10) queries (IGPGPUPP.hpp:278-281)
  const uint32_t n_warm = std::min(n_query, 10u);
  if (n_warm) {
    std::vector<float> ws((size_t)n_warm * topk);
    std::vector<uint32_t> wi((size_t)n_warm * topk);
    if (mvr_search(h_, query_l, nullptr, n_warm, query_n_vec, topk, nprobe, probe_topk, flags,
                   ws.data(), wi.data(), nullptr, nullptr) != MVR_OK)
      throw std::invalid_argument(mvr_last_error());
  }
  score.assign((size_t)n_query * topk, 0.f);
  id.assign((size_t)n_query * topk, 0u);
  qtime.assign(n_query, 0.0);
  if (stage) stage->assign((size_t)n_query * 6, 0.0);
  mvr_stats st{};
  if (mvr_search_staged(h_, query_l, nullptr, n_query, query_n_vec, topk, nprobe, probe_topk,
                        flags, score.data(), id.data(), qtime.data(),
                        stage ? stage->data() : nullptr, &st) != MVR_OK)
    throw std::invalid_argument(mvr_last_error());
  if (wall_s) *wall_s = st.wall_s;
}

IGPGPUBasicResult IGPGPUBasic::search(const float *query_l, uint32_t n_query,
                                      uint32_t query_n_vec, uint32_t topk, uint32_t nprobe,
                                      uint32_t probe_topk) {
  IGPGPUBasicResult r;
  std::vector<double> stage;
  run(query_l, n_query, query_n_vec, topk, nprobe, probe_topk, MVR_SEM_BASIC, r.result_score_l,
      r.result_ID_l, r.compute_time_l, &stage, nullptr);
  r.n_query = n_query;
  r.topk = topk;
  r.reset_time_l.assign(n_query, 0.0);  // nothing to reset: scratch is restored in-kernel
  r.transmit_query_time_l.resize(n_query);
  r.cand_gen_time_l.resize(n_query);
  r.filter_time_l.resize(n_query);
  r.filter_transmit_time_l.assign(n_query, 0.0);  // IVF lists are HBM-resident
  r.filter_compute_time_l.resize(n_query);
  r.rerank_time_l.resize(n_query);
  r.rerank_transmit_time_l.resize(n_query);
  r.rerank_compute_time_l.resize(n_query);
  for (uint32_t i = 0; i < n_query; i++) {
    const double *s = stage.data() + (size_t)i * 6;
    r.transmit_query_time_l[i] = s[0];
    r.cand_gen_time_l[i] = s[1];
    r.filter_time_l[i] = s[2];
    r.filter_compute_time_l[i] = s[2];
    r.rerank_compute_time_l[i] = s[3] + s[4];
    r.rerank_transmit_time_l[i] = s[5];
    r.rerank_time_l[i] = s[3] + s[4] + s[5];
  }
  return r;
}

IGPGPUPPResult IGPGPUPP::search(const float *query_l, uint32_t n_query, uint32_t query_n_vec,
                                uint32_t topk, uint32_t nprobe, uint32_t probe_topk) {
  IGPGPUPPResult r;
  run(query_l, n_query, query_n_vec, topk, nprobe, probe_topk, MVR_SEM_PP, r.result_score_l,
      r.result_ID_l, r.compute_time_l, nullptr, &r.batch_query_time);
  r.n_query = n_query;
  r.topk = topk;
  return r;
}

}  // namespace mvr::Method
