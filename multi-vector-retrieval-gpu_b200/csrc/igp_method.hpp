// igp_method.hpp -- C++ mirror of the reference's method facades
// IGPGPUBasic (src/impl/IGPGPUBasic.hpp:17-313) and IGPGPUPP
// (src/impl/IGPGPUPP.hpp:17-335): same constructors, buildIndex(...) and
// search(...) signatures and result structs, implemented over the libmvr
// C ABI.  Differences in behaviour:
//   - errors raise std::invalid_argument / std::runtime_error (or make
//     buildIndex return false) instead of calling exit();
//   - the index stays usable after search() (the reference frees it);
//   - n_cpu_thread is accepted and ignored: queries run in device batches.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

struct mvr_index;

namespace mvr::Method {

struct IGPGPUBasicResult {
  std::vector<float> result_score_l;     // n_query * topk
  std::vector<uint32_t> result_ID_l;     // n_query * topk
  std::vector<double> compute_time_l;    // n_query
  std::vector<double> reset_time_l;
  std::vector<double> transmit_query_time_l;
  std::vector<double> cand_gen_time_l;
  std::vector<double> filter_time_l;
  std::vector<double> filter_transmit_time_l;
  std::vector<double> filter_compute_time_l;
  std::vector<double> rerank_time_l;
  std::vector<double> rerank_transmit_time_l;
  std::vector<double> rerank_compute_time_l;
  uint32_t n_query = 0, topk = 0;
};

struct IGPGPUPPResult {
  std::vector<float> result_score_l;   // n_query * topk
  std::vector<uint32_t> result_ID_l;   // n_query * topk
  std::vector<double> compute_time_l;  // n_query
  double batch_query_time = 0;
  uint32_t n_query = 0, topk = 0;
};

class IndexBase {
 public:
  explicit IndexBase(const std::string &item_n_vec_l_fname, int device = 0);
  virtual ~IndexBase();
  IndexBase(const IndexBase &) = delete;
  IndexBase &operator=(const IndexBase &) = delete;
  bool buildIndex(const std::string &centroid_l_fname, const std::string &vq_code_l_fname,
                  const std::string &ivf_index_fname, const std::string &weight_l_fname,
                  const std::string &residual_code_l_fname, uint32_t n_centroid, uint32_t n_bit);
  const std::string &last_error() const { return err_; }
  uint32_t vec_dim() const { return 128; }
  mvr_index *handle() const { return h_; }

 protected:
  void run(const float *query_l, uint32_t n_query, uint32_t query_n_vec, uint32_t topk,
           uint32_t nprobe, uint32_t probe_topk, uint32_t flags, std::vector<float> &score,
           std::vector<uint32_t> &id, std::vector<double> &qtime, std::vector<double> *stage,
           double *wall_s);
  std::string item_n_vec_l_fname_;
  int device_;
  mvr_index *h_ = nullptr;
  std::string err_;
};

class IGPGPUBasic : public IndexBase {
 public:
  explicit IGPGPUBasic(const std::string &item_n_vec_l_fname, int device = 0)
      : IndexBase(item_n_vec_l_fname, device) {}
  IGPGPUBasicResult search(const float *query_l, uint32_t n_query, uint32_t query_n_vec,
                           uint32_t topk, uint32_t nprobe, uint32_t probe_topk);
};

class IGPGPUPP : public IndexBase {
 public:
  IGPGPUPP(const std::string &item_n_vec_l_fname, uint32_t n_cpu_thread, int device = 0)
      : IndexBase(item_n_vec_l_fname, device), n_cpu_thread_(n_cpu_thread) {}
  IGPGPUPPResult search(const float *query_l, uint32_t n_query, uint32_t query_n_vec,
                        uint32_t topk, uint32_t nprobe, uint32_t probe_topk);

 private:
  uint32_t n_cpu_thread_;
};

}  // namespace mvr::Method
