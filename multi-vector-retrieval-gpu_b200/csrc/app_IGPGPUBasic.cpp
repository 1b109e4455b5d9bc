// IGPGPUBasic executable: same argv, inputs and output files as the
// reference's src/app/IGPGPUBasic.cpp:81-206, served by libmvr with the
// padded-rerank ("basic") semantics.
#include <cstdio>
#include <fstream>
#include <iostream>

#include "app_common.hpp"
#include "igp_method.hpp"

int main(int argc, char **argv) {
  using namespace mvr;
  app::Args a;
  if (!a.parse(argc, argv, {"username", "dataset", "method-name", "num-centroid", "num-bit",
                            "topk", "nprobe", "probe_topk", "is_profile"})) {
    std::cerr << "Error parsing command line\n";
    return 1;
  }
  const std::string username = a.s("username"), dataset = a.s("dataset"),
                    method_name = a.s("method-name");
  const uint32_t n_centroid = a.u("num-centroid"), n_bit = a.u("num-bit");
  const uint32_t topk = a.u("topk"), nprobe = a.u("nprobe"), probe_topk = a.u("probe_topk");
  const bool is_profile = a.b("is_profile");
  char suffix[256];
  std::snprintf(suffix, sizeof(suffix), "n_centroid_%u-n_bit_%u", n_centroid, n_bit);
  auto fm = app::filename_map(username, dataset, method_name, suffix);

  Method::IGPGPUBasic index(fm["item_n_vec_l"]);
  if (!index.buildIndex(fm["centroid_l"], fm["vq_code_l"], fm["ivf_index"], fm["weight_l"],
                        fm["residual_code_l"], n_centroid, n_bit)) {
    std::cerr << "buildIndex failed: " << index.last_error() << "\n";
    return 1;
  }
  NpyArray q;
  uint32_t n_query = 0, query_n_vec = 0;
  if (!app::load_queries(fm["query_l"], q, n_query, query_n_vec)) return 1;
  Method::IGPGPUBasicResult r;
  try {
    r = index.search(reinterpret_cast<const float *>(q.data.data()), n_query, query_n_vec, topk,
                     nprobe, probe_topk);
  } catch (const std::exception &e) {
    std::cerr << "search failed: " << e.what() << "\n";
    return 1;
  }
  std::vector<uint32_t> qid;
  if (!app::read_query_ids(fm["query_id"], qid) || qid.size() != n_query) {
    std::cerr << "Error: Could not read " << n_query << " query ids from " << fm["query_id"] << "\n";
    return 1;
  }
  char rsuffix[256];
  std::snprintf(rsuffix, sizeof(rsuffix), "nprobe_%d-probe_topk_%d", nprobe, probe_topk);
  const std::string prof = is_profile ? "-profile" : "";
  const std::string ans = fm["answer_path"] + "/" + dataset + "-" + method_name + "-top" +
                          std::to_string(topk) + "-" + suffix + "-" + rsuffix + prof + ".tsv";
  std::ofstream out(ans);
  for (uint32_t i = 0; i < n_query; i++)
    for (uint32_t k = 0; k < topk; k++)
      out << qid[i] << "\t" << r.result_ID_l[(size_t)i * topk + k] << "\t" << k + 1 << "\t"
          << r.result_score_l[(size_t)i * topk + k] << std::endl;
  const std::string perf = fm["answer_path"] + "/" + dataset + "-" + method_name +
                           "-performance-top" + std::to_string(topk) + "-" + suffix + "-" +
                           rsuffix + prof + ".tsv";
  std::ofstream po(perf);
  po << "search_time\treset_time\ttransmit_query_time\tcand_gen_time\tfilter_time\t"
        "filter_transmit_time\tfilter_compute_time\trerank_time\trerank_transmit_time\t"
        "rerank_compute_time"
     << std::endl;
  for (uint32_t i = 0; i < n_query; i++)
    po << r.compute_time_l[i] << "\t" << r.reset_time_l[i] << "\t" << r.transmit_query_time_l[i]
       << "\t" << r.cand_gen_time_l[i] << "\t" << r.filter_time_l[i] << "\t"
       << r.filter_transmit_time_l[i] << "\t" << r.filter_compute_time_l[i] << "\t"
       << r.rerank_time_l[i] << "\t" << r.rerank_transmit_time_l[i] << "\t"
       << r.rerank_compute_time_l[i] << std::endl;
  return 0;
}
