// app_common.hpp -- shared argv / file handling of the IGPGPUBasic and
// IGPGPUPP executables, which keep the reference's command line
// (src/app/IGPGPUBasic.cpp:15-30, src/app/IGPGPUPP.cpp:15-30), input layout
// (getFilenameMap, IGPGPUBasic.cpp:32-73) and output files, so the reference's
// evaluation drivers run them unchanged.  The data root defaults to the
// reference's /home/<username>/Dataset/multi-vector-retrieval-GPU; the
// environment variable MVR_DATASET_ROOT replaces the "/home/<username>" part.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "mvr_io.hpp"

namespace mvr::app {

struct Args {
  std::map<std::string, std::string> kv;
  bool parse(int argc, char **argv, const std::vector<std::string> &required) {
    for (int i = 1; i + 1 < argc; i += 2) {
      if (argv[i][0] != '-') {
        std::cerr << "unexpected argument " << argv[i] << "\n";
        return false;
      }
      kv[argv[i] + 1] = argv[i + 1];
    }
    for (const auto &r : required)
      if (!kv.count(r)) {
        std::cerr << "missing required argument -" << r << "\n";
        return false;
      }
    return true;
  }
  std::string s(const std::string &k) const { return kv.at(k); }
  uint32_t u(const std::string &k) const { return (uint32_t)std::stoul(kv.at(k)); }
  bool b(const std::string &k) const {
    const std::string v = kv.at(k);
    return v == "true" || v == "1" || v == "True";
  }
};

inline std::string data_root(const std::string &username) {
  const char *env = std::getenv("MVR_DATASET_ROOT");
  const std::string home = env ? std::string(env) : "/home/" + username;
  return home + "/Dataset/multi-vector-retrieval-GPU";
}

inline std::map<std::string, std::string> filename_map(const std::string &username,
                                                       const std::string &dataset,
                                                       const std::string &method_name,
                                                       const std::string &suffix) {
  const std::string root = data_root(username);
  const std::string index = root + "/Index/" + dataset + "/" + method_name + "-" + suffix;
  const std::string emb = root + "/Embedding/" + dataset;
  return {{"centroid_l", index + "/centroid_l.npy"},
          {"vq_code_l", index + "/vq_code_l.npy"},
          {"weight_l", index + "/weight_l.npy"},
          {"residual_code_l", index + "/residual_code_l.npy"},
          {"ivf_index", index + "/ivf.index"},
          {"query_l", emb + "/query_embedding.npy"},
          {"item_n_vec_l", index + "/item_n_vec_l.npy"},
          {"answer_path", root + "/Result/answer"},
          {"query_id", root + "/RawData/" + dataset + "/document/queries.dev.tsv"}};
}

// First tab-separated column of queries.dev.tsv (CPPIOUtil.hpp:11-39).
inline bool read_query_ids(const std::string &path, std::vector<uint32_t> &ids) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    const size_t tab = line.find('\t');
    if (tab == std::string::npos) continue;
    ids.push_back((uint32_t)std::stoul(line.substr(0, tab)));
  }
  return true;
}

inline bool load_queries(const std::string &path, NpyArray &q, uint32_t &n_query,
                         uint32_t &query_n_vec) {
  std::string err;
  if (!npy_load(path, q, err)) {
    std::cerr << err << "\n";
    return false;
  }
  if (q.shape.size() != 3 || q.descr.substr(1) != "f4" || q.shape[2] != 128) {
    std::cerr << "query_embedding.npy must be float32 [n_query, n_vec, 128]\n";
    return false;
  }
  n_query = (uint32_t)q.shape[0];
  query_n_vec = (uint32_t)q.shape[1];
  return true;
}

}  // namespace mvr::app
