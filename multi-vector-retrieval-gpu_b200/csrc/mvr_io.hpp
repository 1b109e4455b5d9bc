// mvr_io.hpp -- readers for the reference's on-disk index formats: numpy
// .npy (format version 1.0/2.0/3.0, C order, little endian) and the binary
// ivf.index CSR written by IVFIndex::save (IVFIndex.hpp:168-183).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mvr {

struct NpyArray {
  std::string descr;               // e.g. "<f4", "<u4", "<i4", "|u1"
  std::vector<uint64_t> shape;
  size_t word_size = 0;
  std::vector<uint8_t> data;       // raw little-endian payload
  uint64_t numel() const {
    uint64_t n = 1;
    for (auto s : shape) n *= s;
    return n;
  }
};

// Returns false and fills err on failure.
bool npy_load(const std::string &path, NpyArray &out, std::string &err);

struct IvfCsr {
  uint32_t n_centroid = 0;
  uint64_t n_ele = 0;
  std::vector<uint64_t> offset;    // [n_centroid]
  std::vector<uint32_t> size;      // [n_centroid]
  std::vector<uint32_t> ids;       // [n_ele]
};

bool ivf_load(const std::string &path, IvfCsr &out, std::string &err);

}  // namespace mvr
