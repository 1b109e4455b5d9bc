// GPGPUBuildIndexPackGPU -- a pybind11 module with the names, arguments and
// return shapes of the reference's build-side module
// (src/app/build_index/GPGPUBuildIndexPackGPU.cpp:14-44), so that the
// reference's index-build script (script/evaluation/technique/vq_sq_pack.py,
// `module.compute_quantized_scalar`, `module.CompressResidualCode`, and the
// IVF builder) runs on this library unchanged:
//
//   compute_quantized_scalar(item_vec_l, centroid_l, code_l, n_bit)
//       -> (cutoff_l, weight_l): the residual quantizer's bucket cutoffs and
//          weights (ResidualScalarQuantizationPack.hpp:17-100), selected
//          exactly on the GPU (mvr_residual_quantiles_device);
//   CompressResidualCode(centroid_l, cutoff_l, weight_l, n_bit)
//       .n_val_per_vec: packed residual bytes per vector;
//       .compute_residual_code(vec_l, code_l) -> (residual_code_l,): packed
//          MSB-first bucket codes (ResidualScalarQuantizationPackGPU.hpp:220-268),
//          on the GPU (mvr_pack_residual_device);
//   IVFIndex(vq_code_l, item_n_vec_l, n_vec, n_item, n_centroid)
//       .build(): per centroid the ascending ids of the items that have a
//          token assigned to it (IVFIndex.hpp:92-166);
//       .save(location): the binary CSR file (IVFIndex.hpp:168-183).
//
// Vectors are 128-dimensional (the library's token width); other widths
// raise ValueError.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mvr.h"

namespace py = pybind11;

namespace {

using FloatArr = py::array_t<float, py::array::c_style | py::array::forcecast>;
using U32Arr = py::array_t<uint32_t, py::array::c_style | py::array::forcecast>;
constexpr uint32_t kVecDim = 128;

void cuda_check(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}
void mvr_check(int rc) {
  if (rc != MVR_OK) throw std::runtime_error(mvr_last_error());
}

// device copy of a host array, freed with the object
struct DeviceCopy {
  void *ptr = nullptr;
  DeviceCopy(const void *host, size_t bytes) {
    cuda_check(cudaMalloc(&ptr, bytes ? bytes : 1));
    if (bytes) cuda_check(cudaMemcpy(ptr, host, bytes, cudaMemcpyHostToDevice));
  }
  explicit DeviceCopy(size_t bytes) { cuda_check(cudaMalloc(&ptr, bytes ? bytes : 1)); }
  ~DeviceCopy() { cudaFree(ptr); }
  DeviceCopy(const DeviceCopy &) = delete;
  DeviceCopy &operator=(const DeviceCopy &) = delete;
};

void check_vectors(const FloatArr &a, const char *name) {
  if (a.ndim() != 2 || (uint32_t)a.shape(1) != kVecDim)
    throw py::value_error(std::string(name) + ": expected shape [n, 128]");
}

void check_n_bit(uint32_t n_bit) {
  if (n_bit != 1 && n_bit != 2 && n_bit != 4 && n_bit != 8)
    throw py::value_error("n_bit must be 1, 2, 4 or 8");
}

py::tuple compute_quantized_scalar(const FloatArr &item_vec_l, const FloatArr &centroid_l,
                                   const U32Arr &code_l, uint32_t n_bit) {
  check_vectors(item_vec_l, "item_vec_l");
  check_vectors(centroid_l, "centroid_l");
  check_n_bit(n_bit);
  const size_t n_vec = item_vec_l.shape(0);
  if (code_l.ndim() != 1 || (size_t)code_l.shape(0) != n_vec)
    throw py::value_error("code_l: expected one code per vector");
  const uint32_t n_cent = (uint32_t)centroid_l.shape(0);
  const uint32_t *code = code_l.data();
  for (size_t i = 0; i < n_vec; i++)
    if (code[i] >= n_cent) throw py::value_error("code_l: code out of range");
  std::vector<float> cutoff((1u << n_bit) - 1u), weight(1u << n_bit);
  {
    DeviceCopy v(item_vec_l.data(), n_vec * kVecDim * sizeof(float));
    DeviceCopy c(centroid_l.data(), (size_t)n_cent * kVecDim * sizeof(float));
    DeviceCopy k(code, n_vec * sizeof(uint32_t));
    py::gil_scoped_release unlocked;
    mvr_check(mvr_residual_quantiles_device(
        static_cast<const float *>(v.ptr), n_vec, static_cast<const float *>(c.ptr), kVecDim,
        static_cast<const uint32_t *>(k.ptr), n_bit, cutoff.data(), weight.data(), nullptr));
  }
  return py::make_tuple(cutoff, weight);
}

class CompressResidualCode {
 public:
  uint32_t n_val_per_vec;

  CompressResidualCode(const FloatArr &centroid_l, const FloatArr &cutoff_l,
                       const FloatArr &weight_l, uint32_t n_bit)
      : n_val_per_vec(0), n_bit_(n_bit) {
    check_vectors(centroid_l, "centroid_l");
    check_n_bit(n_bit);
    if ((uint32_t)cutoff_l.size() + 1 != (1u << n_bit) || (uint32_t)weight_l.size() != (1u << n_bit))
      throw py::value_error("cutoff_l / weight_l: 2^n_bit - 1 cutoffs and 2^n_bit weights");
    n_cent_ = (uint32_t)centroid_l.shape(0);
    centroid_.assign(centroid_l.data(), centroid_l.data() + (size_t)n_cent_ * kVecDim);
    cutoff_.assign(cutoff_l.data(), cutoff_l.data() + cutoff_l.size());
    n_val_per_vec = kVecDim * n_bit / 8;
  }

  py::tuple compute_residual_code(const FloatArr &vec_l, const U32Arr &code_l) const {
    check_vectors(vec_l, "vec_l");
    const size_t n_vec = vec_l.shape(0);
    if (code_l.ndim() != 1 || (size_t)code_l.shape(0) != n_vec)
      throw py::value_error("code_l: expected one code per vector");
    const uint32_t *code = code_l.data();
    for (size_t i = 0; i < n_vec; i++)
      if (code[i] >= n_cent_) throw py::value_error("code_l: code out of range");
    py::array_t<uint8_t> out((py::ssize_t)(n_vec * n_val_per_vec));
    {
      DeviceCopy v(vec_l.data(), n_vec * kVecDim * sizeof(float));
      DeviceCopy c(centroid_.data(), centroid_.size() * sizeof(float));
      DeviceCopy k(code, n_vec * sizeof(uint32_t));
      DeviceCopy r(n_vec * n_val_per_vec);
      uint8_t *host = out.mutable_data();
      py::gil_scoped_release unlocked;
      mvr_check(mvr_pack_residual_device(static_cast<const float *>(v.ptr), n_vec,
                                         static_cast<const float *>(c.ptr), kVecDim,
                                         static_cast<const uint32_t *>(k.ptr), cutoff_.data(),
                                         n_bit_, static_cast<uint8_t *>(r.ptr), nullptr));
      cuda_check(cudaMemcpy(host, r.ptr, n_vec * n_val_per_vec, cudaMemcpyDeviceToHost));
    }
    return py::make_tuple(out);
  }

 private:
  uint32_t n_bit_, n_cent_ = 0;
  std::vector<float> centroid_, cutoff_;
};

class IVFIndex {
 public:
  IVFIndex(const U32Arr &vq_code_l, const U32Arr &item_n_vec_l, size_t n_vec, uint32_t n_item,
           uint32_t n_centroid)
      : n_vec_(n_vec), n_item_(n_item), n_centroid_(n_centroid) {
    if ((size_t)vq_code_l.size() != n_vec) throw py::value_error("vq_code_l: n_vec codes");
    if ((size_t)item_n_vec_l.size() != n_item) throw py::value_error("item_n_vec_l: n_item sizes");
    code_.assign(vq_code_l.data(), vq_code_l.data() + n_vec);
    item_n_vec_.assign(item_n_vec_l.data(), item_n_vec_l.data() + n_item);
    size_t tot = 0;
    for (uint32_t n : item_n_vec_) tot += n;
    if (tot != n_vec) throw py::value_error("item_n_vec_l must sum to n_vec");
    for (uint32_t c : code_)
      if (c >= n_centroid) throw py::value_error("vq_code_l: code out of range");
  }

  // two passes of a counting sort: list sizes, then item ids in item order
  void build() {
    std::vector<uint32_t> cents;
    size_.assign(n_centroid_, 0u);
    auto each_item = [&](auto &&visit) {
      size_t v0 = 0;
      for (uint32_t it = 0; it < n_item_; it++) {
        cents.assign(code_.begin() + v0, code_.begin() + v0 + item_n_vec_[it]);
        std::sort(cents.begin(), cents.end());
        cents.erase(std::unique(cents.begin(), cents.end()), cents.end());
        for (uint32_t c : cents) visit(c, it);
        v0 += item_n_vec_[it];
      }
    };
    each_item([&](uint32_t c, uint32_t) { size_[c]++; });
    offset_.assign(n_centroid_, 0);
    for (uint32_t c = 1; c < n_centroid_; c++) offset_[c] = offset_[c - 1] + size_[c - 1];
    const size_t n_ele = n_centroid_ ? offset_[n_centroid_ - 1] + size_[n_centroid_ - 1] : 0;
    ids_.assign(n_ele, 0u);
    std::vector<size_t> fill(offset_);
    each_item([&](uint32_t c, uint32_t it) { ids_[fill[c]++] = it; });
  }

  void save(const std::string &location) const {
    std::ofstream out(location, std::ios::binary | std::ios::out);
    if (!out) throw std::runtime_error("cannot write " + location);
    const size_t n_ele = ids_.size();
    out.write(reinterpret_cast<const char *>(&n_centroid_), sizeof(uint32_t));
    out.write(reinterpret_cast<const char *>(&n_ele), sizeof(size_t));
    out.write(reinterpret_cast<const char *>(offset_.data()), offset_.size() * sizeof(size_t));
    out.write(reinterpret_cast<const char *>(size_.data()), size_.size() * sizeof(uint32_t));
    out.write(reinterpret_cast<const char *>(ids_.data()), n_ele * sizeof(uint32_t));
    if (!out) throw std::runtime_error("write failed: " + location);
  }

 private:
  size_t n_vec_;
  uint32_t n_item_, n_centroid_;
  std::vector<uint32_t> code_, item_n_vec_, size_, ids_;
  std::vector<size_t> offset_;
};

}  // namespace

PYBIND11_MODULE(GPGPUBuildIndexPackGPU, m) {
  m.doc() = "Index-build functions of the GPU multi-vector search (libmvr), with the reference "
            "build module's names and arguments";
  m.def("compute_quantized_scalar", &compute_quantized_scalar, py::arg("item_vec_l"),
        py::arg("centroid_l"), py::arg("code_l"), py::arg("n_bit"));
  py::class_<CompressResidualCode>(m, "CompressResidualCode")
      .def(py::init<const FloatArr &, const FloatArr &, const FloatArr &, uint32_t>(),
           py::arg("centroid_l"), py::arg("cutoff_l"), py::arg("weight_l"), py::arg("n_bit"))
      .def_readonly("n_val_per_vec", &CompressResidualCode::n_val_per_vec)
      .def("compute_residual_code", &CompressResidualCode::compute_residual_code,
           py::arg("vec_l"), py::arg("code_l"));
  py::class_<IVFIndex>(m, "IVFIndex")
      .def(py::init<const U32Arr &, const U32Arr &, size_t, uint32_t, uint32_t>(),
           py::arg("vq_code_l"), py::arg("item_n_vec_l"), py::arg("n_vec"), py::arg("n_item"),
           py::arg("n_centroid"))
      .def("build", &IVFIndex::build)
      .def("save", &IVFIndex::save, py::arg("location"));
}
