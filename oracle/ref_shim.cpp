// ref_shim.cpp -- binds the reference's own codec, IVF and MaxSim code,
// compiled from its unmodified headers where they lie (see oracle/Makefile,
// target `ref`),
// into a Python module used only to pin the oracle and to generate the golden
// fixtures under tests/golden/.  This file adds no arithmetic of its own: every
// result below is produced by reference code.
#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include <algorithm>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "include/struct/TypeDef.hpp"
#include "include/alg/refine/ResidualScalarQuantizationPack.hpp"
#include "include/struct/IVFIndex.hpp"
#include "include/alg/Distance.hpp"

namespace py = pybind11;
using namespace VectorSetSearch;

// ResidualCodePack::Decode over every item; returns [n_vec, dim] float32.
static py::array_t<float> decode_all(const pyarray_uint8 &residual,
                                     const pyarray_float &weight,
                                     const pyarray_uint32 &item_n_vec,
                                     const pyarray_float &centroid,
                                     const pyarray_uint32 &vq_code,
                                     uint32_t n_bit) {
  const uint32_t n_item = item_n_vec.shape(0);
  const uint32_t dim = centroid.shape(1);
  std::vector<size_t> accu(n_item);
  size_t n_vec = 0;
  for (uint32_t i = 0; i < n_item; i++) { accu[i] = n_vec; n_vec += item_n_vec.data()[i]; }
  ResidualCodePack pack(residual.data(), weight.data(), item_n_vec.data(), accu.data(),
                        centroid.data(), vq_code.data(), weight.shape(0), n_item,
                        n_vec, dim, n_bit);
  py::array_t<float> out({(py::ssize_t)n_vec, (py::ssize_t)dim});
  float *o = out.mutable_data();
  for (uint32_t i = 0; i < n_item; i++) pack.Decode(i, o + accu[i] * dim);
  return out;
}

static py::array_t<float> decode_table(uint32_t n_bit, const pyarray_float &weight) {
  const uint32_t vpb = 8 / n_bit;
  std::vector<uint32_t> nv{1};
  std::vector<size_t> acc{0};
  std::vector<uint8_t> dummy_res(1);
  std::vector<uint32_t> dummy_code{0};
  std::vector<float> dummy_cent(vpb, 0.0f);
  ResidualCodePack pack(dummy_res.data(), weight.data(), nv.data(), acc.data(),
                        dummy_cent.data(), dummy_code.data(), weight.shape(0), 1, 1,
                        vpb, n_bit);
  py::array_t<float> out({(py::ssize_t)256, (py::ssize_t)vpb});
  std::memcpy(out.mutable_data(), pack.decompression_table_.data(),
              256 * vpb * sizeof(float));
  return out;
}

static py::tuple ivf_build(const std::vector<uint32_t> &code,
                           const std::vector<uint32_t> &item_n_vec,
                           size_t n_vec, uint32_t n_item, uint32_t n_centroid,
                           const std::string &save_path) {
  Method::IVFIndex ivf(code, item_n_vec, n_vec, n_item, n_centroid);
  ivf.build();
  if (!save_path.empty()) ivf.save(save_path);
  return py::make_tuple(ivf.ivf_offset_l_, ivf.ivf_size_l_, ivf.ivf_);
}

// Distance.hpp's vectorSetDistance (sum over query vectors of the max inner
// product over the item's vectors) of one query set and one item set.
static float vector_set_distance(const pyarray_float &query, const pyarray_float &item) {
  return vectorSetDistance(query.data(), (uint32_t)query.shape(0), item.data(),
                           (uint32_t)item.shape(0), (uint32_t)query.shape(1));
}

PYBIND11_MODULE(mvr_ref, m) {
  m.def("compute_quantized_scalar", &ComputeQuantizedScalarPack,
        py::arg("item_vec_l"), py::arg("centroid_l"), py::arg("code_l"), py::arg("n_bit"));
  py::class_<CompressResidualCode>(m, "CompressResidualCode")
      .def(py::init<const pyarray_float &, const pyarray_float &, const pyarray_float &, const uint32_t>(),
           py::arg("centroid_l"), py::arg("cutoff_l"), py::arg("weight_l"), py::arg("n_bit"))
      .def("compute_residual_code", &CompressResidualCode::compute_residual_code,
           py::arg("vec_l"), py::arg("code_l"));
  m.def("decode_all", &decode_all);
  m.def("decode_table", &decode_table);
  m.def("ivf_build", &ivf_build);
  m.def("read_ivf_index", &Method::readIVFIndex);
  m.def("vector_set_distance", &vector_set_distance, py::arg("query"), py::arg("item"));
}
