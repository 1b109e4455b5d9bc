/* Stand-in for RAFT 25.04's raft/core/device_resources.hpp (not installed
 * here), so that the reference's igp_gpu_pp headers compile unmodified into
 * oracle/_ref.  Declarations only: the reference classes that hold a RAFT
 * handle are never instantiated by the oracle driver (oracle/ref_gpu.cu),
 * which launches the reference's RAFT-free kernels itself. */
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <iostream>
#include <atomic>
#include <thread>
#include <cassert>
#include <algorithm>
#include <stdexcept>
#include <thrust/execution_policy.h>
#include <thrust/sequence.h>
#include <thrust/scan.h>
#include <thrust/copy.h>
#include <thrust/sort.h>
#include <thrust/unique.h>
#include <thrust/binary_search.h>
#include <thrust/transform.h>
#include <thrust/for_each.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/tuple.h>
#include "raft/util/device_atomics.cuh"

namespace raft {
struct device_resources {};
namespace resource {
inline void set_cuda_stream(device_resources &, cudaStream_t) {}
}  // namespace resource
struct identity_op {
  template <class T> __host__ __device__ T operator()(const T &x) const { return x; }
};
struct add_op {
  template <class T> __host__ __device__ T operator()(const T &a, const T &b) const { return a + b; }
};
struct max_op {
  template <class T> __host__ __device__ T operator()(const T &a, const T &b) const { return a > b ? a : b; }
};
}  // namespace raft
