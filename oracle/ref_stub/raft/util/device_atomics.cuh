/* Project-written stand-in for RAFT's float atomicMax
 * (raft/util/device_atomics.cuh, RAFT 25.04), which the reference's
 * max_qvec_doc_score kernel (FilterPP.hpp:99-142) calls.  A compare-and-swap
 * loop on the word: the stored value ends as the maximum of every value
 * offered, whatever the order of the atomics, so any correct implementation
 * (RAFT's included) leaves the same FP32 result.  Returns the old value. */
#pragma once
#include <cuda_runtime.h>

__device__ inline float atomicMax(float *address, float val) {
  unsigned int *a = reinterpret_cast<unsigned int *>(address);
  unsigned int old = *a, assumed;
  do {
    assumed = old;
    if (!(val > __uint_as_float(assumed))) break;
    old = atomicCAS(a, assumed, __float_as_uint(val));
  } while (old != assumed);
  return __uint_as_float(old);
}
