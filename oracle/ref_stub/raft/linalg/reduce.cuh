/* Stand-in for RAFT 25.04's raft/linalg/reduce.cuh: declared, never defined.
 * The reference calls it only from FilterPP::filter and RerankPP's rerank,
 * which the oracle driver does not instantiate; the row sums it would make
 * are formed by the tests from the reference kernels' per-token maxima. */
#pragma once
#include "raft/core/device_resources.hpp"
namespace raft { namespace linalg {
template <class... A> void reduce(A &&...);
}}  // namespace raft::linalg
