/* Stand-in for RAFT 25.04's select_k: declared, never defined (see
 * raft/linalg/reduce.cuh here).  The oracle driver selects with a restated
 * (score desc, id asc) sort where it needs a selection. */
#pragma once
#include "raft/core/device_resources.hpp"
namespace raft { namespace matrix { namespace detail {
template <class... A> void select_k(A &&...);
}}}  // namespace raft::matrix::detail
