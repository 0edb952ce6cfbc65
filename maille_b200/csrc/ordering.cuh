// ordering.cuh -- the ordering of the free nodes computed on the device (ordering.cu): the
// kept-node graph from the elements, reverse Cuthill-McKee with a George-Liu pseudo-peripheral
// start (solve.rs:200-270, applied to nodes), or a breadth-first order from a minimum-degree node,
// then the greedy colouring in that visit order (multicolour orderings) or the levels of the
// lower-triangular dependency graph (RCM). The same algorithms as the host analysis (setup.cpp)
// on the same graph (neighbours by ascending kept index), so the same permutation, without the
// host's sequential passes on the path of a solve.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"

namespace maille {

// conn: [n_elems * npe] device, caller node numbering; kept_of: [n_nodes] device, kept index of
// each node or -1; ordering: MAILLE_ORDER_MULTICOLOR, _RCM or _MULTICOLOR_BFS. Out (host):
// order[new row] = kept index, rows grouped by level and in visit order inside a level;
// level[kept index] = the row's level (its colour for the multicolour orderings). Throws
// CudaFailure on a CUDA error or when a bounded wait ran out.
void gpu_ordering(int npe, int64_t n_elems, const int32_t* conn, const int32_t* kept_of, int32_t nk,
                  int ordering, cudaStream_t st, std::vector<int32_t>& order, std::vector<int32_t>& level);

}  // namespace maille
