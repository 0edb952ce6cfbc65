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

// out[k] = (int32_t)in[k] for the n entries of a connectivity already checked to lie in [0, 2^31).
void gpu_narrow(const int64_t* in, int64_t n, int32_t* out, cudaStream_t st);
// v[k] = 0 where fixed[k] is 0 (imposed values count at fixed DOFs only).
void gpu_zero_free(int64_t n, const uint8_t* fixed, double* v, cudaStream_t st);
// Node -> element-node incidence of a device connectivity of n entries (n_elems * npe, node ids in
// [0, n_nodes)): inc[q] lists the positions k = e * npe + a grouped by node, ascending inside a
// node, and node v's run is inc[inc_ptr[v] .. inc_ptr[v + 1]) (inc_ptr: n_nodes + 1 entries) --
// the arrays of the host's counting sort (analyse_topology), from a stable radix sort of the node
// ids. Synchronises the stream.
void gpu_incidence(const int32_t* conn, int64_t n, int64_t n_nodes, cudaStream_t st, int64_t* inc_ptr,
                   int32_t* inc);

}  // namespace maille
