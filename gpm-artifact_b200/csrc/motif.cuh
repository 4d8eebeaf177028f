// motif.cuh -- motif pipeline over one graph or a disjoint union of graphs.
#pragma once
#include "common.cuh"

namespace gpm {

// A symmetric graph in rank order (tc_rank.cuh), possibly the disjoint union
// of several graphs whose vertices are contiguous rank ranges.
struct MotifInput {
  int64_t n = 0, nnz = 0;
  const int64_t *roff = nullptr;
  const int32_t *radj = nullptr;
  const int32_t *gid = nullptr;    // per-vertex graph index (nullptr: one graph)
  const int64_t *gbase = nullptr;  // per-graph first vertex (nullptr: 0)
  int ngraphs = 1;
  int64_t max_graph_n = 0;         // largest member graph (sizes 4-cycle counters)
};

// d_acc: ngraphs x 8 scratch sums; d_out: ngraphs x 8 results
//   [0] induced 2-paths, [1] triangles, [2..7] 3-star, 4-path, tailed triangle,
//   4-cycle, diamond, 4-clique.
int motif_pipeline(const MotifInput &in, cudaStream_t st, unsigned long long *d_acc, unsigned long long *d_out);

// k-cliques of an upward graph (every list holds only larger ids); the count
// of each vertex task is added to acc[stride * graph(u) + slot].
int clique_run_upward(int64_t n, const int64_t *off, const int32_t *adj, int max_deg, int k, const int32_t *gid,
                      unsigned long long *acc, int stride, int slot, cudaStream_t st);

}  // namespace gpm
