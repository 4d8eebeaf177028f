// tc_rank.cuh -- plan of the rank-relabelled, smaller-side triangle count.
#pragma once
#include "common.cuh"

namespace gpm {

// Per-graph schedule of GPM_TC_BITMAP (device arrays):
//   roff/radj   stored lists renumbered by (degree, id) rank, sorted
//   poff/padj   partner CSR: for owner x, the vertices whose lists are
//               streamed against N(x); the first plong[x] are long lists
//   cta_tasks / warp_tasks  owners by size class, heaviest first
struct RankPlan {
  int cta_min = 0, long_min = 0;
  int n_cta = 0, n_warp = 0;
  DevBuf<int64_t> roff, poff;
  DevBuf<int32_t> radj, padj, plong;
  DevBuf<int32_t> cta_tasks, warp_tasks;
  DevBuf<int> counters;
};

int rank_build_plan(gpm_graph *g, int cta_min, int long_min, cudaStream_t st);
int rank_launch(gpm_graph *g, cudaStream_t st, unsigned long long *d_out);

}  // namespace gpm
