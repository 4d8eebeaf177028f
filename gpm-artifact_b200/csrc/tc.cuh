// tc.cuh -- triangle-count schedule shared by the heuristic and learned paths.
#pragma once
#include "common.cuh"

namespace gpm {

// Task lists of one graph for the HASH kernel: hubs (CTA tasks) and tail
// vertices (warp tasks), plus the atomic work counters that the persistent
// grid drains them with.
struct TcPlan {
  int warp_min = 0, cta_min = 0;
  int n_cta = 0, n_warp = 0;
  DevBuf<int32_t> cta_tasks, warp_tasks;
  DevBuf<int> counters;  // [0] hub cursor, [1] tail cursor, [2..3] spare
  DevBuf<int> sizes;
};

int tc_build_plan(gpm_graph *g, int warp_min, int cta_min, cudaStream_t st);
int tc_launch(gpm_graph *g, int variant, cudaStream_t st, unsigned long long *d_out);
int tc_hash_grid();
int tc_learned_launch(gpm_graph *g, cudaStream_t st, unsigned long long *d_out);
int orient_on_stream(gpm_graph *g, cudaStream_t st);

}  // namespace gpm
