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
  int64_t max_graph_n = 0;         // largest member graph
  // task-split thresholds (autotuned for batches): triangle-pass owners with
  // more than te_cta_min upward neighbours (<= 128) and 4-cycle tasks whose
  // 2-hop bound exceeds c4_warp_bound (<= 256) run on a CTA; clique tasks
  // with more than cq_warp_max out-neighbours (<= 64) run on a CTA; 4-cycle
  // tasks whose bound exceeds c4_big_min (<= 3072; GPM_C4_BIG_MIN overrides)
  // go to the giant-task kernel
  int te_cta_min = 128, c4_warp_bound = 256, cq_warp_max = 64;
  long long c4_big_min = 3072;
  int size = 4;  // 3: only the per-edge triangle pass and the degree sums (out[0..1])
};

// k-cliques of an upward graph (every list holds only larger ids); the count
// of each vertex task is added to acc[stride * graph(u) + slot].
int clique_run_upward(int64_t n, const int64_t *off, const int32_t *adj, int max_deg, int k, const int32_t *gid,
                      unsigned long long *acc, int stride, int slot, cudaStream_t st);

// The same split into a plan (allocations, task queues, host syncs) and a
// run (launches only, so it can be captured into a CUDA graph).
struct CliquePlan {
  int64_t n = 0;
  const int64_t *roff = nullptr;
  const int32_t *radj = nullptr;
  int k = 0, stride = 0, slot = 0, n_cta = 0, n_warp = 0, grid = 0;
  const int32_t *gid = nullptr;
  unsigned long long *acc = nullptr;
  size_t slab_words = 0;
  DevBuf<int32_t> ctasks, wtasks;
  DevBuf<int> counters;
  DevBuf<uint32_t> slabs;
};
int clique_plan_build(CliquePlan *p, int64_t n, const int64_t *roff, const int32_t *radj, int max_deg, int k,
                      const int32_t *gid, unsigned long long *acc, int stride, int slot, cudaStream_t st,
                      int warp_max = 64);
int clique_plan_run(CliquePlan *p, cudaStream_t st);

// Motif pipeline split the same way; `acc` (scratch sums) and `out` are
// owned by the plan, ngraphs x 8 each.  out per graph: [0] induced 2-paths,
// [1] triangles, [2..7] 3-star, 4-path, tailed triangle, 4-cycle, diamond,
// 4-clique.
struct MotifPlan {
  MotifInput in;
  DevBuf<int64_t> split, doff;
  DevBuf<int32_t> dadj;
  int dag_max = 0;
  DevBuf<unsigned> te;
  DevBuf<int32_t> te_ct, te_wt, c4_ct, c4_wt, c4_bt;
  DevBuf<unsigned long long> c4_bb;  // giant 4-cycle tasks and their 2-hop bounds, largest first
  int te_nc = 0, te_nw = 0, c4_nc = 0, c4_nw = 0, c4_nb = 0, te_grid = 0, c4_grid = 0, c4_big_grid = 0;
  DevBuf<int64_t> c4_cur;  // per-CTA cursors and list ends of the giant tasks
  int64_t c4_scratch = 0;
  DevBuf<int> te_counters, c4_counters;
  CliquePlan k4;
  DevBuf<unsigned long long> acc, out;
};
int motif_plan_build(const MotifInput &in, MotifPlan *p, cudaStream_t st);
int motif_plan_run(MotifPlan *p, cudaStream_t st);
// One stage alone (0 triangles per edge, 1 4-cycles, 2 4-cliques), for tuning.
int motif_plan_run_stage(MotifPlan *p, int stage, cudaStream_t st);

}  // namespace gpm
