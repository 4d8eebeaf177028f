// batch.cu -- many graphs, one launch per pipeline stage, replayed from a
// captured CUDA graph (no counterpart in the reference, which launches one
// solver per graph and synchronises after each kernel, PatternSolver.cuh:177-246).
//
// The member graphs are stored as one disjoint union: graph g's vertices are
// the id range [vbase[g], vbase[g+1]).  The union is rank-relabelled with the
// key (graph id, degree), so each member stays a contiguous range and is
// ranked within itself; every kernel of the motif pipeline (motif.cu) reads a
// per-vertex graph id and accumulates into per-graph sums, so one persistent
// work-stealing launch per stage serves all members.  The plan (task queues,
// scratch) is built once; the run is launches only and is captured into a
// CUDA graph that each step replays.
//
// Autotuner: the three task-split thresholds of the pipeline (CTA vs warp
// for triangle owners, 4-cycle tasks and clique tasks) are chosen per batch
// by timing each stage alone with CUDA events over a small candidate set.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "motif.cuh"
#include "tc_rank.cuh"

struct gpm_batch {
  int ngraphs = 0;
  std::vector<int64_t> vbase;  // host copy, ngraphs + 1
  int64_t max_n = 0;
  gpm_graph g;                 // the union
  gpm::DevBuf<int32_t> gid;
  gpm::DevBuf<int64_t> gbase;
  gpm::MotifPlan *plan = nullptr;
  int tune[3] = {128, 256, 64};
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~gpm_batch();
};

namespace gpm {

__global__ void k_fill_gid(int64_t lo, int64_t hi, int32_t g, int32_t *__restrict__ gid) {
  for (int64_t v = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < hi; v += (int64_t)gridDim.x * blockDim.x)
    gid[v] = g;
}
__global__ void k_shift(int64_t m, int32_t by, int32_t *__restrict__ a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    a[i] += by;
}
__global__ void k_gen_cl(int64_t m, ChungLu p, uint64_t seed, int32_t base, int32_t *__restrict__ s,
                         int32_t *__restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    s[i] = base + chung_lu_vertex(p, draw(seed, 201, (uint64_t)i));
    d[i] = base + chung_lu_vertex(p, draw(seed, 202, (uint64_t)i));
  }
}

static int grid_of(int64_t w) { return (int)std::max<int64_t>(1, std::min<int64_t>((w + 255) / 256, num_sms() * 16)); }

static void drop_graph(gpm_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

static void drop_plan(gpm_batch *b) {
  drop_graph(b);
  delete b->plan;
  b->plan = nullptr;
}

// union built from device edge lists with global ids
static int finish_union(gpm_batch *b, int64_t m_total, const int32_t *ds, const int32_t *dd) {
  const int64_t n_total = b->vbase.back();
  GPM_TRY(build_csr_device(&b->g, n_total, m_total, ds, dd, 1, 0));
  GPM_TRY(b->gid.reserve(n_total));
  GPM_TRY(b->gbase.reserve(b->ngraphs + 1));
  for (int g = 0; g < b->ngraphs; ++g)
    if (b->vbase[g + 1] > b->vbase[g])
      k_fill_gid<<<grid_of(b->vbase[g + 1] - b->vbase[g]), 256>>>(b->vbase[g], b->vbase[g + 1], g, b->gid.p);
  GPM_CUDA(cudaMemcpy(b->gbase.p, b->vbase.data(), sizeof(int64_t) * (b->ngraphs + 1), cudaMemcpyHostToDevice));
  GPM_TRY(ensure_rank_graph(&b->g, 0, b->gid.p, b->ngraphs));
  GPM_CUDA(cudaDeviceSynchronize());
  return GPM_OK;
}

static int ensure_plan(gpm_batch *b) {
  if (b->plan) return GPM_OK;
  MotifInput in;
  in.n = b->g.n;
  in.nnz = b->g.nnz;
  in.roff = b->g.rg->roff.p;
  in.radj = b->g.rg->radj.p;
  in.gid = b->gid.p;
  in.gbase = b->gbase.p;
  in.ngraphs = b->ngraphs;
  in.max_graph_n = b->max_n;
  in.te_cta_min = b->tune[0];
  in.c4_warp_bound = b->tune[1];
  in.cq_warp_max = b->tune[2];
  MotifPlan *p = new MotifPlan();
  int s = motif_plan_build(in, p, 0);
  if (s != GPM_OK) {
    delete p;
    return s;
  }
  b->plan = p;
  return GPM_OK;
}

static int ensure_graph(gpm_batch *b) {
  if (b->exec) return GPM_OK;
  GPM_TRY(ensure_plan(b));
  if (!b->cap) GPM_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  GPM_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  int s = motif_plan_run(b->plan, b->cap);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
  if (s != GPM_OK) {
    if (graph) cudaGraphDestroy(graph);
    return s;
  }
  if (e != cudaSuccess) return fail(GPM_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  b->graph = graph;
  GPM_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return GPM_OK;
}

}  // namespace gpm

using namespace gpm;

gpm_batch::~gpm_batch() {
  drop_plan(this);
  if (cap) cudaStreamDestroy(cap);
}

extern "C" {

int gpm_batch_create(int ngraphs, const int64_t *n, const int64_t *m, const int32_t *src, const int32_t *dst,
                     gpm_batch **out) {
  if (!out || ngraphs < 1 || !n || !m) return fail(GPM_EINVAL, "gpm_batch_create: bad argument");
  GPM_TRY(ensure_device());
  gpm_batch *b = new gpm_batch();
  b->ngraphs = ngraphs;
  b->vbase.assign(ngraphs + 1, 0);
  int64_t m_total = 0;
  for (int g = 0; g < ngraphs; ++g) {
    if (n[g] < 0 || m[g] < 0) {
      delete b;
      return fail(GPM_EINVAL, "negative member size");
    }
    b->vbase[g + 1] = b->vbase[g] + n[g];
    b->max_n = std::max(b->max_n, n[g]);
    m_total += m[g];
  }
  if (b->vbase.back() >= (1ll << 31)) {
    delete b;
    return fail(GPM_EUNSUPPORTED, "more than 2^31 vertices in a batch");
  }
  std::vector<int32_t> hs(m_total), hd(m_total);
  int64_t e = 0;
  for (int g = 0; g < ngraphs; ++g)
    for (int64_t i = 0; i < m[g]; ++i, ++e) {
      if (src[e] < 0 || dst[e] < 0 || src[e] >= n[g] || dst[e] >= n[g]) {
        delete b;
        return fail(GPM_EINVAL, "member edge out of range");
      }
      hs[e] = (int32_t)(src[e] + b->vbase[g]);
      hd[e] = (int32_t)(dst[e] + b->vbase[g]);
    }
  DevBuf<int32_t> ds, dd;
  int s = ds.reserve(m_total);
  if (s == GPM_OK) s = dd.reserve(m_total);
  if (s == GPM_OK && m_total > 0) {
    cudaMemcpy(ds.p, hs.data(), sizeof(int32_t) * m_total, cudaMemcpyHostToDevice);
    cudaMemcpy(dd.p, hd.data(), sizeof(int32_t) * m_total, cudaMemcpyHostToDevice);
  }
  if (s == GPM_OK) s = finish_union(b, m_total, ds.p, dd.p);
  if (s != GPM_OK) {
    delete b;
    return s;
  }
  *out = b;
  return GPM_OK;
}

int gpm_batch_generate_chung_lu(int ngraphs, const int64_t *n, const double *gamma, const double *mean_deg,
                                uint64_t seed, gpm_batch **out) {
  if (!out || ngraphs < 1 || !n || !gamma || !mean_deg) return fail(GPM_EINVAL, "gpm_batch_generate_chung_lu: bad argument");
  GPM_TRY(ensure_device());
  gpm_batch *b = new gpm_batch();
  b->ngraphs = ngraphs;
  b->vbase.assign(ngraphs + 1, 0);
  std::vector<int64_t> mm(ngraphs), ebase(ngraphs + 1, 0);
  for (int g = 0; g < ngraphs; ++g) {
    if (n[g] < 2 || gamma[g] <= 2.0 || mean_deg[g] <= 0) {
      delete b;
      return fail(GPM_EINVAL, "bad Chung-Lu member parameters");
    }
    b->vbase[g + 1] = b->vbase[g] + n[g];
    b->max_n = std::max(b->max_n, n[g]);
    mm[g] = (int64_t)llround((double)n[g] * mean_deg[g] / 2.0);
    ebase[g + 1] = ebase[g] + mm[g];
  }
  if (b->vbase.back() >= (1ll << 31) || 2 * ebase.back() >= (1ll << 31)) {
    delete b;
    return fail(GPM_EUNSUPPORTED, "batch exceeds 2^31 vertices or directed entries");
  }
  DevBuf<int32_t> ds, dd;
  int s = ds.reserve(ebase.back());
  if (s == GPM_OK) s = dd.reserve(ebase.back());
  if (s == GPM_OK) {
    for (int g = 0; g < ngraphs; ++g) {
      ChungLu p = chung_lu_params(n[g], gamma[g], mean_deg[g]);
      if (mm[g] > 0)
        k_gen_cl<<<grid_of(mm[g]), 256>>>(mm[g], p, mix64(seed + (uint64_t)g), (int32_t)b->vbase[g],
                                          ds.p + ebase[g], dd.p + ebase[g]);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = fail(GPM_ECUDA, cudaGetErrorString(e));
  }
  if (s == GPM_OK) s = finish_union(b, ebase.back(), ds.p, dd.p);
  if (s != GPM_OK) {
    delete b;
    return s;
  }
  *out = b;
  return GPM_OK;
}

int gpm_batch_info(const gpm_batch *b, int *ngraphs, int64_t *n_total, int64_t *nnz_total) {
  if (!b) return fail(GPM_EINVAL, "NULL batch");
  if (ngraphs) *ngraphs = b->ngraphs;
  if (n_total) *n_total = b->g.n;
  if (nnz_total) *nnz_total = b->g.nnz;
  return GPM_OK;
}

int gpm_batch_member_csr(const gpm_batch *b, int g, int64_t *offsets, int32_t *indices, int64_t *n, int64_t *nnz) {
  if (!b || g < 0 || g >= b->ngraphs) return fail(GPM_EINVAL, "bad member index");
  int64_t lo = b->vbase[g], hi = b->vbase[g + 1];
  int64_t e0 = 0, e1 = 0;
  GPM_CUDA(cudaMemcpy(&e0, b->g.off.p + lo, sizeof(int64_t), cudaMemcpyDeviceToHost));
  GPM_CUDA(cudaMemcpy(&e1, b->g.off.p + hi, sizeof(int64_t), cudaMemcpyDeviceToHost));
  if (n) *n = hi - lo;
  if (nnz) *nnz = e1 - e0;
  if (offsets) {
    GPM_CUDA(cudaMemcpy(offsets, b->g.off.p + lo, sizeof(int64_t) * (hi - lo + 1), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i <= hi - lo; ++i) offsets[i] -= e0;
  }
  if (indices && e1 > e0) {
    GPM_CUDA(cudaMemcpy(indices, b->g.adj.p + e0, sizeof(int32_t) * (e1 - e0), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < e1 - e0; ++i) indices[i] -= (int32_t)lo;
  }
  return GPM_OK;
}

int gpm_batch_autotune(gpm_batch *b, int *tuned) {
  if (!b) return fail(GPM_EINVAL, "NULL batch");
  static const int cand[3][4] = {{32, 64, 128, 128}, {64, 128, 256, 256}, {16, 32, 64, 64}};
  cudaEvent_t e0, e1;
  GPM_CUDA(cudaEventCreate(&e0));
  GPM_CUDA(cudaEventCreate(&e1));
  for (int stage = 0; stage < 3; ++stage) {
    float best = 1e30f;
    int best_v = b->tune[stage];
    for (int c = 0; c < 3; ++c) {
      drop_plan(b);
      b->tune[stage] = cand[stage][c];
      GPM_TRY(ensure_plan(b));
      GPM_TRY(motif_plan_run_stage(b->plan, stage, 0));  // warm-up
      GPM_CUDA(cudaEventRecord(e0, 0));
      for (int r = 0; r < 2; ++r) GPM_TRY(motif_plan_run_stage(b->plan, stage, 0));
      GPM_CUDA(cudaEventRecord(e1, 0));
      GPM_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      GPM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        best_v = cand[stage][c];
      }
    }
    b->tune[stage] = best_v;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  drop_plan(b);
  GPM_TRY(ensure_plan(b));
  if (tuned)
    for (int i = 0; i < 3; ++i) tuned[i] = b->tune[i];
  return GPM_OK;
}

int gpm_batch_stage_ms(gpm_batch *b, float *ms) {
  if (!b || !ms) return fail(GPM_EINVAL, "NULL argument");
  GPM_TRY(ensure_plan(b));
  cudaEvent_t e0, e1;
  GPM_CUDA(cudaEventCreate(&e0));
  GPM_CUDA(cudaEventCreate(&e1));
  for (int stage = 0; stage < 3; ++stage) {
    GPM_CUDA(cudaEventRecord(e0, 0));
    GPM_TRY(motif_plan_run_stage(b->plan, stage, 0));
    GPM_CUDA(cudaEventRecord(e1, 0));
    GPM_CUDA(cudaEventSynchronize(e1));
    GPM_CUDA(cudaEventElapsedTime(&ms[stage], e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return GPM_OK;
}

int gpm_batch_motif_async(gpm_batch *b, int use_graph, void *stream, uint64_t *d_out) {
  if (!b || !d_out) return fail(GPM_EINVAL, "gpm_batch_motif_async: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (use_graph) {
    if (!b->exec) return fail(GPM_EINVAL, "call gpm_batch_motif once first (it captures the graph)");
    GPM_CUDA(cudaGraphLaunch(b->exec, st));
  } else {
    if (!b->plan) return fail(GPM_EINVAL, "call gpm_batch_motif once first (it builds the plan)");
    GPM_TRY(motif_plan_run(b->plan, st));
  }
  GPM_CUDA(cudaMemcpyAsync(d_out, b->plan->out.p, sizeof(uint64_t) * 8 * b->ngraphs, cudaMemcpyDeviceToDevice, st));
  return GPM_OK;
}

int gpm_batch_motif(gpm_batch *b, int use_graph, void *stream, uint64_t *out) {
  if (!b || !out) return fail(GPM_EINVAL, "gpm_batch_motif: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  GPM_TRY(ensure_plan(b));
  if (use_graph) {
    GPM_TRY(ensure_graph(b));
    GPM_CUDA(cudaGraphLaunch(b->exec, st));
  } else {
    GPM_TRY(motif_plan_run(b->plan, st));
  }
  GPM_CUDA(cudaMemcpyAsync(out, b->plan->out.p, sizeof(uint64_t) * 8 * b->ngraphs, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

int gpm_batch_destroy(gpm_batch *b) {
  delete b;
  return GPM_OK;
}

}  // extern "C"
