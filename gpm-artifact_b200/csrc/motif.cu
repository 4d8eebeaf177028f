// motif.cu -- 3- and 4-vertex induced motif counts on a symmetric graph.
//
// The reference enumerates the six induced 4-vertex motifs edge by edge
// (Motif4_G2Miner, src/gpu_kernels/G2Miner_kernels.cuh:438-552); its loops
// visit every 3-star leaf triple, which costs sum over edges of d^2 on hub
// graphs.  The B200 path counts non-induced subgraphs instead and inverts the
// containment matrix (each induced 4-vertex graph contains a fixed number of
// copies of each smaller pattern):
//   S  = sum_v C(d_v,3)                          3-stars
//   P  = sum_e (d_a-1)(d_b-1) - 3T               4-paths
//   TT = sum_e t_e (d_a + d_b - 4) / 2           tailed triangles
//   C  = 4-cycles (highest-rank vertex + 2-hop counters)
//   D  = sum_e C(t_e,2)                          diamonds
//   K  = 4-cliques (clique kernel, k = 4)
//   k = K, d = D-6K, c = C-d-3K, tt = TT-4d-12K, p = P-2tt-4c-6d-12K,
//   s = S-tt-2d-4K
// where t_e is the number of triangles on edge e.  All sums are exact uint64
// (modular arithmetic, so the differences are exact whenever the induced
// counts fit in 64 bits).  3-vertex motifs: triangles T = sum t_e / 3, induced
// 2-paths = sum_v C(d_v,2) - 3T.
//
// Kernels run on the rank-relabelled graph (tc_rank.cuh); the upward part of
// each sorted list is the degree-oriented DAG.  Every kernel takes an
// optional per-vertex graph id so one launch serves a disjoint union of many
// graphs (batch.cu) with per-graph accumulators.
#include <cub/cub.cuh>

#include <algorithm>

#include "common.cuh"
#include "motif.cuh"
#include "tc_rank.cuh"

namespace gpm {

static int grid_for(int64_t work, int block = 256) {
  int64_t g = (work + block - 1) / block;
  int64_t cap = (int64_t)num_sms() * 16;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}

__device__ __forceinline__ unsigned long long choose2(unsigned long long d) {
  return d < 2 ? 0ull : (d & 1ull) ? d * ((d - 1) >> 1) : (d >> 1) * (d - 1);
}
__device__ __forceinline__ unsigned long long choose3(unsigned long long d) {
  if (d < 3) return 0ull;
  unsigned long long a = d, b = d - 1, c = d - 2;
  if (a % 2 == 0) a >>= 1; else b >>= 1;
  if (a % 3 == 0) a /= 3; else if (b % 3 == 0) b /= 3; else c /= 3;
  return a * b * c;
}

__device__ __forceinline__ int graph_of(const int32_t *gid, int64_t x) { return gid ? gid[x] : 0; }

// split[x] = first index of x's sorted list holding an id > x
__global__ void k_split(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                        int64_t *__restrict__ split) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = roff[x], hi = roff[x + 1];
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (radj[mid] <= (int32_t)x) lo = mid + 1; else hi = mid;
    }
    split[x] = lo;
  }
}

// ------------------------------------------------------------ triangles per DAG edge
// Vertex task x, U = N+(x) held in a shared-memory (key, position) table.
// For v in U (edge e1 = (x,v)) and w in N+(v) (edge e2 = (v,w)) with w in U
// (edge e3 = (x,w)): te[e1]++, te[e2]++, te[e3]++ -- every triangle once.
constexpr int kTeWarpCap = 256;   // slots per warp (int2), tasks with |U| <= 128
constexpr int kTeCtaCap = 2048;   // slots per CTA, chunks of 1024 keys
constexpr size_t kTeSmem = kTeCtaCap * sizeof(int2);
static_assert(kTeWarpCap * 8 == kTeCtaCap, "warp tables tile the CTA table");

__device__ __forceinline__ int te_lookup(const int2 *tab, int logcap, int32_t key) {
  uint32_t mask = (1u << logcap) - 1u;
  uint32_t h = ((uint32_t)key * 2654435769u) >> (32 - logcap);
  while (true) {
    int2 s = tab[h];
    if (s.x == key) return s.y;
    if (s.x < 0) return -1;
    h = (h + 1) & mask;
  }
}
__device__ __forceinline__ void te_insert(int2 *tab, int logcap, int32_t key, int pos) {
  uint32_t mask = (1u << logcap) - 1u;
  uint32_t h = ((uint32_t)key * 2654435769u) >> (32 - logcap);
  while (atomicCAS(&tab[h].x, -1, key) != -1) h = (h + 1) & mask;
  tab[h].y = pos;
}
__device__ __forceinline__ int ilog2ceil(int x) { return x <= 1 ? 0 : 32 - __clz(x - 1); }

// stream N+(v) for one v of the current chunk; `group` lanes cooperate
__device__ __forceinline__ unsigned te_stream(const int32_t *__restrict__ radj, int64_t s, int64_t e, int32_t kmax,
                                              const int2 *tab, int logcap, int64_t xbase,
                                              unsigned *__restrict__ te, unsigned t, unsigned stride) {
  unsigned hits = 0;
  for (int64_t i = s + t; i < e; i += stride) {
    int32_t w = __ldg(radj + i);
    if (w > kmax) break;
    int p = te_lookup(tab, logcap, w);
    if (p >= 0) {
      ++hits;
      atomicAdd(&te[i], 1u);
      atomicAdd(&te[xbase + p], 1u);
    }
  }
  return hits;
}

__device__ void te_task(int32_t x, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                        const int32_t *__restrict__ radj, unsigned *__restrict__ te, int2 *tab, int cap_slots,
                        int chunk, bool cta) {
  const int tid = cta ? threadIdx.x : (int)lane_id();
  const int nthr = cta ? blockDim.x : 32;
  const unsigned lane = lane_id();
  const int wid = cta ? (threadIdx.x >> 5) : 0, nw = cta ? (blockDim.x >> 5) : 1;
  const int64_t s0 = split[x], e0 = roff[x + 1];
  const int d = (int)(e0 - s0);
  const int32_t kmax = radj[e0 - 1];
  for (int c0 = 0; c0 < d; c0 += chunk) {
    const int ck = min(chunk, d - c0);
    const int logcap = max(5, ilog2ceil(2 * ck));
    if (cta) __syncthreads(); else __syncwarp();
    for (int i = tid; i < (1 << logcap); i += nthr) tab[i] = make_int2(-1, 0);
    if (cta) __syncthreads(); else __syncwarp();
    for (int i = tid; i < ck; i += nthr) te_insert(tab, logcap, radj[s0 + c0 + i], c0 + i);
    if (cta) __syncthreads(); else __syncwarp();
    // every v of U (all chunks) against this chunk's table
    for (int j = wid; j < d; j += nw) {
      int32_t v = radj[s0 + j];
      // table positions are relative to s0 (the whole upward list of x)
      unsigned h = te_stream(radj, split[v], roff[v + 1], kmax, tab, logcap, s0, te, lane, 32);
      h = warp_sum(h);
      if (lane == 0 && h) atomicAdd(&te[s0 + j], h);
    }
  }
  if (cta) __syncthreads(); else __syncwarp();
  (void)cap_slots;
}

__global__ void __launch_bounds__(256) k_edge_tri(const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                                                  const int32_t *__restrict__ radj, const int32_t *__restrict__ cta_tasks,
                                                  int n_cta, const int32_t *__restrict__ warp_tasks, int n_warp,
                                                  int *__restrict__ counters, unsigned *__restrict__ te) {
  extern __shared__ __align__(16) int2 tsm[];
  __shared__ int s_task;
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    te_task(cta_tasks[t], roff, split, radj, te, tsm, kTeCtaCap, kTeCtaCap / 2, true);
  }
  const int wid = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31;
  int2 *tab = tsm + wid * kTeWarpCap;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    te_task(warp_tasks[t], roff, split, radj, te, tab, kTeWarpCap, kTeWarpCap / 2, false);
  }
}

// ------------------------------------------------------------ per-edge / per-vertex sums
// acc[g*8 + 0] S, 1 A4 = sum (da-1)(db-1), 2 A1 = sum t, 3 A2 = sum C(t,2),
// 4 A3 = sum t(da+db-4), 5 K4, 6 C4, 7 sum C(d,2)
__global__ void k_edge_sums(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                            const int32_t *__restrict__ radj, const unsigned *__restrict__ te,
                            const int32_t *__restrict__ gid, unsigned long long *__restrict__ acc) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = lane_id();
  for (int64_t x = warp; x < n; x += nw) {
    const unsigned long long da = (unsigned long long)(roff[x + 1] - roff[x]);
    unsigned long long a4 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int64_t k = split[x] + lane; k < roff[x + 1]; k += 32) {
      int32_t v = radj[k];
      unsigned long long db = (unsigned long long)(roff[v + 1] - roff[v]);
      unsigned long long t = te[k];
      a4 += (da - 1) * (db - 1);
      a1 += t;
      a2 += choose2(t);
      a3 += t * (da + db - 4);
    }
    a4 = warp_sum(a4);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    a3 = warp_sum(a3);
    if (lane == 0) {
      unsigned long long *A = acc + 8 * graph_of(gid, x);
      atomicAdd(&A[0], choose3(da));
      atomicAdd(&A[7], choose2(da));
      if (a4) atomicAdd(&A[1], a4);
      if (a1) atomicAdd(&A[2], a1);
      if (a2) atomicAdd(&A[3], a2);
      if (a3) atomicAdd(&A[4], a3);
    }
  }
}

// ------------------------------------------------------------ 4-cycles
// Task x = highest-rank vertex of the cycle: for a in N(x) with a < x and
// y in N(a) with y < x, cnt[y]++; the task adds sum_y C(cnt[y], 2).
constexpr int kC4WarpCap = 512;  // (key, count) slots per warp -> tasks with bound <= 256

__global__ void k_c4_tasks(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                           const int32_t *__restrict__ radj, int warp_bound, int32_t *__restrict__ cta_tasks,
                           int32_t *__restrict__ warp_tasks, int *__restrict__ sizes) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = lane_id();
  for (int64_t x = warp; x < n; x += nw) {
    unsigned long long b = 0;
    for (int64_t k = roff[x] + lane; k < split[x]; k += 32) {
      int32_t a = radj[k];
      b += (unsigned long long)(roff[a + 1] - roff[a]);
    }
    b = warp_sum(b);
    if (lane == 0 && split[x] - roff[x] >= 2) {
      if (b > (unsigned long long)warp_bound) cta_tasks[atomicAdd(&sizes[0], 1)] = (int32_t)x;
      else warp_tasks[atomicAdd(&sizes[1], 1)] = (int32_t)x;
    }
  }
}

__global__ void __launch_bounds__(256) k_c4(const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                                            const int32_t *__restrict__ radj, const int32_t *__restrict__ gid,
                                            const int64_t *__restrict__ gbase, const int32_t *__restrict__ cta_tasks,
                                            int n_cta, const int32_t *__restrict__ warp_tasks, int n_warp,
                                            int *__restrict__ counters, unsigned *__restrict__ dense,
                                            int64_t dense_len, unsigned long long *__restrict__ acc) {
  __shared__ int2 c4sm[8 * kC4WarpCap];
  __shared__ int s_task;
  const unsigned lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  unsigned *cnt = dense + (int64_t)blockIdx.x * dense_len;
  // hub tasks: per-CTA dense counters in global memory, two passes
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    const int32_t x = cta_tasks[t];
    const int g = graph_of(gid, x);
    const int64_t base = gbase ? gbase[g] : 0;
    const int64_t a0 = roff[x], a1 = split[x];
    for (int pass = 0; pass < 2; ++pass) {
      unsigned long long c = 0;
      for (int64_t k = a0 + wid; k < a1; k += 8) {
        int32_t a = radj[k];
        for (int64_t j = roff[a] + lane; j < roff[a + 1]; j += 32) {
          int32_t y = __ldg(radj + j);
          if (y >= x) break;
          if (pass == 0) atomicAdd(&cnt[y - base], 1u);
          else c += choose2(atomicExch(&cnt[y - base], 0u));
        }
      }
      if (pass == 1) {
        c = warp_sum(c);
        if (lane == 0 && c) atomicAdd(&acc[8 * g + 6], c);
      }
      __syncthreads();
    }
  }
  // tail tasks: shared-memory (key, count) table per warp
  int2 *tab = c4sm + wid * kC4WarpCap;
  for (int i = lane; i < kC4WarpCap; i += 32) tab[i] = make_int2(-1, 0);
  __syncwarp();
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    const int32_t x = warp_tasks[t];
    for (int64_t k = roff[x]; k < split[x]; ++k) {
      int32_t a = radj[k];
      for (int64_t j = roff[a] + lane; j < roff[a + 1]; j += 32) {
        int32_t y = __ldg(radj + j);
        if (y >= x) break;
        uint32_t h = ((uint32_t)y * 2654435769u) >> (32 - 9);
        while (true) {
          int prev = atomicCAS(&tab[h].x, -1, y);
          if (prev == -1 || prev == y) break;
          h = (h + 1) & (kC4WarpCap - 1);
        }
        atomicAdd(&tab[h].y, 1);
      }
    }
    __syncwarp();
    unsigned long long c = 0;
    for (int i = lane; i < kC4WarpCap; i += 32) {
      int2 s = tab[i];
      if (s.x >= 0) {
        c += choose2((unsigned long long)s.y);
        tab[i] = make_int2(-1, 0);
      }
    }
    __syncwarp();
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(&acc[8 * graph_of(gid, x) + 6], c);
  }
}

// ------------------------------------------------------------ combine
__global__ void k_motif_combine(int ngraphs, const unsigned long long *__restrict__ acc,
                                unsigned long long *__restrict__ out /* ngraphs x 8 */) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngraphs; g += gridDim.x * blockDim.x) {
    const unsigned long long *A = acc + 8 * g;
    unsigned long long T = A[2] / 3, S = A[0], P = A[1] - 3 * T, TT = A[4] / 2, D = A[3], C = A[6], K = A[5];
    unsigned long long k = K, d = D - 6 * K, c = C - d - 3 * K, tt = TT - 4 * d - 12 * K;
    unsigned long long p = P - 2 * tt - 4 * c - 6 * d - 12 * K, s = S - tt - 2 * d - 4 * K;
    unsigned long long *o = out + 8 * g;
    o[0] = A[7] - 3 * T;  // induced 2-paths
    o[1] = T;
    o[2] = s;
    o[3] = p;
    o[4] = tt;
    o[5] = c;
    o[6] = d;
    o[7] = k;
  }
}

// ------------------------------------------------------------ pipeline
__global__ void k_up_len(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                         int64_t *__restrict__ len) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x)
    len[x] = roff[x + 1] - split[x];
}
__global__ void k_up_copy(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                          const int32_t *__restrict__ radj, const int64_t *__restrict__ doff,
                          int32_t *__restrict__ dadj) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t x = warp; x < n; x += nw)
    for (int64_t k = split[x] + lane_id(); k < roff[x + 1]; k += 32) dadj[doff[x] + (k - split[x])] = radj[k];
}
// tasks of the per-edge triangle pass: vertices with >= 2 upward neighbours
__global__ void k_te_tasks(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                           int cta_min, int32_t *__restrict__ cta_tasks, int32_t *__restrict__ warp_tasks,
                           int *__restrict__ sizes) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    int64_t d = roff[x + 1] - split[x];
    if (d < 2) continue;
    if (d > cta_min) cta_tasks[atomicAdd(&sizes[0], 1)] = (int32_t)x;
    else warp_tasks[atomicAdd(&sizes[1], 1)] = (int32_t)x;
  }
}

// The upward parts of a rank-ordered symmetric graph as a CSR of its own
// (the degree-oriented DAG, every list pointing to larger ids).
static int dag_from_split(int64_t n, const int64_t *roff, const int64_t *split, const int32_t *radj,
                          DevBuf<int64_t> &doff, DevBuf<int32_t> &dadj, int *max_deg, cudaStream_t st) {
  DevBuf<int64_t> len;
  GPM_TRY(len.reserve(n));
  GPM_TRY(doff.reserve(n + 1));
  if (n > 0) k_up_len<<<grid_for(n), 256, 0, st>>>(n, roff, split, len.p);
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, len.p, doff.p + 1, (int)n, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cudaMemsetAsync(doff.p, 0, sizeof(int64_t), st));
  if (n > 0) GPM_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, len.p, doff.p + 1, (int)n, st));
  int64_t m = 0;
  GPM_CUDA(cudaMemcpyAsync(&m, doff.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  DevBuf<int64_t> mx;
  GPM_TRY(mx.reserve(1));
  size_t tmp2 = 0;
  GPM_CUDA(cub::DeviceReduce::Max(nullptr, tmp2, len.p, mx.p, (int)std::max<int64_t>(n, 1), st));
  DevBuf<char> t2;
  GPM_TRY(t2.reserve(tmp2));
  int64_t hmx = 0;
  if (n > 0) {
    GPM_CUDA(cub::DeviceReduce::Max(t2.p, tmp2, len.p, mx.p, (int)n, st));
    GPM_CUDA(cudaMemcpyAsync(&hmx, mx.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  }
  GPM_CUDA(cudaStreamSynchronize(st));
  GPM_TRY(dadj.reserve(std::max<int64_t>(m, 1)));
  if (n > 0) k_up_copy<<<grid_for(n * 32), 256, 0, st>>>(n, roff, split, radj, doff.p, dadj.p);
  *max_deg = (int)hmx;
  return GPM_OK;
}

static int te_grid() {
  static int grid = 0;
  if (!grid) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edge_tri, 256, kTeSmem);
    grid = std::max(1, per_sm) * num_sms();
  }
  return grid;
}

// Builds every schedule and scratch buffer of the pipeline (host syncs and
// allocations happen here, never in motif_plan_run).
int motif_plan_build(const MotifInput &in, MotifPlan *p, cudaStream_t st) {
  p->in = in;
  const int64_t n = in.n;
  const int64_t *roff = in.roff;
  const int32_t *radj = in.radj;
  GPM_TRY(p->acc.reserve(8 * (size_t)in.ngraphs));
  GPM_TRY(p->out.reserve(8 * (size_t)in.ngraphs));
  GPM_TRY(p->split.reserve(n));
  if (n > 0) k_split<<<grid_for(n), 256, 0, st>>>(n, roff, radj, p->split.p);
  GPM_TRY(dag_from_split(n, roff, p->split.p, radj, p->doff, p->dadj, &p->dag_max, st));
  GPM_TRY(p->te.reserve(std::max<int64_t>(in.nnz, 1)));
  // queues of the per-edge triangle pass and of the 4-cycle pass
  DevBuf<int> sizes;
  GPM_TRY(sizes.reserve(4));
  GPM_TRY(p->te_ct.reserve(n));
  GPM_TRY(p->te_wt.reserve(n));
  GPM_TRY(p->c4_ct.reserve(n));
  GPM_TRY(p->c4_wt.reserve(n));
  GPM_TRY(p->te_counters.reserve(2));
  GPM_TRY(p->c4_counters.reserve(2));
  GPM_CUDA(cudaMemsetAsync(sizes.p, 0, 4 * sizeof(int), st));
  if (n > 0) {
    k_te_tasks<<<grid_for(n), 256, 0, st>>>(n, roff, p->split.p, std::min(in.te_cta_min, kTeWarpCap / 2), p->te_ct.p, p->te_wt.p, sizes.p);
    k_c4_tasks<<<grid_for(n * 32), 256, 0, st>>>(n, roff, p->split.p, radj, std::min(in.c4_warp_bound, kC4WarpCap / 2), p->c4_ct.p, p->c4_wt.p, sizes.p + 2);
  }
  int h[4];
  GPM_CUDA(cudaMemcpyAsync(h, sizes.p, sizeof h, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  p->te_nc = h[0];
  p->te_nw = h[1];
  p->c4_nc = h[2];
  p->c4_nw = h[3];
  p->te_grid = te_grid();
  p->c4_grid = 2 * num_sms();
  // per-CTA dense 4-cycle counters over the largest member graph; kept zero
  // between runs (the second pass of k_c4 clears what the first set)
  p->dense_len = std::max<int64_t>(in.max_graph_n, 1);
  GPM_TRY(p->dense.reserve((size_t)p->dense_len * p->c4_grid));
  GPM_CUDA(cudaMemsetAsync(p->dense.p, 0, sizeof(unsigned) * (size_t)p->dense_len * p->c4_grid, st));
  GPM_TRY(clique_plan_build(&p->k4, n, p->doff.p, p->dadj.p, p->dag_max, 4, in.gid, p->acc.p, 8, 5, st,
                            in.cq_warp_max));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

// Launches only (capturable): zero the sums, triangles per edge, per-edge
// and per-vertex sums, 4-cycles, 4-cliques, inversion.
int motif_plan_run(MotifPlan *p, cudaStream_t st) {
  const MotifInput &in = p->in;
  const int64_t n = in.n;
  GPM_CUDA(cudaMemsetAsync(p->acc.p, 0, sizeof(unsigned long long) * 8 * in.ngraphs, st));
  GPM_CUDA(cudaMemsetAsync(p->te.p, 0, sizeof(unsigned) * std::max<int64_t>(in.nnz, 1), st));
  GPM_CUDA(cudaMemsetAsync(p->te_counters.p, 0, 2 * sizeof(int), st));
  GPM_CUDA(cudaMemsetAsync(p->c4_counters.p, 0, 2 * sizeof(int), st));
  if (p->te_nc + p->te_nw > 0)
    k_edge_tri<<<p->te_grid, 256, kTeSmem, st>>>(in.roff, p->split.p, in.radj, p->te_ct.p, p->te_nc, p->te_wt.p,
                                                 p->te_nw, p->te_counters.p, p->te.p);
  if (n > 0)
    k_edge_sums<<<grid_for(n * 32), 256, 0, st>>>(n, in.roff, p->split.p, in.radj, p->te.p, in.gid, p->acc.p);
  if (p->c4_nc + p->c4_nw > 0)
    k_c4<<<p->c4_grid, 256, 0, st>>>(in.roff, p->split.p, in.radj, in.gid, in.gbase, p->c4_ct.p, p->c4_nc,
                                     p->c4_wt.p, p->c4_nw, p->c4_counters.p, p->dense.p, p->dense_len, p->acc.p);
  GPM_LAUNCH_CHECK();
  GPM_TRY(clique_plan_run(&p->k4, st));
  k_motif_combine<<<std::max(1, (in.ngraphs + 255) / 256), 256, 0, st>>>(in.ngraphs, p->acc.p, p->out.p);
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

int motif_plan_run_stage(MotifPlan *p, int stage, cudaStream_t st) {
  const MotifInput &in = p->in;
  if (stage == 0) {
    GPM_CUDA(cudaMemsetAsync(p->te.p, 0, sizeof(unsigned) * std::max<int64_t>(in.nnz, 1), st));
    GPM_CUDA(cudaMemsetAsync(p->te_counters.p, 0, 2 * sizeof(int), st));
    if (p->te_nc + p->te_nw > 0)
      k_edge_tri<<<p->te_grid, 256, kTeSmem, st>>>(in.roff, p->split.p, in.radj, p->te_ct.p, p->te_nc, p->te_wt.p,
                                                   p->te_nw, p->te_counters.p, p->te.p);
  } else if (stage == 1) {
    GPM_CUDA(cudaMemsetAsync(p->c4_counters.p, 0, 2 * sizeof(int), st));
    if (p->c4_nc + p->c4_nw > 0)
      k_c4<<<p->c4_grid, 256, 0, st>>>(in.roff, p->split.p, in.radj, in.gid, in.gbase, p->c4_ct.p, p->c4_nc,
                                       p->c4_wt.p, p->c4_nw, p->c4_counters.p, p->dense.p, p->dense_len, p->acc.p);
  } else {
    GPM_TRY(clique_plan_run(&p->k4, st));
  }
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

}  // namespace gpm

using namespace gpm;

extern "C" int gpm_motif(gpm_graph *g, int k, uint64_t *out) {
  if (!g || !out) return fail(GPM_EINVAL, "gpm_motif: NULL argument");
  if (k != 3 && k != 4) return fail(GPM_EUNSUPPORTED, "motif size must be 3 or 4");
  if (g->oriented) return fail(GPM_EINVAL, "motif counting needs the symmetric (unoriented) graph");
  GPM_TRY(ensure_rank_graph(g, 0));
  MotifInput in;
  in.n = g->n;
  in.nnz = g->nnz;
  in.roff = g->rg->roff.p;
  in.radj = g->rg->radj.p;
  in.max_graph_n = g->n;
  MotifPlan plan;
  GPM_TRY(motif_plan_build(in, &plan, 0));
  GPM_TRY(motif_plan_run(&plan, 0));
  unsigned long long h[8];
  GPM_CUDA(cudaMemcpy(h, plan.out.p, sizeof h, cudaMemcpyDeviceToHost));
  if (k == 3) {
    out[0] = h[0];
    out[1] = h[1];
  } else {
    for (int i = 0; i < 6; ++i) out[i] = h[2 + i];
  }
  return GPM_OK;
}
