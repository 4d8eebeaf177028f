// tc.cu -- triangle counting (TCSolver, src/TCSolver.cuh:9-121).
//
// Every variant computes  T = sum over stored u->v of |N(u) & N(v)|  exactly
// (uint64).  On a degree-oriented DAG that is the triangle count.
//
//  * BSEARCH: warp per stored edge (the shape of the reference's e-centric
//    lambda, TCSolver.cuh:27-59): the shorter list's keys are looked up in
//    the longer list by binary search.
//  * MERGE: warp per stored edge; the shorter list is cut into 32 runs and
//    each lane merges its run against the matching window of the longer one.
//  * HASH: vertex tasks (the reference's tc_hi_warp_vertex idea,
//    tc_hi_warp_vertex.cuh:37-116, redesigned): N(u) goes into a
//    shared-memory open-addressing table, then the 2-hop lists N(v), v in
//    N(u), are streamed flattened (one coalesced element per lane per step,
//    no idle lanes on short lists) and probed.  Hubs (deg > cta_threshold)
//    are CTA tasks, the tail are warp tasks; both queues are drained by a
//    persistent grid through atomic work counters.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "tc.cuh"
#include "tc_rank.cuh"

namespace gpm {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ uint32_t hash_slot(int32_t key, int logcap) {
  return ((uint32_t)key * 2654435769u) >> (32 - logcap);
}

// lower bound in a sorted global list
__device__ __forceinline__ int64_t lower_bound_g(const int32_t *__restrict__ a, int64_t n, int32_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool bsearch_g(const int32_t *__restrict__ a, int64_t n, int32_t key) {
  int64_t lo = 0, hi = n - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) >> 1;
    int32_t x = __ldg(a + mid);
    if (x == key) return true;
    if (x < key) lo = mid + 1; else hi = mid - 1;
  }
  return false;
}

// ------------------------------------------------------------------ BSEARCH
__global__ void __launch_bounds__(256) k_tc_bsearch(int64_t nnz, const int64_t *__restrict__ off,
                                                    const int32_t *__restrict__ adj,
                                                    const int32_t *__restrict__ src,
                                                    unsigned long long *__restrict__ out) {
  const unsigned lane = lane_id();
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long c = 0;
  for (int64_t e = warp; e < nnz; e += nw) {
    int32_t u = src[e], v = adj[e];
    int64_t su = off[u], du = off[u + 1] - su;
    int64_t sv = off[v], dv = off[v + 1] - sv;
    const int32_t *look = adj + su, *srch = adj + sv;
    int64_t nl = du, ns = dv;
    if (du > dv) { look = adj + sv; srch = adj + su; nl = dv; ns = du; }
    for (int64_t i = lane; i < nl; i += 32) c += bsearch_g(srch, ns, __ldg(look + i));
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

// ------------------------------------------------------------------ MERGE
__global__ void __launch_bounds__(256) k_tc_merge(int64_t nnz, const int64_t *__restrict__ off,
                                                  const int32_t *__restrict__ adj,
                                                  const int32_t *__restrict__ src,
                                                  unsigned long long *__restrict__ out) {
  const unsigned lane = lane_id();
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long c = 0;
  for (int64_t e = warp; e < nnz; e += nw) {
    int32_t u = src[e], v = adj[e];
    int64_t su = off[u], du = off[u + 1] - su;
    int64_t sv = off[v], dv = off[v + 1] - sv;
    const int32_t *a = adj + su, *b = adj + sv;
    int64_t na = du, nb = dv;
    if (du > dv) { a = adj + sv; b = adj + su; na = dv; nb = du; }
    if (na == 0) continue;
    // lane's run of the short list
    int64_t per = (na + 31) >> 5;
    int64_t i0 = lane * per, i1 = min(na, i0 + per);
    if (i0 >= i1) continue;
    int64_t j = lower_bound_g(b, nb, __ldg(a + i0));
    int64_t i = i0;
    while (i < i1 && j < nb) {
      int32_t x = __ldg(a + i), y = __ldg(b + j);
      if (x < y) ++i;
      else if (y < x) ++j;
      else { ++c; ++i; ++j; }
    }
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

// ------------------------------------------------------------------ HASH
// Shared memory of one CTA (TC_SMEM bytes), used either whole for a CTA task
// or split into 8 equal per-warp regions for warp tasks.
//   CTA region : table[2048] int32 | pre[1024] int64 | base[1024] int64
//   warp region: table[256]  int32 | pre[128]  int64 | base[128]  int64
constexpr int kCtaTable = 2048, kCtaChunk = 1024;
constexpr int kWarpTable = 256, kWarpChunk = 128;
constexpr int kWarps = 8;
constexpr size_t kCtaBytes = kCtaTable * 4 + kCtaChunk * 16;
constexpr size_t kWarpBytes = kWarpTable * 4 + kWarpChunk * 16;
static_assert(kWarpBytes * kWarps == kCtaBytes, "CTA and warp layouts share one region");
constexpr size_t TC_SMEM = kCtaBytes;

// Probe flattened indices [x_lo, x_hi) of the staged 2-hop lists with a
// stride of `stride` starting at x_lo + t.  pre[] is the inclusive prefix of
// the staged list lengths, base[i] = start(i) - exclusive prefix(i), so the
// element of flattened index x in segment i is adj[base[i] + x].
__device__ __forceinline__ unsigned long long probe_range(
    const int32_t *__restrict__ adj, const int32_t *tab, int logcap, const int64_t *pre,
    const int64_t *base, int nseg, int64_t x_lo, int64_t x_hi, int seg, int t, int stride) {
  unsigned long long c = 0;
  const uint32_t mask = (1u << logcap) - 1u;
  for (int64_t x = x_lo + t; x < x_hi; x += stride) {
    while (seg < nseg && pre[seg] <= x) ++seg;
    int32_t w = __ldg(adj + base[seg] + x);
    uint32_t h = hash_slot(w, logcap);
    while (true) {
      int32_t k = tab[h];
      if (k == w) { ++c; break; }
      if (k < 0) break;
      h = (h + 1) & mask;
    }
  }
  return c;
}

// first index i in [0, n) with pre[i] > x
__device__ __forceinline__ int upper_seg(const int64_t *pre, int n, int64_t x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (pre[mid] <= x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int ceil_log2(int x) { return x <= 1 ? 0 : 32 - __clz(x - 1); }

// One hub task on the whole CTA.  Chunked so any degree fits: each chunk of
// N(u) (<= kCtaChunk keys) is probed by every chunk of staged 2-hop lists.
__device__ unsigned long long cta_task(int32_t u, const int64_t *__restrict__ off,
                                       const int32_t *__restrict__ adj, char *smem) {
  int32_t *tab = reinterpret_cast<int32_t *>(smem);
  int64_t *pre = reinterpret_cast<int64_t *>(smem + kCtaTable * 4);
  int64_t *base = pre + kCtaChunk;
  __shared__ int64_t s_carry[kWarps + 1];
  const int tid = threadIdx.x, nthr = blockDim.x, warp = tid >> 5, lane = tid & 31;
  const int64_t s0 = off[u];
  const int d = (int)(off[u + 1] - s0);
  unsigned long long c = 0;
  for (int t0 = 0; t0 < d; t0 += kCtaChunk) {
    const int tk = min(kCtaChunk, d - t0);
    const int logcap = max(5, ceil_log2(2 * tk));
    const int cap = 1 << logcap;
    const uint32_t mask = cap - 1;
    __syncthreads();
    for (int i = tid; i < cap; i += nthr) tab[i] = -1;
    __syncthreads();
    for (int i = tid; i < tk; i += nthr) {
      int32_t key = adj[s0 + t0 + i];
      uint32_t h = hash_slot(key, logcap);
      while (atomicCAS(&tab[h], -1, key) != -1) h = (h + 1) & mask;
    }
    for (int v0 = 0; v0 < d; v0 += kCtaChunk) {
      const int vk = min(kCtaChunk, d - v0);
      __syncthreads();
      // stage lengths with a CTA-wide inclusive scan (warp scans + carries)
      for (int i0 = 0; i0 < vk; i0 += nthr) {
        int i = i0 + tid;
        int64_t len = 0, st = 0;
        if (i < vk) {
          int32_t v = adj[s0 + v0 + i];
          st = off[v];
          len = off[v + 1] - st;
        }
        int64_t x = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          int64_t y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (lane == 31) s_carry[warp + 1] = x;
        __syncthreads();
        if (tid == 0) {
          int64_t run = i0 == 0 ? 0 : pre[i0 - 1];
          s_carry[0] = run;
          for (int w = 1; w <= nthr / 32; ++w) {
            run += s_carry[w];
            s_carry[w] = run;
          }
        }
        __syncthreads();
        int64_t incl = s_carry[warp] + x;
        if (i < vk) {
          pre[i] = incl;
          base[i] = st - (incl - len);
        }
        __syncthreads();
      }
      const int64_t W = pre[vk - 1];
      // each warp takes an equal share of the flattened work
      const int nwarps = nthr >> 5;
      int64_t lo = W * warp / nwarps, hi = W * (warp + 1) / nwarps;
      if (lo < hi) {
        int seg = upper_seg(pre, vk, lo);
        c += probe_range(adj, tab, logcap, pre, base, vk, lo, hi, seg, lane, 32);
      }
    }
  }
  __syncthreads();
  return c;
}

// One tail task on one warp (deg <= kWarpChunk).
__device__ unsigned long long warp_task(int32_t u, const int64_t *__restrict__ off,
                                        const int32_t *__restrict__ adj, char *region) {
  int32_t *tab = reinterpret_cast<int32_t *>(region);
  int64_t *pre = reinterpret_cast<int64_t *>(region + kWarpTable * 4);
  int64_t *base = pre + kWarpChunk;
  const int lane = lane_id();
  const int64_t s0 = off[u];
  const int d = (int)(off[u + 1] - s0);
  const int logcap = max(5, ceil_log2(2 * d));
  const int cap = 1 << logcap;
  const uint32_t mask = cap - 1;
  for (int i = lane; i < cap; i += 32) tab[i] = -1;
  __syncwarp();
  int64_t carry = 0;
  for (int i0 = 0; i0 < d; i0 += 32) {
    int i = i0 + lane;
    int64_t len = 0, st = 0;
    if (i < d) {
      int32_t v = adj[s0 + i];
      uint32_t h = hash_slot(v, logcap);
      while (atomicCAS(&tab[h], -1, v) != -1) h = (h + 1) & mask;
      st = off[v];
      len = off[v + 1] - st;
    }
    int64_t x = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    int64_t incl = carry + x;
    if (i < d) {
      pre[i] = incl;
      base[i] = st - (incl - len);
    }
    carry = __shfl_sync(0xffffffffu, incl, 31);
  }
  __syncwarp();
  unsigned long long c = probe_range(adj, tab, logcap, pre, base, d, 0, carry, 0, lane, 32);
  __syncwarp();
  return c;
}

__global__ void __launch_bounds__(256) k_tc_hash(const int64_t *__restrict__ off,
                                                 const int32_t *__restrict__ adj,
                                                 const int32_t *__restrict__ cta_tasks, int n_cta,
                                                 const int32_t *__restrict__ warp_tasks, int n_warp,
                                                 int *__restrict__ counters,
                                                 unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) char smem[];
  __shared__ int s_task;
  unsigned long long c = 0;
  // hub queue: one task per CTA at a time
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    c += cta_task(cta_tasks[t], off, adj, smem);
  }
  // tail queue: one task per warp at a time
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  char *region = smem + warp * kWarpBytes;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    c += warp_task(warp_tasks[t], off, adj, region);
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

// Task split by degree (the reference's USE_WARP / USE_CTA thresholds).
__global__ void k_tc_split(int64_t n, const int64_t *__restrict__ off, int warp_min, int cta_min,
                           int32_t *__restrict__ cta_tasks, int32_t *__restrict__ warp_tasks,
                           int *__restrict__ sizes) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    int64_t d = off[u + 1] - off[u];
    if (d < warp_min) continue;
    if (d >= cta_min) cta_tasks[atomicAdd(&sizes[0], 1)] = (int32_t)u;
    else warp_tasks[atomicAdd(&sizes[1], 1)] = (int32_t)u;
  }
}

// ------------------------------------------------------------------ plan
void free_tc_plan(TcPlan *p) { delete p; }

int tc_hash_grid() {
  static PerDevice grid;
  return grid.get([] {
    int per_sm = 0;
    cudaFuncSetAttribute(k_tc_hash, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_hash, 256, TC_SMEM);
    return std::max(1, per_sm) * num_sms();
  });
}

int tc_build_plan(gpm_graph *g, int warp_min, int cta_min, cudaStream_t st) {
  if (g->tc && g->tc->warp_min == warp_min && g->tc->cta_min == cta_min) return GPM_OK;
  free_tc_plan(g->tc);
  g->tc = nullptr;
  TcPlan *p = new TcPlan();
  p->warp_min = warp_min;
  p->cta_min = cta_min;
  int64_t n = g->n;
  int s = GPM_OK;
  if ((s = p->cta_tasks.reserve(n)) || (s = p->warp_tasks.reserve(n)) || (s = p->counters.reserve(4)) ||
      (s = p->sizes.reserve(2))) {
    delete p;
    return s;
  }
  cudaMemsetAsync(p->sizes.p, 0, 2 * sizeof(int), st);
  if (n > 0) {
    int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8);
    k_tc_split<<<grid, 256, 0, st>>>(n, g->off.p, warp_min, cta_min, p->cta_tasks.p, p->warp_tasks.p, p->sizes.p);
  }
  int h[2] = {0, 0};
  cudaMemcpyAsync(h, p->sizes.p, sizeof h, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete p;
    return fail(GPM_ECUDA, std::string("tc plan: ") + cudaGetErrorString(e));
  }
  p->n_cta = h[0];
  p->n_warp = h[1];
  g->tc = p;
  return GPM_OK;
}

int tc_launch(gpm_graph *g, int variant, cudaStream_t st, unsigned long long *d_out) {
  GPM_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
  if (g->nnz == 0) return GPM_OK;
  if (variant == GPM_TC_BSEARCH || variant == GPM_TC_MERGE) {
    GPM_TRY(ensure_src(g, st));
    int grid = num_sms() * 8;
    if (variant == GPM_TC_BSEARCH)
      k_tc_bsearch<<<grid, 256, 0, st>>>(g->nnz, g->off.p, g->adj.p, g->src.p, d_out);
    else
      k_tc_merge<<<grid, 256, 0, st>>>(g->nnz, g->off.p, g->adj.p, g->src.p, d_out);
    GPM_LAUNCH_CHECK();
    return GPM_OK;
  }
  if (variant == GPM_TC_HASH) {
    // reference thresholds: USE_WARP = 2, USE_CTA = 100 (tuning_schedules.cuh:196-197)
    GPM_TRY(tc_build_plan(g, 2, 101, st));
    TcPlan *p = g->tc;
    if (p->cta_min - 1 > kWarpChunk) return fail(GPM_EINVAL, "warp tasks exceed the warp table");
    GPM_CUDA(cudaMemsetAsync(p->counters.p, 0, 4 * sizeof(int), st));
    k_tc_hash<<<tc_hash_grid(), 256, TC_SMEM, st>>>(g->off.p, g->adj.p, p->cta_tasks.p, p->n_cta,
                                                    p->warp_tasks.p, p->n_warp, p->counters.p, d_out);
    GPM_LAUNCH_CHECK();
    return GPM_OK;
  }
  if (variant == GPM_TC_BITMAP) return rank_launch(g, st, d_out);
  return fail(GPM_EINVAL, "unknown triangle-count variant " + std::to_string(variant));
}

}  // namespace gpm

using namespace gpm;

extern "C" {

int gpm_tc_async(gpm_graph *g, int variant, void *stream, uint64_t *d_out) {
  if (!g || !d_out) return fail(GPM_EINVAL, "gpm_tc_async: NULL argument");
  if (variant == GPM_TC_AUTO) variant = GPM_TC_BITMAP;
  if (variant == GPM_TC_LEARNED) return tc_learned_launch(g, (cudaStream_t)stream, (unsigned long long *)d_out);
  return tc_launch(g, variant, (cudaStream_t)stream, (unsigned long long *)d_out);
}

int gpm_tc(gpm_graph *g, int mode, uint64_t *out) {
  if (!g || !out) return fail(GPM_EINVAL, "gpm_tc: NULL argument");
  if (mode != GPM_V_CENTRIC && mode != GPM_E_CENTRIC) return fail(GPM_EINVAL, "Wrong Calculation Mode.");
  GPM_TRY(g->result.reserve(8));
  int variant = mode == GPM_V_CENTRIC ? GPM_TC_HASH : GPM_TC_BSEARCH;
  GPM_TRY(tc_launch(g, variant, 0, (unsigned long long *)g->result.p));
  GPM_CUDA(cudaMemcpy(out, g->result.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return GPM_OK;
}

int gpm_tc_host_csr(int64_t n, const int64_t *offsets, const int32_t *indices, int variant,
                    void *stream, uint64_t *out) {
  if (!offsets || !out || n < 0) return fail(GPM_EINVAL, "gpm_tc_host_csr: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  GPM_TRY(ensure_device());
  int64_t nnz = offsets[n];
  // every buffer below comes from this thread's reusable device pool; all
  // work runs on `st` and is synchronised before returning
  ArenaScope pool;
  gpm_graph g;
  g.n = n;
  g.nnz = nnz;
  GPM_TRY(g.off.reserve(n + 1));
  GPM_TRY(g.adj.reserve(nnz));
  GPM_CUDA(cudaMemcpyAsync(g.off.p, offsets, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
  if (variant == GPM_TC_AUTO) variant = GPM_TC_BITMAP;
  if (variant == GPM_TC_BITMAP || variant == GPM_TC_LEARNED) {
    // orientation folded into the rank relabel, the adjacency uploaded in
    // chunks that are relabelled as they land
    GPM_TRY(build_upward_rank_graph(&g, st, offsets, indices));
    g.oriented = 1;
  } else {
    if (nnz > 0) GPM_CUDA(cudaMemcpyAsync(g.adj.p, indices, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
    GPM_TRY(orient_on_stream(&g, st));
  }
  GPM_TRY(g.result.reserve(8));
  if (variant == GPM_TC_LEARNED) GPM_TRY(tc_learned_launch(&g, st, (unsigned long long *)g.result.p));
  else GPM_TRY(tc_launch(&g, variant, st, (unsigned long long *)g.result.p));
  GPM_CUDA(cudaMemcpyAsync(out, g.result.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Triangle count without any allocation.
//
// Some callers cannot allocate device memory at all: code running inside a
// framework that owns every byte of the device through its own pool, hosts
// that forbid allocation after start-up (real-time and embedded services),
// and callers that must not trigger the implicit synchronisation a
// cudaMalloc/cudaFree can cause.  For them the hash-kernel triangle count
// below keeps its scratch -- the hub and tail task queues, their sizes and
// the two work cursors -- in one file-scope __device__ array of fixed size,
// so the call performs no cudaMalloc, cudaFree or other allocating call.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxVertices (1,048,576) vertices; larger graphs are
//     rejected with GPM_EINVAL before anything is launched;
//   * the array (8 MiB + 256 B) is part of this library's device image, so
//     every GPU that loads the library keeps it until the process exits;
//   * every call shares the array: the call clears the parts that must
//     start at zero itself, but calls whose work overlaps on the GPU (two
//     streams, or two host threads) race on it and must be serialised by the
//     caller;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.
// ---------------------------------------------------------------------------
#include <mutex>

namespace gpm {

constexpr int64_t kNoAllocMaxVertices = 1 << 20;
constexpr int kNoAllocHeader = 64;  // words: [0..1] queue sizes, [16..19] work cursors
static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocHeader + 2 * kNoAllocMaxVertices];

// In host code the array's name is only a stand-in for its device address,
// so the address is looked up once per device and kept here.
constexpr int kNoAllocMaxDevices = 64;
static int32_t *g_noalloc_ptr[kNoAllocMaxDevices];
static int g_noalloc_grid[kNoAllocMaxDevices];  // resident CTAs of k_tc_hash_noalloc x SMs, per device
static std::mutex g_noalloc_mu;

__global__ void __launch_bounds__(256) k_tc_hash_noalloc(const int64_t *__restrict__ off,
                                                         const int32_t *__restrict__ adj,
                                                         const int32_t *__restrict__ cta_tasks,
                                                         const int32_t *__restrict__ warp_tasks,
                                                         const int *__restrict__ sizes, int *__restrict__ counters,
                                                         unsigned long long *__restrict__ out);

static int noalloc_scratch(int32_t **out, int *grid) {
  int dev = 0;
  GPM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(GPM_EUNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(GPM_ECUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_hash_noalloc, 256, TC_SMEM);
    g_noalloc_grid[dev] = std::max(1, per_sm) * num_sms();
    g_noalloc_ptr[dev] = static_cast<int32_t *>(p);
  }
  *out = g_noalloc_ptr[dev];
  *grid = g_noalloc_grid[dev];
  return GPM_OK;
}

// k_tc_hash with the queue sizes read from device memory, so no host round
// trip (and no host-visible buffer) is needed between the split and the count.
__global__ void __launch_bounds__(256) k_tc_hash_noalloc(const int64_t *__restrict__ off,
                                                         const int32_t *__restrict__ adj,
                                                         const int32_t *__restrict__ cta_tasks,
                                                         const int32_t *__restrict__ warp_tasks,
                                                         const int *__restrict__ sizes, int *__restrict__ counters,
                                                         unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) char smem[];
  __shared__ int s_task;
  const int n_cta = sizes[0], n_warp = sizes[1];
  unsigned long long c = 0;
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    c += cta_task(cta_tasks[t], off, adj, smem);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  char *region = smem + warp * kWarpBytes;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    c += warp_task(warp_tasks[t], off, adj, region);
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

}  // namespace gpm

extern "C" int gpm_tc_csr_noalloc(int64_t n, const int64_t *d_offsets, const int32_t *d_indices, void *stream,
                                  uint64_t *d_out) {
  if (n < 0 || !d_offsets || !d_out || (n > 0 && !d_indices))
    return fail(GPM_EINVAL, "gpm_tc_csr_noalloc: bad argument");
  if (n > kNoAllocMaxVertices)
    return fail(GPM_EINVAL, "gpm_tc_csr_noalloc: " + std::to_string(n) +
                                " vertices exceed the 1048576-vertex limit of the no-allocation entry point");
  cudaStream_t st = (cudaStream_t)stream;
  int32_t *scratch = nullptr;
  int hash_grid = 0;
  GPM_TRY(noalloc_scratch(&scratch, &hash_grid));
  int *sizes = scratch, *counters = scratch + 16;
  int32_t *cta_tasks = scratch + kNoAllocHeader, *warp_tasks = cta_tasks + kNoAllocMaxVertices;
  GPM_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int32_t) * kNoAllocHeader, st));
  GPM_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint64_t), st));
  if (n == 0) return GPM_OK;
  // same split as the allocating path: USE_WARP = 2, USE_CTA = 100
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8);
  k_tc_split<<<grid, 256, 0, st>>>(n, d_offsets, 2, 101, cta_tasks, warp_tasks, sizes);
  GPM_LAUNCH_CHECK();
  k_tc_hash_noalloc<<<hash_grid, 256, TC_SMEM, st>>>(d_offsets, d_indices, cta_tasks, warp_tasks, sizes,
                                                              counters, (unsigned long long *)d_out);
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}
