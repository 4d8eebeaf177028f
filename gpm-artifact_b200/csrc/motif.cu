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
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "motif.cuh"
#include "tc_rank.cuh"

namespace gpm {

namespace cg = cooperative_groups;

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
constexpr int kC4CtaSlots = 8 * kC4WarpCap;  // a hub task's shared table: the 8 warps' tables together
// Hub tasks have a 2-hop bound of at most kC4HubMax (larger ones go to
// k_c4_big), so at most that many distinct keys meet kC4CtaSlots slots: the
// table never fills and every probe sequence ends.
constexpr long long kC4HubMax = kC4CtaSlots * 3 / 4;
static_assert(kC4HubMax < kC4CtaSlots, "a hub task's keys must leave its table a free slot: c4_slot never fails");

// Slot of y in a hub task's shared table, found or newly claimed.
__device__ __forceinline__ int c4_slot(int2 *tab, int32_t y) {
  uint32_t h = ((uint32_t)y * 2654435769u) >> (32 - 12);
  for (int p = 0; p < kC4CtaSlots; ++p) {
    int cur = tab[h].x;
    if (cur == -1) {
      cur = atomicCAS(&tab[h].x, -1, y);
      if (cur == -1) cur = y;
    }
    if (cur == y) return (int)h;
    h = (h + 1) & (kC4CtaSlots - 1);
  }
  return -1;
}

// Empties a (key, count) table of `slots` entries (16-byte aligned, slots
// even) with 16-byte stores.  Counts need no scan before it: every increment
// adds the counter's old value to the task's sum (C(c+1,2) - C(c,2) = c).
__device__ __forceinline__ void c4_reset(int2 *tab, int slots, int t, int nt) {
  uint4 *v = reinterpret_cast<uint4 *>(tab);
  for (int i = t; i < slots / 2; i += nt) v[i] = make_uint4(0xffffffffu, 0u, 0xffffffffu, 0u);
}

__global__ void k_c4_tasks(int64_t n, const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                           const int32_t *__restrict__ radj, int warp_bound, long long big_min,
                           int32_t *__restrict__ cta_tasks, int32_t *__restrict__ warp_tasks,
                           int32_t *__restrict__ big_tasks, unsigned long long *__restrict__ big_b,
                           int *__restrict__ sizes) {
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
    const int64_t dx = split[x] - roff[x];
    if (lane == 0 && dx >= 2) {
      if (b > (unsigned long long)big_min) {
        const int i = atomicAdd(&sizes[2], 1);
        big_tasks[i] = (int32_t)x;
        big_b[i] = b;
        atomicMax(&sizes[3], (int)dx);
      } else if (b > (unsigned long long)warp_bound) {
        cta_tasks[atomicAdd(&sizes[0], 1)] = (int32_t)x;
      } else {
        warp_tasks[atomicAdd(&sizes[1], 1)] = (int32_t)x;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_c4(const int64_t *__restrict__ roff, const int64_t *__restrict__ split,
                                            const int32_t *__restrict__ radj, const int32_t *__restrict__ gid,
                                            const int64_t *__restrict__ gbase, const int32_t *__restrict__ cta_tasks,
                                            int n_cta, const int32_t *__restrict__ warp_tasks, int n_warp,
                                            int *__restrict__ counters, unsigned long long *__restrict__ acc) {
  __shared__ __align__(16) int2 c4sm[8 * kC4WarpCap];
  __shared__ int s_task;
  const unsigned lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  // hub tasks: counters in a shared-memory hash table over the 8 warps' tables
  static_assert(kC4CtaSlots == 4096, "c4_slot hashes to 12 bits");
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    const int32_t x = cta_tasks[t];
    const int g = graph_of(gid, x);
    const int64_t a0 = roff[x], a1 = split[x];
    c4_reset(c4sm, kC4CtaSlots, threadIdx.x, blockDim.x);
    __syncthreads();
    unsigned long long c = 0;
    for (int64_t k = a0 + wid; k < a1; k += 8) {
      int32_t a = radj[k];
      for (int64_t j = roff[a] + lane; j < roff[a + 1]; j += 32) {
        int32_t y = __ldg(radj + j);
        if (y >= x) break;
        const int h = c4_slot(c4sm, y);
        if (h >= 0) c += (unsigned long long)atomicAdd(&c4sm[h].y, 1);
      }
    }
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(&acc[8 * g + 6], c);
    __syncthreads();
  }
  // tail tasks: shared-memory (key, count) table per warp
  int2 *tab = c4sm + wid * kC4WarpCap;
  c4_reset(tab, kC4WarpCap, lane, 32);
  __syncwarp();
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    const int32_t x = warp_tasks[t];
    unsigned long long c = 0;
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
        c += (unsigned long long)atomicAdd(&tab[h].y, 1);
      }
    }
    __syncwarp();
    c4_reset(tab, kC4WarpCap, lane, 32);
    __syncwarp();
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(&acc[8 * graph_of(gid, x) + 6], c);
  }
}

// ------------------------------------------------------------ giant 4-cycle tasks
// A task whose 2-hop bound passes big_min has far more distinct y than any
// shared-memory table holds (nearly every wedge ends at its own y).  Its key
// range [base, x) is cut into chunks that fit dense counters in shared memory
// -- 16-bit halves of 32-bit words while x has fewer than 65536 neighbours
// below it, so no count can carry into the next key.  Each a in N(x), a < x,
// keeps a cursor into its sorted list, so a chunk walks only its own segment
// [cur, first y >= hi) and records where it stopped.  Every increment adds
// the counter's old value to the sum (C(c+1,2) - C(c,2) = c), so a chunk needs
// no scan.  A dense chunk is then cleared by a vector memset, a sparse one by
// re-walking the recorded segments.
// Neighbours are handed out highest rank (longest list) first through a
// shared counter, one atomic per warp, to lane groups of P = 1..32 lanes (P
// grows as x has fewer neighbours below it); each lane reads four keys per
// 16-byte load.  Lists longer than twice the task's mean go first, to whole
// warps.  Tasks with a bound of at most kC4HashMax skip the chunks and count
// in one pass in a hash table over the same memory (below).
// CTA shape: one 1024-thread CTA with 200 KB of counters per SM measured
// ahead of two 512-thread CTAs with 100 or 110 KB each.
#ifndef GPM_C4_BIG_THREADS
#define GPM_C4_BIG_THREADS 1024
#endif
#ifndef GPM_C4_BIG_KB
#define GPM_C4_BIG_KB 200
#endif
constexpr int kC4BigThreads = GPM_C4_BIG_THREADS;
constexpr int kC4BigSmem = GPM_C4_BIG_KB * 1024;
constexpr int kC4BigWords = kC4BigSmem / 4;

struct C4Chunk {
  const int32_t *radj;
  int64_t nnz;  // radj length: 16-byte loads only inside it
  int sh;
  int32_t lo, hi;
};

// Hash mode: a task whose bound is at most kC4HashMax counts in one pass in an
// open-addressing table over the same shared memory, slots of (key + 1,
// count) with 0 = empty, so a cleared array is an empty table and the dense
// chunks find it zeroed.  The bound caps the distinct keys below the slot
// count, so every probe sequence ends.
constexpr unsigned kC4HashSlots = kC4BigWords / 2;
constexpr unsigned long long kC4HashMax = kC4HashSlots * 6 / 10;
__device__ __forceinline__ unsigned c4_hash_add(unsigned *cw, unsigned key1) {
  unsigned h = (unsigned)(((unsigned long long)(key1 * 2654435761u) * kC4HashSlots) >> 32);
  for (unsigned p = 0; p < kC4HashSlots; ++p) {
    unsigned cur = cw[2 * h];
    if (cur == 0u) {
      cur = atomicCAS(&cw[2 * h], 0u, key1);
      if (cur == 0u) cur = key1;
    }
    if (cur == key1) return atomicAdd(&cw[2 * h + 1], 1u);
    if (++h == kC4HashSlots) h = 0;
  }
  return 0u;
}

// One step of a group of P lanes over a segment at j (< e): lane gl takes the
// four keys at (j rounded down to 4) + 4 gl.  Keys at or after j that are
// below hi and before e form a prefix of the step (the list is sorted); they
// are counted into cw.  Returns the stop position (first key >= hi, or e)
// when the segment ends inside the step, else -1.
template <bool HASH>
__device__ __forceinline__ int64_t c4_step(const C4Chunk &q, unsigned *cw, int64_t j, int64_t e, unsigned gl,
                                           unsigned gfirst, unsigned gmask, unsigned gbits,
                                           unsigned long long &c, unsigned &nw) {
  const int64_t jb = j & ~(int64_t)3;
  const int64_t p0 = jb + 4 * (int64_t)gl;
  int32_t v[4];
  if (p0 + 4 <= q.nnz) {
    const int4 t = __ldg(reinterpret_cast<const int4 *>(q.radj + p0));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = p0 + k < q.nnz ? __ldg(q.radj + p0 + k) : INT32_MAX;
  }
  const unsigned hmask = q.sh ? 0xffffu : 0xffffffffu;
  const int64_t dj = j - p0, de = e - p0;
  const int skip = dj <= 0 ? 0 : dj >= 4 ? 4 : (int)dj;  // keys of this lane before j
  const int lim = de <= 0 ? 0 : de >= 4 ? 4 : (int)de;   // keys of this lane before e
  int n_ok = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const bool ok = k >= skip && k < lim && v[k] < q.hi;
    if (ok) {
      const unsigned key = (unsigned)(v[k] - q.lo);
      if (HASH) {
        c += c4_hash_add(cw, key + 1);
      } else {
        const unsigned w = key >> q.sh, s = (key & (unsigned)q.sh) << 4;
        const unsigned old = atomicAdd(&cw[w], 1u << s);
        c += (old >> s) & hmask;
      }
      ++n_ok;
    }
  }
  nw += n_ok;
  const bool out = skip + n_ok < 4;  // this lane saw the end of the segment
  const unsigned has = (__ballot_sync(gmask, out) >> gfirst) & gbits;
  if (!has) return -1;
  const int rel = __shfl_sync(gmask, 4 * (int)gl + skip + n_ok, (int)gfirst + __ffs(has) - 1);
  return jb + rel;
}

__global__ void __launch_bounds__(kC4BigThreads, 1024 / kC4BigThreads)
    k_c4_big(const int64_t *__restrict__ roff, const int64_t *__restrict__ split, const int32_t *__restrict__ radj,
             int64_t nnz, const int32_t *__restrict__ gid, const int64_t *__restrict__ gbase,
             const int32_t *__restrict__ tasks, const unsigned long long *__restrict__ task_b, int n_tasks,
             int *__restrict__ counters, int64_t *__restrict__ scratch, int64_t scratch_len,
             unsigned long long *__restrict__ acc) {
  extern __shared__ __align__(16) unsigned cw[];
  __shared__ int s_task, s_nlong, s_next, s_lnext;
  __shared__ unsigned s_nw[2];
  __shared__ unsigned long long s_sum;
  // per-CTA scratch: cursor pairs (two arrays, swapped per chunk), list ends
  // (bitwise-not for long lists), long-list indices
  int64_t *cur = scratch + (int64_t)blockIdx.x * 4 * scratch_len;
  int64_t *nxt = cur + scratch_len;
  int64_t *end = nxt + scratch_len;
  int32_t *lng = reinterpret_cast<int32_t *>(end + scratch_len);
  const unsigned lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kC4BigWords; i += blockDim.x) cw[i] = 0u;
  C4Chunk q;
  q.radj = radj;
  q.nnz = nnz;
  while (true) {
    if (threadIdx.x == 0) {
      s_task = atomicAdd(&counters[2], 1);
      s_nlong = 0;
      s_sum = 0;
      s_next = 0;
      s_lnext = 0;
      s_nw[0] = s_nw[1] = 0;
    }
    __syncthreads();
    const int t = s_task;
    if (t >= n_tasks) break;
    const int32_t x = tasks[t];
    const int g = graph_of(gid, x);
    const int64_t base = gbase ? gbase[g] : 0;
    const int64_t a0 = roff[x];
    const int dx = (int)(split[x] - a0);
    q.sh = dx < 65536 ? 1 : 0;
    int P = 1;
    while (P < 32 && (int64_t)P * 2 * dx <= (int64_t)blockDim.x * 2) P *= 2;
    const long long mean = (long long)(task_b[t] / (unsigned long long)dx);
    const long long long_min = max(64ll * P, 2 * mean);
    for (int i = threadIdx.x; i < dx; i += blockDim.x) {
      const int32_t a = radj[a0 + i];
      const int64_t s = roff[a], e = roff[a + 1];
      cur[i] = s;
      const bool lg = P < 32 && e - s > long_min;
      end[i] = lg ? ~e : e;
      if (lg) lng[atomicAdd(&s_nlong, 1)] = i;
    }
    __syncthreads();
    const int nlong = s_nlong;
    const bool hash = task_b[t] <= kC4HashMax;  // one pass over [base, x) in the hash table
    const int64_t keys = hash ? (int64_t)x - base : (int64_t)kC4BigWords << q.sh;
    const unsigned gl = lane & (P - 1);
    const unsigned gfirst = lane & ~(unsigned)(P - 1);
    const unsigned gmask = P == 32 ? 0xffffffffu : (((1u << P) - 1) << gfirst);
    const unsigned gbits = P == 32 ? 0xffffffffu : ((1u << P) - 1);
    unsigned long long c = 0;
    int parity = 0;
    for (int64_t lo = base; lo < x; lo += keys, parity ^= 1) {
      q.lo = (int32_t)lo;
      q.hi = (int32_t)(lo + keys < (int64_t)x ? lo + keys : (int64_t)x);
      unsigned nw = 0;
      // long lists first, one warp each, handed out through s_lnext
      while (true) {
        int li = 0;
        if (lane == 0) li = atomicAdd(&s_lnext, 1);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= nlong) break;
        const int i = lng[li];
        const int64_t e = ~end[i];
        int64_t j = cur[i];
        while (j < e) {
          const int64_t stop = hash ? c4_step<true>(q, cw, j, e, lane, 0, 0xffffffffu, 0xffffffffu, c, nw)
                                    : c4_step<false>(q, cw, j, e, lane, 0, 0xffffffffu, 0xffffffffu, c, nw);
          if (stop >= 0) {
            j = stop;
            break;
          }
          j = (j & ~(int64_t)3) + 128;
        }
        if (lane == 0) nxt[i] = j < e ? j : e;
      }
      // short lists: flattened walk, one step or one refill per iteration
      {
        int i = -1;
        int64_t j = 0, e = 0;
        while (true) {
          if (j >= e) {
            if (i >= 0 && gl == 0) nxt[i] = j;
            int ni = 0;
            if (gl == 0) {  // one shared atomic for all group leaders of the warp that need an a
              const cg::coalesced_group ct = cg::coalesced_threads();
              int base = 0;
              if (ct.thread_rank() == 0) base = atomicAdd(&s_next, (int)ct.size());
              ni = ct.shfl(base, 0) + (int)ct.thread_rank();
            }
            ni = __shfl_sync(gmask, ni, gfirst);
            if (ni >= dx) break;
            i = dx - 1 - ni;  // highest rank (longest lists) first
            e = end[i];
            j = cur[i];
            if (e < 0) {  // long list: walked above
              i = -1;
              j = e = 0;
            }
            continue;
          }
          const int64_t stop = hash ? c4_step<true>(q, cw, j, e, gl, gfirst, gmask, gbits, c, nw)
                                    : c4_step<false>(q, cw, j, e, gl, gfirst, gmask, gbits, c, nw);
          if (stop >= 0) j = e = stop;
          else j = (j & ~(int64_t)3) + 4 * P;
        }
      }
      nw = warp_sum(nw);
      if (lane == 0 && nw) atomicAdd(&s_nw[parity], nw);
      __syncthreads();
      // clear: memset when dense, else re-walk [cur, nxt)
      const bool dense = hash || (unsigned long long)s_nw[parity] * 4 > (unsigned long long)kC4BigWords;
      if (threadIdx.x == 0) {
        s_next = 0;
        s_lnext = 0;
        s_nw[parity ^ 1] = 0;
      }
      if (dense) {
        uint4 *v = reinterpret_cast<uint4 *>(cw);
        for (int k = threadIdx.x; k < kC4BigWords / 4; k += blockDim.x) v[k] = make_uint4(0u, 0u, 0u, 0u);
      } else {
        for (int i = threadIdx.x; i < dx; i += blockDim.x) {
          const int64_t j1 = nxt[i];
          for (int64_t j = cur[i]; j < j1; ++j) cw[(unsigned)(__ldg(radj + j) - q.lo) >> q.sh] = 0u;
        }
      }
      __syncthreads();
      int64_t *tmp = cur;
      cur = nxt;
      nxt = tmp;
    }
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(&s_sum, c);
    __syncthreads();
    if (threadIdx.x == 0 && s_sum) atomicAdd(&acc[8 * g + 6], s_sum);
    // cur and nxt swap once per chunk: restore the base layout for the next task
    if (cur != scratch + (int64_t)blockIdx.x * 4 * scratch_len) {
      int64_t *tmp = cur;
      cur = nxt;
      nxt = tmp;
    }
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
  static PerDevice grid;
  return grid.get([] {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edge_tri, 256, kTeSmem);
    return std::max(1, per_sm) * num_sms();
  });
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
  if (in.size == 4) GPM_TRY(dag_from_split(n, roff, p->split.p, radj, p->doff, p->dadj, &p->dag_max, st));
  GPM_TRY(p->te.reserve(std::max<int64_t>(in.nnz, 1)));
  // queues of the per-edge triangle pass and of the 4-cycle pass
  DevBuf<int> sizes;
  GPM_TRY(sizes.reserve(6));
  GPM_TRY(p->te_ct.reserve(n));
  GPM_TRY(p->te_wt.reserve(n));
  GPM_TRY(p->c4_ct.reserve(n));
  GPM_TRY(p->c4_wt.reserve(n));
  DevBuf<int32_t> bt;
  DevBuf<unsigned long long> bb;
  GPM_TRY(bt.reserve(n));
  GPM_TRY(bb.reserve(n));
  GPM_TRY(p->te_counters.reserve(2));
  GPM_TRY(p->c4_counters.reserve(4));
  GPM_CUDA(cudaMemsetAsync(sizes.p, 0, 6 * sizeof(int), st));
  if (n > 0) {
    k_te_tasks<<<grid_for(n), 256, 0, st>>>(n, roff, p->split.p, std::min(in.te_cta_min, kTeWarpCap / 2), p->te_ct.p, p->te_wt.p, sizes.p);
    if (in.size == 4) {
      const int wb = std::min(in.c4_warp_bound, kC4WarpCap / 2);
      long long big_min = in.c4_big_min;
      if (const char *e = getenv("GPM_C4_BIG_MIN")) big_min = atoll(e);
      big_min = std::min(std::max<long long>(big_min, (long long)wb), kC4HubMax);
      // hub tasks (bound <= big_min) must fit c4_slot's table, or they would drop wedges
      if (big_min > kC4HubMax) return fail(GPM_EINVAL, "4-cycle hub bound above the hub table");
      k_c4_tasks<<<grid_for(n * 32), 256, 0, st>>>(n, roff, p->split.p, radj, wb, big_min,
                                                   p->c4_ct.p, p->c4_wt.p, bt.p, bb.p, sizes.p + 2);
    }
  }
  int h[6];
  GPM_CUDA(cudaMemcpyAsync(h, sizes.p, sizeof h, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  p->te_nc = h[0];
  p->te_nw = h[1];
  p->c4_nc = h[2];
  p->c4_nw = h[3];
  p->c4_nb = h[4];
  p->te_grid = te_grid();
  if (in.size == 3) {
    GPM_CUDA(cudaStreamSynchronize(st));
    return GPM_OK;
  }
  // giant tasks, largest bound first
  GPM_TRY(p->c4_bt.reserve(std::max(p->c4_nb, 1)));
  GPM_TRY(p->c4_bb.reserve(std::max(p->c4_nb, 1)));
  if (p->c4_nb > 0) {
    size_t tmp = 0;
    GPM_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, bb.p, p->c4_bb.p, bt.p, p->c4_bt.p, p->c4_nb, 0,
                                                       64, st));
    DevBuf<char> t;
    GPM_TRY(t.reserve(tmp));
    GPM_CUDA(cub::DeviceRadixSort::SortPairsDescending(t.p, tmp, bb.p, p->c4_bb.p, bt.p, p->c4_bt.p, p->c4_nb, 0,
                                                       64, st));
    GPM_CUDA(cudaFuncSetAttribute(k_c4_big, cudaFuncAttributeMaxDynamicSharedMemorySize, kC4BigSmem));
    int per_sm = 0;
    GPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_big, kC4BigThreads, kC4BigSmem));
    p->c4_big_grid = std::max(1, per_sm) * num_sms();
    p->c4_scratch = std::max(h[5], 1);
    // per CTA: cursors, next cursors, list ends (int64 each), long-list indices (int32, padded)
    GPM_TRY(p->c4_cur.reserve((size_t)p->c4_scratch * 4 * p->c4_big_grid));
    if ((reinterpret_cast<uintptr_t>(in.radj) & 15) != 0)
      return fail(GPM_EINVAL, "motif: adjacency not 16-byte aligned");
    GPM_CUDA(cudaStreamSynchronize(st));
  }
  {
    int per_sm = 0;
    GPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4, 256, 0));
    p->c4_grid = std::max(1, per_sm) * num_sms();
  }
  GPM_TRY(clique_plan_build(&p->k4, n, p->doff.p, p->dadj.p, p->dag_max, 4, in.gid, p->acc.p, 8, 5, st,
                            in.cq_warp_max));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

// The 4-cycle launches: giant tasks first (largest bound first), then hub and tail tasks.
static int c4_launch(MotifPlan *p, cudaStream_t st) {
  const MotifInput &in = p->in;
  if (p->c4_nb > 0)
    k_c4_big<<<p->c4_big_grid, kC4BigThreads, kC4BigSmem, st>>>(
        in.roff, p->split.p, in.radj, in.nnz, in.gid, in.gbase, p->c4_bt.p, p->c4_bb.p, p->c4_nb, p->c4_counters.p,
        p->c4_cur.p, p->c4_scratch, p->acc.p);
  if (p->c4_nc + p->c4_nw > 0)
    k_c4<<<p->c4_grid, 256, 0, st>>>(in.roff, p->split.p, in.radj, in.gid, in.gbase, p->c4_ct.p, p->c4_nc,
                                     p->c4_wt.p, p->c4_nw, p->c4_counters.p, p->acc.p);
  GPM_LAUNCH_CHECK();
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
  GPM_CUDA(cudaMemsetAsync(p->c4_counters.p, 0, 4 * sizeof(int), st));
  if (p->te_nc + p->te_nw > 0)
    k_edge_tri<<<p->te_grid, 256, kTeSmem, st>>>(in.roff, p->split.p, in.radj, p->te_ct.p, p->te_nc, p->te_wt.p,
                                                 p->te_nw, p->te_counters.p, p->te.p);
  if (n > 0)
    k_edge_sums<<<grid_for(n * 32), 256, 0, st>>>(n, in.roff, p->split.p, in.radj, p->te.p, in.gid, p->acc.p);
  if (in.size == 4) {
    GPM_TRY(c4_launch(p, st));
    GPM_TRY(clique_plan_run(&p->k4, st));
  }
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
    GPM_CUDA(cudaMemsetAsync(p->c4_counters.p, 0, 4 * sizeof(int), st));
    GPM_TRY(c4_launch(p, st));
  } else {
    GPM_TRY(clique_plan_run(&p->k4, st));
  }
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

}  // namespace gpm

namespace gpm {
void free_motif_plan(MotifPlan *p) { delete p; }
}  // namespace gpm

using namespace gpm;

extern "C" int gpm_motif(gpm_graph *g, int k, uint64_t *out) {
  if (!g || !out) return fail(GPM_EINVAL, "gpm_motif: NULL argument");
  if (k != 3 && k != 4) return fail(GPM_EUNSUPPORTED, "motif size must be 3 or 4");
  if (g->oriented) return fail(GPM_EINVAL, "motif counting needs the symmetric (unoriented) graph");
  GPM_TRY(ensure_rank_graph(g, 0));
  // the pipeline (task queues, scratch) is built on the first call of each
  // size and kept with the graph, so later calls only launch
  MotifPlan *&plan = g->motif[k - 3];
  if (!plan) {
    MotifInput in;
    in.n = g->n;
    in.nnz = g->nnz;
    in.roff = g->rg->roff.p;
    in.radj = g->rg->radj.p;
    in.max_graph_n = g->n;
    in.size = k;
    MotifPlan *p = new MotifPlan();
    const int s = motif_plan_build(in, p, 0);
    if (s != GPM_OK) {
      delete p;
      return s;
    }
    plan = p;
  }
  GPM_TRY(motif_plan_run(plan, 0));
  unsigned long long h[8];
  GPM_CUDA(cudaMemcpy(h, plan->out.p, sizeof h, cudaMemcpyDeviceToHost));
  if (k == 3) {
    out[0] = h[0];
    out[1] = h[1];
  } else {
    for (int i = 0; i < 6; ++i) out[i] = h[2 + i];
  }
  return GPM_OK;
}
