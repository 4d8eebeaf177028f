// clique.cu -- k-clique counting (CFSolver, src/CFSolver.cuh:15-158).
//
// The reference counts, for every stored edge (v0,v1), the cliques grown by
// nested materialised intersections W1 = N(v0) & N(v1), W2 = W1 & N(v2), ...
// (clique_4_edge_warp / clique_5_edge_warp).  On a degree-oriented DAG that
// is the number of k-cliques.
//
// B200 path (upward rank graph, see tc_rank.cuh): a vertex task u turns its
// out-list L = N+(u) into a local DAG whose adjacency rows are bitsets
// (row_i = {j : L[j] in N+(L[i])}).  Because the rank graph points upward,
// row_i only has bits j > i, so the (k-1)-cliques of the local DAG are found
// by consuming bits in increasing order and AND-ing rows -- popcounts instead
// of list intersections.
//   * tasks with |L| <= 64: one warp, rows are uint64 held in shared memory,
//     one lane per starting row;
//   * tasks with 64 < |L| <= 2048: one CTA, rows of W = ceil(|L|/32) words
//     in shared memory (or a per-CTA global slab when they do not fit), each
//     warp walks rows with the bitset spread over its lanes.
// Graphs whose stored edges do not all point upward in rank order, or with
// an out-list longer than 2048, use an edge-centric kernel shaped like the
// reference (materialised lists in per-warp global scratch).
#include <cub/cub.cuh>

#include <algorithm>

#include "common.cuh"
#include "motif.cuh"
#include "tc_rank.cuh"

namespace gpm {

constexpr int kCqWarpMax = 64;      // warp tasks: |L| <= 64
constexpr int kCqCtaMax = 2048;     // CTA tasks: |L| <= 2048 (W <= 64)
constexpr int kCqMaxK = 8;
#ifndef GPM_CQ_SMEM_KB
// 32 KB: 5 CTAs per SM (registers allow 5; 48 KB allowed 4).  R-MAT 20 with
// the lane-parallel last levels: 4-cliques 24.1 ms, 5-cliques 188 ms against
// 27.0 / 194 ms at 48 KB and 24.3 / 195 ms at 40 KB (motif batch replay 809
// against 835 ms).  Earlier, 48 KB beat 96 KB (2 CTAs per SM) by 1.6x.
// Tasks whose rows do not fit use their CTA's global slab.
#define GPM_CQ_SMEM_KB 32
#endif
constexpr size_t kCqSmem = GPM_CQ_SMEM_KB * 1024;  // dynamic shared memory per CTA

static int grid_for(int64_t work, int block = 256) {
  int64_t g = (work + block - 1) / block;
  int64_t cap = (int64_t)num_sms() * 16;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}

// position of key in sorted L[0..d), or -1
__device__ __forceinline__ int find_pos(const int32_t *L, int d, int32_t key) {
  int lo = 0, hi = d - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int32_t x = L[mid];
    if (x == key) return mid;
    if (x < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// first index in sorted a[0..n) with a[i] > key
__device__ __forceinline__ int64_t upper_bound_g(const int32_t *__restrict__ a, int64_t n, int32_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------ warp tasks (|L| <= 64)
// number of q-cliques inside bitset X of the local DAG (q >= 1)
__device__ unsigned long long local_count64(const unsigned long long *rows, unsigned long long X, int q) {
  if (q == 1) return __popcll(X);
  if (q == 2) {
    unsigned long long c = 0;
    while (X) {
      int l = __ffsll(X) - 1;
      X &= X - 1;
      c += __popcll(X & rows[l]);
    }
    return c;
  }
  unsigned long long stk[kCqMaxK];
  int depth = 0;
  stk[0] = X;
  unsigned long long c = 0;
  // stk[depth] holds the candidates still to extend at level depth; a set
  // at level depth needs q - depth more vertices.
  while (depth >= 0) {
    unsigned long long &S = stk[depth];
    if (!S) { --depth; continue; }
    int l = __ffsll(S) - 1;
    S &= S - 1;
    unsigned long long Y = S & rows[l];
    int left = q - depth - 1;  // vertices still needed after picking l
    if (left == 1) c += __popcll(Y);
    else if (left == 2) {
      while (Y) {
        int m = __ffsll(Y) - 1;
        Y &= Y - 1;
        c += __popcll(Y & rows[m]);
      }
    } else if (Y) stk[++depth] = Y;
  }
  return c;
}

__device__ unsigned long long clique_warp_task(int32_t u, int k, const int64_t *__restrict__ roff,
                                               const int32_t *__restrict__ radj, int32_t *L,
                                               unsigned long long *rows) {
  const unsigned lane = lane_id();
  const int64_t s0 = roff[u];
  const int d = (int)(roff[u + 1] - s0);
  for (int i = lane; i < d; i += 32) {
    L[i] = radj[s0 + i];
    rows[i] = 0ull;
  }
  __syncwarp();
  const int32_t kmax = L[d - 1];
  // row i: members of L inside N+(L[i]) (all > L[i]); only N+(L[i]) up to
  // kmax can hit.  Lane j finds the scan ranges of rows j and j + 32 (one
  // binary search each, in parallel), then the ranges are laid end to end
  // and every lane takes one entry of the concatenation per round, so short
  // lists do not leave lanes idle.
  long long sa = 0, la = 0, sb = 0, lb = 0;
  if ((int)lane < d) {
    const int32_t v = L[lane];
    sa = roff[v];
    la = upper_bound_g(radj + sa, roff[v + 1] - sa, kmax);
  }
  if ((int)lane + 32 < d) {
    const int32_t v = L[lane + 32];
    sb = roff[v];
    lb = upper_bound_g(radj + sb, roff[v + 1] - sb, kmax);
  }
  long long ia = la, ib = lb;  // inclusive prefixes over rows 0..31 and 32..63
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long va = __shfl_up_sync(0xffffffffu, ia, o), vb = __shfl_up_sync(0xffffffffu, ib, o);
    if ((int)lane >= o) {
      ia += va;
      ib += vb;
    }
  }
  const long long ta = __shfl_sync(0xffffffffu, ia, 31), total = ta + __shfl_sync(0xffffffffu, ib, 31);
  for (long long base = 0; base < total; base += 32) {
    const long long idx = base + lane;
    const bool hi = idx >= ta;
    const long long key = hi ? idx - ta : idx;
    int lo = 0, up = 31;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int mid = (lo + up) >> 1;
      const long long pa = __shfl_sync(0xffffffffu, ia, mid), pb = __shfl_sync(0xffffffffu, ib, mid);
      if ((hi ? pb : pa) > key) up = mid; else lo = mid + 1;
    }
    const long long pa = __shfl_sync(0xffffffffu, ia, lo), pb = __shfl_sync(0xffffffffu, ib, lo);
    const long long ra = __shfl_sync(0xffffffffu, la, lo), rb = __shfl_sync(0xffffffffu, lb, lo);
    const long long xa = __shfl_sync(0xffffffffu, sa, lo), xb = __shfl_sync(0xffffffffu, sb, lo);
    if (idx < total) {
      const int row = lo + (hi ? 32 : 0);
      const long long t = (hi ? xb : xa) + key - ((hi ? pb : pa) - (hi ? rb : ra));
      const int p = find_pos(L, d, __ldg(radj + t));
      if (p >= 0) atomicOr(&rows[row], 1ull << p);
    }
  }
  __syncwarp();
  unsigned long long c = 0;
  for (int i = lane; i < d; i += 32) c += local_count64(rows, rows[i], k - 2);
  __syncwarp();
  return c;
}

// ------------------------------------------------------------ CTA tasks (64 < |L| <= 2048)
// Bitsets of W <= 64 words spread over a warp: lane w holds words w, w + 32.
struct WarpSet {
  uint32_t a, b;
};
__device__ __forceinline__ int wpop(WarpSet s) { return __popc(s.a) + __popc(s.b); }

// Lowest set bit of a warp-spread set, cleared in place; -1 if empty.
__device__ __forceinline__ int wtake(WarpSet &s, unsigned lane) {
  unsigned m = __ballot_sync(0xffffffffu, s.a != 0);
  int base = 0;
  uint32_t word;
  int f;
  if (m) {
    f = __ffs(m) - 1;
    word = __shfl_sync(0xffffffffu, s.a, f);
  } else {
    m = __ballot_sync(0xffffffffu, s.b != 0);
    if (!m) return -1;
    f = __ffs(m) - 1;
    word = __shfl_sync(0xffffffffu, s.b, f);
    base = 1024;
  }
  int bit = __ffs(word) - 1;
  if ((int)lane == f) {
    if (base) s.b &= s.b - 1; else s.a &= s.a - 1;
  }
  return base + f * 32 + bit;
}

__device__ __forceinline__ WarpSet wrow(const uint32_t *rows, int W, int j, unsigned lane) {
  const uint32_t *r = rows + (size_t)j * W;
  WarpSet s;
  s.a = (int)lane < W ? r[lane] : 0u;
  s.b = (int)lane + 32 < W ? r[lane + 32] : 0u;
  return s;
}

// index of the k-th (0-based) set bit of w (k < popc(w))
__device__ __forceinline__ int kth_bit(uint32_t w, int k) {
  int pos = 0;
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    const int c = __popc(w & ((1u << s) - 1u));
    if (k >= c) {
      k -= c;
      w >>= s;
      pos += s;
    }
  }
  return pos;
}

// Sum over l in X of |X & row_l| -- the 2-cliques inside warp-spread X --
// with the members l of X spread over the lanes: lane t takes the t-th
// member of each round of 32 and ANDs X (staged in the warp's shared words
// xs) with its row word by word from l's own word on (row_l has no bits
// below l).  Each lane returns its partial sum.
__device__ unsigned long long wsum_pairs(const uint32_t *rows, int W, WarpSet X, uint32_t *xs, unsigned lane) {
  __syncwarp();
  xs[lane] = X.a;
  xs[lane + 32] = X.b;
  __syncwarp();
  // members are numbered word by word: words 0..31 (X.a of lanes 0..31), then 32..63
  int inc = __popc(X.a), incb = __popc(X.b);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int va = __shfl_up_sync(0xffffffffu, inc, o), vb = __shfl_up_sync(0xffffffffu, incb, o);
    if ((int)lane >= o) {
      inc += va;
      incb += vb;
    }
  }
  const int ta = __shfl_sync(0xffffffffu, inc, 31), total = ta + __shfl_sync(0xffffffffu, incb, 31);
  unsigned long long c = 0;
  for (int base = 0; base < total; base += 32) {
    const int idx = base + (int)lane;
    // word holding member idx: first word whose inclusive prefix exceeds it
    const bool hi = idx >= ta;
    const int key = hi ? idx - ta : idx;
    int lo = 0, up = 31;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const int mid = (lo + up) >> 1;
      const int pa = __shfl_sync(0xffffffffu, inc, mid), pb = __shfl_sync(0xffffffffu, incb, mid);
      if ((hi ? pb : pa) > key) up = mid; else lo = mid + 1;
    }
    const int pa_lo = __shfl_sync(0xffffffffu, inc, lo), pb_lo = __shfl_sync(0xffffffffu, incb, lo);
    if (idx < total) {
      const int w = lo + (hi ? 32 : 0);
      const uint32_t word = xs[w];
      const int excl = (hi ? pb_lo : pa_lo) - __popc(word);
      const int l = w * 32 + kth_bit(word, key - excl);
      const uint32_t *rl = rows + (size_t)l * W;
      unsigned s = 0;
      for (int ww = l >> 5; ww < W; ++ww) s += __popc(xs[ww] & rl[ww]);
      c += s;
    }
  }
  return c;
}

// q-cliques inside warp-spread X; stk holds (q) levels of W words per warp
__device__ unsigned long long warp_count_set(const uint32_t *rows, int W, WarpSet X, int q, uint32_t *xs,
                                             unsigned lane) {
  if (q == 1) return (unsigned long long)wpop(X);
  if (q == 2) return wsum_pairs(rows, W, X, xs, lane);
  WarpSet stk[kCqMaxK];
  int depth = 0;
  stk[0] = X;
  unsigned long long c = 0;
  while (depth >= 0) {
    int l = wtake(stk[depth], lane);
    if (l < 0) { --depth; continue; }
    WarpSet r = wrow(rows, W, l, lane);
    WarpSet Y{stk[depth].a & r.a, stk[depth].b & r.b};
    int left = q - depth - 1;
    if (left == 1) c += (unsigned long long)wpop(Y);
    else if (left == 2) c += wsum_pairs(rows, W, Y, xs, lane);
    else stk[++depth] = Y;
  }
  return c;
}

__device__ unsigned long long clique_cta_task(int32_t u, int k, const int64_t *__restrict__ roff,
                                              const int32_t *__restrict__ radj, char *smem, uint32_t *slab,
                                              uint32_t *xs) {
  const int tid = threadIdx.x, nthr = blockDim.x, wid = tid >> 5, nw = nthr >> 5;
  const unsigned lane = tid & 31;
  const int64_t s0 = roff[u];
  const int d = (int)(roff[u + 1] - s0);
  const int W = (d + 31) >> 5;
  int32_t *L = reinterpret_cast<int32_t *>(smem);
  size_t lbytes = ((size_t)d * 4 + 15) & ~(size_t)15;
  size_t rbytes = (size_t)d * W * 4;
  uint32_t *rows = lbytes + rbytes <= kCqSmem ? reinterpret_cast<uint32_t *>(smem + lbytes) : slab;
  for (int i = tid; i < d; i += nthr) L[i] = radj[s0 + i];
  for (size_t i = tid; i < (size_t)d * W; i += nthr) rows[i] = 0u;
  __syncthreads();
  const int32_t kmax = L[d - 1];
  // warp wid builds rows wid, wid + nw, ...; the scan ranges of 32 of them at
  // a time are found in parallel, one lane per row
  for (int i0 = wid; i0 < d; i0 += nw * 32) {
    const int mine = i0 + (int)lane * nw;
    long long ms = 0, mstop = 0;
    if (mine < d) {
      const int32_t v = L[mine];
      ms = roff[v];
      mstop = ms + upper_bound_g(radj + ms, roff[v + 1] - ms, kmax);
    }
    for (int j = 0; j < 32 && i0 + j * nw < d; ++j) {
      const int i = i0 + j * nw;
      const long long s = __shfl_sync(0xffffffffu, ms, j), stop = __shfl_sync(0xffffffffu, mstop, j);
      uint32_t *ri = rows + (size_t)i * W;
      for (long long t = s + lane; t < stop; t += 32) {
        int p = find_pos(L, d, __ldg(radj + t));
        if (p >= 0) atomicOr(&ri[p >> 5], 1u << (p & 31));
      }
    }
  }
  __syncthreads();
  unsigned long long c = 0;
  // each lane accumulates the popcounts of its own words; the warp sum is the count
  for (int i = wid; i < d; i += nw) c += warp_count_set(rows, W, wrow(rows, W, i, lane), k - 2, xs, lane);
  __syncthreads();
  return c;
}

__global__ void __launch_bounds__(256) k_clique_local(int k, const int64_t *__restrict__ roff,
                                                      const int32_t *__restrict__ radj,
                                                      const int32_t *__restrict__ cta_tasks, int n_cta,
                                                      const int32_t *__restrict__ warp_tasks, int n_warp,
                                                      int *__restrict__ counters, uint32_t *__restrict__ slabs,
                                                      size_t slab_words, const int32_t *__restrict__ gid,
                                                      unsigned long long *__restrict__ acc, int stride, int slot) {
  extern __shared__ __align__(16) char csm[];
  __shared__ int s_task;
  __shared__ uint32_t sxs[8][64];  // each warp's staged set (wsum_pairs)
  const int wid = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31;
  uint32_t *slab = slabs + (size_t)blockIdx.x * slab_words;
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    const int32_t u = cta_tasks[t];
    unsigned long long c = warp_sum(clique_cta_task(u, k, roff, radj, csm, slab, sxs[wid]));
    if (lane == 0 && c) atomicAdd(&acc[(size_t)stride * (gid ? gid[u] : 0) + slot], c);
  }
  int32_t *L = reinterpret_cast<int32_t *>(csm + wid * (kCqWarpMax * 12));
  unsigned long long *rows = reinterpret_cast<unsigned long long *>(csm + wid * (kCqWarpMax * 12) + kCqWarpMax * 4);
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    const int32_t u = warp_tasks[t];
    unsigned long long c = warp_sum(clique_warp_task(u, k, roff, radj, L, rows));
    if (lane == 0 && c) atomicAdd(&acc[(size_t)stride * (gid ? gid[u] : 0) + slot], c);
  }
}

__global__ void k_clique_tasks(int64_t n, const int64_t *__restrict__ roff, int k, int warp_max,
                               uint32_t *__restrict__ ckey,
                               int32_t *__restrict__ cval, uint32_t *__restrict__ wkey, int32_t *__restrict__ wval,
                               int *__restrict__ sizes) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    int64_t d = roff[u + 1] - roff[u];
    if (d < k - 1) continue;
    if (d > warp_max) {
      int i = atomicAdd(&sizes[0], 1);
      ckey[i] = ~(uint32_t)d;
      cval[i] = (int32_t)u;
    } else {
      int i = atomicAdd(&sizes[1], 1);
      wkey[i] = ~(uint32_t)d;
      wval[i] = (int32_t)u;
    }
  }
}

// ------------------------------------------------------------ edge-centric (reference-shaped)
// Warp-cooperative c = a & b by binary search of the shorter list's keys in
// the longer one, compacted in order with ballots; returns |c|.
__device__ int warp_isect_store(const int32_t *a, int na, const int32_t *b, int nb, int32_t *c, unsigned lane) {
  const int32_t *look = a, *srch = b;
  int nl = na, ns = nb;
  if (na > nb) { look = b; srch = a; nl = nb; ns = na; }
  int cnt = 0;
  for (int base = 0; base < nl; base += 32) {
    int i = base + lane;
    bool f = false;
    int32_t key = 0;
    if (i < nl) {
      key = look[i];
      int lo = 0, hi = ns - 1;
      while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int32_t x = srch[mid];
        if (x == key) { f = true; break; }
        if (x < key) lo = mid + 1; else hi = mid - 1;
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, f);
    if (f) c[cnt + __popc(m & ((1u << lane) - 1u))] = key;
    cnt += __popc(m);
  }
  __syncwarp();
  return cnt;
}

__device__ unsigned long long warp_isect_count(const int32_t *a, int na, const int32_t *b, int nb, unsigned lane) {
  const int32_t *look = a, *srch = b;
  int nl = na, ns = nb;
  if (na > nb) { look = b; srch = a; nl = nb; ns = na; }
  unsigned long long c = 0;
  for (int i = lane; i < nl; i += 32) {
    int32_t key = look[i];
    int lo = 0, hi = ns - 1;
    while (lo <= hi) {
      int mid = (lo + hi) >> 1;
      int32_t x = srch[mid];
      if (x == key) { ++c; break; }
      if (x < key) lo = mid + 1; else hi = mid - 1;
    }
  }
  return c;
}

__global__ void __launch_bounds__(256) k_clique_edge(int64_t nnz, int k, const int64_t *__restrict__ off,
                                                     const int32_t *__restrict__ adj, const int32_t *__restrict__ src,
                                                     int32_t *__restrict__ scratch, int maxd,
                                                     unsigned long long *__restrict__ out) {
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int32_t *lists = scratch + warp * (int64_t)maxd * (kCqMaxK - 2);
  int sizes[kCqMaxK], cursor[kCqMaxK];
  unsigned long long c = 0;
  for (int64_t e = warp; e < nnz; e += nw) {
    int32_t v0 = src[e], v1 = adj[e];
    int n1 = warp_isect_store(adj + off[v0], (int)(off[v0 + 1] - off[v0]), adj + off[v1],
                              (int)(off[v1 + 1] - off[v1]), lists, lane);
    // lists[l] holds the candidates after l+2 clique vertices
    if (k == 3) { c += lane == 0 ? (unsigned long long)n1 : 0ull; continue; }
    sizes[0] = n1;
    cursor[0] = 0;
    int depth = 0;
    while (depth >= 0) {
      if (cursor[depth] >= sizes[depth]) { --depth; continue; }
      int32_t *cur = lists + (int64_t)depth * maxd;
      int32_t x = cur[cursor[depth]++];
      const int32_t *nx = adj + off[x];
      int dx = (int)(off[x + 1] - off[x]);
      if (depth + 3 == k - 1) {
        c += warp_isect_count(cur, sizes[depth], nx, dx, lane);
      } else {
        int32_t *nxt = lists + (int64_t)(depth + 1) * maxd;
        sizes[depth + 1] = warp_isect_store(cur, sizes[depth], nx, dx, nxt, lane);
        cursor[depth + 1] = 0;
        ++depth;
      }
    }
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

// ------------------------------------------------------------ host
static int clique_local_grid() {
  static PerDevice grid;
  return grid.get([] {
    cudaFuncSetAttribute(k_clique_local, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCqSmem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clique_local, 256, kCqSmem);
    return std::max(1, per_sm) * num_sms();
  });
}

// Plan: task queues (heaviest first) and row slabs; the run is launches only.
int clique_plan_build(CliquePlan *p, int64_t n, const int64_t *roff, const int32_t *radj, int max_deg, int k,
                      const int32_t *gid, unsigned long long *acc, int stride, int slot, cudaStream_t st,
                      int warp_max) {
  warp_max = std::max(1, std::min(warp_max, kCqWarpMax));
  p->n = n;
  p->roff = roff;
  p->radj = radj;
  p->k = k;
  p->gid = gid;
  p->acc = acc;
  p->stride = stride;
  p->slot = slot;
  p->n_cta = p->n_warp = 0;
  if (n == 0) return GPM_OK;
  if (max_deg > kCqCtaMax) return fail(GPM_EUNSUPPORTED, "out-list longer than 2048 on the bitset clique path");
  DevBuf<uint32_t> ckey, wkey;
  DevBuf<int32_t> cval, wval;
  DevBuf<int> sizes;
  GPM_TRY(ckey.reserve(n));
  GPM_TRY(wkey.reserve(n));
  GPM_TRY(cval.reserve(n));
  GPM_TRY(wval.reserve(n));
  GPM_TRY(p->ctasks.reserve(n));
  GPM_TRY(p->wtasks.reserve(n));
  GPM_TRY(sizes.reserve(2));
  GPM_TRY(p->counters.reserve(2));
  GPM_CUDA(cudaMemsetAsync(sizes.p, 0, 2 * sizeof(int), st));
  k_clique_tasks<<<grid_for(n), 256, 0, st>>>(n, roff, k, warp_max, ckey.p, cval.p, wkey.p, wval.p, sizes.p);
  int h[2];
  GPM_CUDA(cudaMemcpyAsync(h, sizes.p, sizeof h, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  for (int which = 0; which < 2; ++which) {
    int cnt = h[which];
    if (cnt <= 0) continue;
    DevBuf<uint32_t> k2;
    GPM_TRY(k2.reserve(cnt));
    size_t tmp = 0;
    uint32_t *kin = which ? wkey.p : ckey.p;
    int32_t *vin = which ? wval.p : cval.p, *vout = which ? p->wtasks.p : p->ctasks.p;
    GPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, k2.p, vin, vout, cnt, 0, 32, st));
    DevBuf<char> t;
    GPM_TRY(t.reserve(tmp));
    GPM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, k2.p, vin, vout, cnt, 0, 32, st));
  }
  p->n_cta = h[0];
  p->n_warp = h[1];
  // per-CTA slabs for rows that do not fit in shared memory
  p->grid = clique_local_grid();
  size_t W = (size_t)(max_deg + 31) / 32;
  p->slab_words = (size_t)max_deg * W * 4 + (size_t)max_deg * 4 > kCqSmem ? (size_t)max_deg * W : 1;
  GPM_TRY(p->slabs.reserve(p->slab_words * p->grid));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

int clique_plan_run(CliquePlan *p, cudaStream_t st) {
  if (p->n_cta + p->n_warp == 0) return GPM_OK;
  GPM_CUDA(cudaMemsetAsync(p->counters.p, 0, 2 * sizeof(int), st));
  k_clique_local<<<p->grid, 256, kCqSmem, st>>>(p->k, p->roff, p->radj, p->ctasks.p, p->n_cta, p->wtasks.p,
                                                p->n_warp, p->counters.p, p->slabs.p, p->slab_words, p->gid, p->acc,
                                                p->stride, p->slot);
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

int clique_run_upward(int64_t n, const int64_t *roff, const int32_t *radj, int max_deg, int k, const int32_t *gid,
                      unsigned long long *acc, int stride, int slot, cudaStream_t st) {
  CliquePlan p;
  GPM_TRY(clique_plan_build(&p, n, roff, radj, max_deg, k, gid, acc, stride, slot, st));
  GPM_TRY(clique_plan_run(&p, st));
  GPM_CUDA(cudaStreamSynchronize(st));  // the plan's scratch is released on return
  return GPM_OK;
}

void free_clique_plan(CliquePlan *p) { delete p; }

int clique_launch(gpm_graph *g, int k, cudaStream_t st, unsigned long long *d_out, bool edge_centric = false) {
  GPM_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
  if (g->nnz == 0) return GPM_OK;
  GPM_TRY(ensure_rank_graph(g, st));
  if (!edge_centric && g->rg->upward && g->max_deg <= kCqCtaMax) {
    // the schedule (task queues, per-CTA bitset slabs) is built on the first
    // call for this k and kept with the graph
    CliquePlan *&p = g->clique[k];
    if (!p) {
      CliquePlan *q = new CliquePlan();
      const int s = clique_plan_build(q, g->n, g->rg->roff.p, g->rg->radj.p, g->max_deg, k, nullptr, d_out, 0, 0, st);
      if (s != GPM_OK) {
        delete q;
        return s;
      }
      p = q;
    }
    p->acc = d_out;
    return clique_plan_run(p, st);
  }
  // edge-centric path on the stored graph
  GPM_TRY(ensure_src(g, st));
  int grid = num_sms() * 8;
  int64_t warps = (int64_t)grid * 8;
  int maxd = std::max(1, g->max_deg);
  DevBuf<int32_t> scratch;
  GPM_TRY(scratch.reserve((size_t)warps * maxd * (kCqMaxK - 2)));
  k_clique_edge<<<grid, 256, 0, st>>>(g->nnz, k, g->off.p, g->adj.p, g->src.p, scratch.p, maxd, d_out);
  GPM_LAUNCH_CHECK();
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

}  // namespace gpm

using namespace gpm;

extern "C" int gpm_clique_ex(gpm_graph *g, int k, int variant, uint64_t *out) {
  if (!g || !out) return fail(GPM_EINVAL, "gpm_clique: NULL argument");
  if (k < 3 || k > kCqMaxK) return fail(GPM_EUNSUPPORTED, "k-clique supports 3 <= k <= 8");
  if (variant != GPM_CLIQUE_AUTO && variant != GPM_CLIQUE_EDGE) return fail(GPM_EINVAL, "unknown clique variant");
  GPM_TRY(g->result.reserve(8));
  GPM_TRY(clique_launch(g, k, 0, (unsigned long long *)g->result.p, variant == GPM_CLIQUE_EDGE));
  GPM_CUDA(cudaMemcpy(out, g->result.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return GPM_OK;
}

extern "C" int gpm_clique(gpm_graph *g, int k, uint64_t *out) { return gpm_clique_ex(g, k, GPM_CLIQUE_AUTO, out); }
