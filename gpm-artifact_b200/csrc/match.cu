// match.cu -- labelled subgraph matching with sub_ceci's semantics.
//
// sub_ceci (sub_ceci/myceci.cpp:540-668) counts every injective map phi of
// the query vertices into the data graph with label(phi(u)) == label(u) and
// every query edge mapped onto a data edge (non-induced; automorphic images
// are separate embeddings).  Its CECI filter and tree only prune; the count
// is that number.
//
// GPU design: the query (<= 64 vertices, sub_ceci's MAX_QUERY_VERTEX in
// sub_ceci/configuration/config.h:12) is ordered on the host -- start at
// the vertex whose label is rarest in the data graph (ties: higher degree),
// then repeatedly the unplaced vertex with most placed neighbours.  The data
// graph's lists are partitioned by label, so the candidates of a query
// vertex are one label segment of a mapped neighbour's list (the shortest
// one), and the other back-edges are checked by one bit test (vertices with
// an adjacency bitmap) or a binary search inside a label segment.  Tasks are
// the (root, second vertex) pairs -- extended breadth first to longer
// partial embeddings while they are too few to fill the GPU -- drained from
// an atomic cursor by a persistent grid; each warp walks its task depth first
// (k_match).
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"

constexpr int kMaxQ = 64;     // query vertices (sub_ceci/configuration/config.h:12)
constexpr int kNarrowQ = 16;  // plans up to this size take the narrow kernels

struct gpm_query {
  int n = 0;
  int32_t labels[kMaxQ];
  unsigned long long adjmask[kMaxQ];  // bit j set iff query edge (i, j)
  int deg[kMaxQ];
};

namespace gpm {

// A query in matching order, for queries of at most Q vertices.  Q = 16:
// 32-bit position masks and the kernels' static shared buffers (the common
// case, 6 CTAs per SM); Q = 64: 64-bit masks and buffers in dynamic shared
// memory.
template <int Q>
struct QueryPlanT {
  using Mask = typename std::conditional<(Q <= 32), uint32_t, unsigned long long>::type;
  int n;
  int order[Q];
  int parent_pos[Q];  // position (in order) of the parent, -1 for the root
  Mask back_pos[Q];   // bitmask of earlier positions that must be adjacent (parent excluded)
  int32_t label[Q];   // label of the vertex at each position
  int mindeg[Q];      // query degree at each position
};
using QueryPlan = QueryPlanT<kNarrowQ>;
using WidePlan = QueryPlanT<kMaxQ>;

// The plan of a query of at most Q vertices in the Q-wide layout.
template <int Q>
static void narrow_plan(const WidePlan &w, QueryPlanT<Q> *p) {
  memset(p, 0, sizeof *p);
  p->n = w.n;
  for (int k = 0; k < w.n && k < Q; ++k) {
    p->order[k] = w.order[k];
    p->parent_pos[k] = w.parent_pos[k];
    p->back_pos[k] = (typename QueryPlanT<Q>::Mask)w.back_pos[k];
    p->label[k] = w.label[k];
    p->mindeg[k] = w.mindeg[k];
  }
}

// Index of the lowest set bit of a non-zero position mask.
__device__ __forceinline__ int low_bit(uint32_t m) { return __ffs(m) - 1; }
__device__ __forceinline__ int low_bit(unsigned long long m) { return __ffsll((long long)m) - 1; }

__device__ __forceinline__ bool has_edge(const int64_t *__restrict__ off, const int32_t *__restrict__ adj, int32_t a,
                                         int32_t key) {
  int64_t lo = off[a], hi = off[a + 1] - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) >> 1;
    int32_t x = __ldg(adj + mid);
    if (x == key) return true;
    if (x < key) lo = mid + 1; else hi = mid - 1;
  }
  return false;
}

// [s, e): v's neighbours with label l inside its label-partitioned list,
// relative to off[v].  L == 0: the lists are not partitioned (labels >= 64),
// the whole list is scanned and the label test filters.
__device__ __forceinline__ void seg_range(const int64_t *__restrict__ off, const int32_t *__restrict__ loff, int L,
                                          int32_t v, int l, int64_t *s, int64_t *e) {
  if (L == 0) {
    *s = 0;
    *e = off[v + 1] - off[v];
  } else if (l < 0 || l >= L) {
    *s = *e = 0;
  } else {
    *s = loff[(int64_t)v * (L + 1) + l];
    *e = loff[(int64_t)v * (L + 1) + l + 1];
  }
}

// Is x in a's neighbours with label l?  Binary search inside a's label
// segment (the whole list when the lists are not partitioned).
__device__ __forceinline__ bool has_edge_label(const int64_t *__restrict__ off, const int32_t *__restrict__ adj,
                                               const int32_t *__restrict__ ladj, const int32_t *__restrict__ loff,
                                               int L, int32_t a, int l, int32_t x) {
  if (L == 0) return has_edge(off, adj, a, x);
  int64_t s, e;
  seg_range(off, loff, L, a, l, &s, &e);
  const int32_t *seg = ladj + off[a];
  int64_t lo = s, hi = e - 1;
  while (lo <= hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int32_t y = __ldg(seg + mid);
    if (y == x) return true;
    if (y < x) lo = mid + 1; else hi = mid - 1;
  }
  return false;
}

// Adjacency bitmaps of the high-degree vertices (cached with the label
// partition): hub slot of v (or -1) and, per hub, one bit per vertex id.  A
// membership test against a hub is one load instead of a binary search of up
// to log2(degree) dependent loads; the index trades HBM capacity (a few GB on
// R-MAT 21) for probe latency.
struct HubIndex {
  const int32_t *slot;  // n: bitmap row of v, -1 when v has no bitmap
  const uint32_t *bm;   // rows x words
  int64_t words;        // (n + 31) / 32
};

// Is x a neighbour of a with label l?  Bit test when a has a bitmap, else a
// binary search in a's label segment (x carries label l).
__device__ __forceinline__ bool adjacent(const HubIndex &hub, const int64_t *__restrict__ off,
                                         const int32_t *__restrict__ adj, const int32_t *__restrict__ ladj,
                                         const int32_t *__restrict__ loff, int L, int32_t a, int l, int32_t x) {
  const int32_t hs = hub.slot[a];
  if (hs >= 0) return (__ldg(hub.bm + hs * hub.words + (x >> 5)) >> (x & 31)) & 1u;
  return has_edge_label(off, adj, ladj, loff, L, a, l, x);
}

// Warp-level depth-first enumeration over (root, second vertex) tasks.
// Positions 2 .. n-2 walk their candidates lazily: the candidate source of a
// position is the shortest label segment among its mapped query-neighbours;
// 32 entries at a time are filtered (label, degree bound, injectivity, the
// other back-edges) and the survivors compacted into the warp's shared
// buffer of that position, so no candidate list is materialised in global
// memory and every SM keeps its full warp complement.  The last position is
// counted without a stack level: for all survivors y of one chunk of
// position n-2 at once, the last vertex's candidate segments (each y's
// shortest) are laid end to end and every lane takes one entry of the
// concatenation, so short segments do not leave lanes idle.
constexpr int kMatchWarps = 8;
struct MatchGraph {
  const int64_t *off;
  const int32_t *adj, *ladj, *loff, *labels;
  int L;
  HubIndex hub;
};

// The embeddings extending one partial embedding `row` (positions 0 .. t-1
// mapped, t >= 2: a (root, second vertex) pair, or a row of a breadth-first
// extension), by one warp; lane 0 returns the count (TRACK: counted into
// *found instead, see k_match).  chunk >= 0 restricts position t's
// candidates to the `span` entries from `chunk` on (tasks split by the batch
// path); buf is the warp's shared
// buffer of Q rows of 32 candidates (rows d - 2 for positions 2 .. n-2,
// the last two for the pool of position n-2's survivors).
template <bool TRACK, int Q>
__device__ __forceinline__ unsigned long long match_task(const QueryPlanT<Q> &q, const MatchGraph &G,
                                                         const int32_t *__restrict__ row, int t, int64_t chunk,
                                                         int64_t span,
                                                         int32_t (*buf)[32], unsigned long long limit,
                                                         unsigned long long *found, int32_t *__restrict__ emb_out) {
  const int64_t *__restrict__ off = G.off;
  const int32_t *__restrict__ adj = G.adj;
  const int32_t *__restrict__ ladj = G.ladj;
  const int32_t *__restrict__ loff = G.loff;
  const int32_t *__restrict__ labels = G.labels;
  const int L = G.L;
  const HubIndex &hub = G.hub;
  using Mask = typename QueryPlanT<Q>::Mask;
  const unsigned lane = lane_id();
  int32_t emb[Q] = {};
  int64_t pos[Q], end[Q];
  Mask chk[Q];
  int bcnt[Q], bcur[Q];
  const int last = q.n - 1, pre = q.n - 2;
  const int llab = q.label[last];
  const Mask lmask = q.back_pos[last] | ((Mask)1 << q.parent_pos[last]);
  unsigned long long c = 0;

  // candidate segment of position d: the shortest label segment among the
  // mapped query-neighbours, the others left to check (chk)
  auto open = [&](int d) {
    const int lab = q.label[d];
    const Mask nb = q.back_pos[d] | ((Mask)1 << q.parent_pos[d]);
    int src = q.parent_pos[d];
    int64_t s, e;
    seg_range(off, loff, L, emb[src], lab, &s, &e);
    if (L > 0)
      for (Mask bm = q.back_pos[d]; bm; bm &= bm - 1) {
        const int j = low_bit(bm);
        int64_t sj, ej;
        seg_range(off, loff, L, emb[j], lab, &sj, &ej);
        if (ej - sj < e - s) {
          src = j;
          s = sj;
          e = ej;
        }
      }
    chk[d] = nb & ~((Mask)1 << src);
    pos[d] = off[emb[src]] + s;
    end[d] = off[emb[src]] + e;
  };

  // next chunk of position d's candidates into buf[d - 2]; returns survivors
  auto fill = [&](int d) -> int {
    const int lab = q.label[d];
    const int64_t i = pos[d] + lane;
    bool ok = false;
    int32_t x = 0;
    if (i < end[d]) {
      x = __ldg(ladj + i);
      ok = (L > 0 || labels[x] == lab) && off[x + 1] - off[x] >= q.mindeg[d];
      for (int j = 0; ok && j < d; ++j) ok = emb[j] != x;
      for (Mask bm = chk[d]; ok && bm; bm &= bm - 1)
        ok = adjacent(hub, off, adj, ladj, loff, L, emb[low_bit(bm)], lab, x);
    }
    pos[d] += 32;
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) buf[d - 2][__popc(m & ((1u << lane) - 1u))] = x;
    __syncwarp();
    return __popc(m);
  };

  // embeddings completing positions 0 .. n-4 with (z, y) at positions
  // (n-3, n-2) (lane t < k holds pair t: pairs from several parents z are
  // pooled) and some last vertex
  auto close = [&](int32_t z, int32_t y, int k) {
    const int par = pre - 1;
    // lane t: its candidate's shortest segment for the last vertex
    int src = -1;
    long long st = 0, len = 0;
    if ((int)lane < k) {
      for (Mask bm = lmask; bm; bm &= bm - 1) {
        const int j = low_bit(bm);
        const int32_t a = j == pre ? y : j == par ? z : emb[j];
        int64_t s, e;
        seg_range(off, loff, L, a, llab, &s, &e);
        if (src < 0 || e - s < len) {
          src = j;
          st = off[a] + s;
          len = e - s;
        }
      }
    }
    long long inc = len;  // inclusive prefix over the lanes
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long v = __shfl_up_sync(0xffffffffu, inc, o);
      if ((int)lane >= o) inc += v;
    }
    const long long total = __shfl_sync(0xffffffffu, inc, 31);
    for (long long base = 0; base < total; base += 32) {
      const long long idx = base + lane;
      // t = first lane whose inclusive prefix exceeds idx
      int lo = 0, hi = 31;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const int mid = (lo + hi) >> 1;
        const long long pm = __shfl_sync(0xffffffffu, inc, mid);
        if (pm > idx) hi = mid; else lo = mid + 1;
      }
      const int t = lo;
      const long long pt = __shfl_sync(0xffffffffu, inc, t), lt = __shfl_sync(0xffffffffu, len, t);
      const long long stt = __shfl_sync(0xffffffffu, st, t);
      const int srct = __shfl_sync(0xffffffffu, src, t);
      const int32_t yt = __shfl_sync(0xffffffffu, y, t), zt = __shfl_sync(0xffffffffu, z, t);
      bool ok = false;
      int32_t x = 0;
      if (idx < total) {
        x = __ldg(ladj + stt + (idx - (pt - lt)));
        ok = (L > 0 || labels[x] == llab) && x != yt && x != zt;
        for (int j = 0; ok && j < par; ++j) ok = emb[j] != x;
        for (Mask bm = lmask & ~((Mask)1 << srct); ok && bm; bm &= bm - 1) {
          const int j = low_bit(bm);
          ok = adjacent(hub, off, adj, ladj, loff, L, j == pre ? yt : j == par ? zt : emb[j], llab, x);
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (TRACK && m) {
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(found, (unsigned long long)__popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        const unsigned long long slot = at + __popc(m & ((1u << lane) - 1u));
        if (emb_out && ok && slot < limit) {
          int32_t *row = emb_out + slot * (unsigned long long)q.n;
          for (int j = 0; j < par; ++j) row[q.order[j]] = emb[j];
          row[q.order[par]] = zt;
          row[q.order[pre]] = yt;
          row[q.order[last]] = x;
        }
      }
      c += lane == 0 ? (unsigned long long)__popc(m) : 0ull;
    }
  };

  for (int j = 0; j < t; ++j) emb[j] = row[j];
  if (pre == t - 1) {  // the row already maps position n-2
    close(emb[pre - 1], emb[pre], 1);
    return c;
  }
  // survivors of position n-2 pooled with their parent at n-3 (rows
  // Q-2 / Q-1 of buf) until 32 are pending or position n-4 moves on
  int np = 0;
  auto flush = [&]() {
    if (np) close((int)lane < np ? buf[Q - 1][lane] : 0, (int)lane < np ? buf[Q - 2][lane] : 0, np);
    np = 0;
  };
  int d = t;
  open(t);
  if (chunk >= 0) {
    pos[t] += chunk;
    end[t] = min(end[t], pos[t] + span);
  }
  bcnt[t] = bcur[t] = 0;
  while (d >= t) {
    if (TRACK && *(volatile unsigned long long *)found >= limit) break;
    if (d == pre) {
      if (pos[d] >= end[d]) {
        --d;
        continue;
      }
      const int k = fill(d);
      if (k) {
        if (np + k > 32) flush();
        if ((int)lane < k) {
          buf[Q - 2][np + lane] = buf[d - 2][lane];
          buf[Q - 1][np + lane] = emb[pre - 1];
        }
        __syncwarp();
        np += k;
      }
      continue;
    }
    if (bcur[d] < bcnt[d]) {
      emb[d] = buf[d - 2][bcur[d]++];
      ++d;
      open(d);
      bcnt[d] = bcur[d] = 0;
      continue;
    }
    if (pos[d] < end[d]) {
      bcnt[d] = fill(d);
      bcur[d] = 0;
      continue;
    }
    if (d == pre - 1) flush();  // position n-4 is about to move on
    --d;
  }
  flush();
  return c;
}

// One query over its partial embeddings (rows of t ids: the (root, second
// vertex) pairs, or the rows of a breadth-first extension), drained from an
// atomic cursor by a persistent grid.  TRACK: every embedding found takes a slot of
// *found; those below `limit` are written to emb_out (when given: q.n
// data-vertex ids per embedding, in query-vertex order), and the whole grid
// stops once `limit` are found (sub_ceci's -num, myceci.cpp:615-617).
// Otherwise the count goes to *out.
#ifndef GPM_MATCH_MIN_BLOCKS
// 6 CTAs per SM (at most 40 registers): R-MAT 21 4-cycle 1.81 s, diamond
// 3.78-3.83 s, R-MAT 18 house 5.25 s against 2.23-2.49 / 4.05 / 5.5 s at the
// 48 registers the compiler picks unbounded (5 CTAs per SM)
#define GPM_MATCH_MIN_BLOCKS 6
#endif
// Candidate rows of the wide kernels (Q > kNarrowQ): Q rows of 32 ids per
// warp in dynamic shared memory (64 KB per CTA at Q = 64).
template <int Q>
constexpr int match_dyn_smem() {
  return Q <= kNarrowQ ? 0 : kMatchWarps * Q * 32 * (int)sizeof(int32_t);
}
extern __shared__ __align__(16) int32_t match_dyn[];
// The calling warp's Q rows of 32 candidates.
template <int Q>
__device__ __forceinline__ int32_t (*warp_rows(int32_t (*narrow)[32]))[32] {
  return Q <= kNarrowQ ? narrow : reinterpret_cast<int32_t(*)[32]>(match_dyn + (threadIdx.x >> 5) * Q * 32);
}

template <bool TRACK, int Q>
__global__ void __launch_bounds__(kMatchWarps * 32, Q <= kNarrowQ ? GPM_MATCH_MIN_BLOCKS : 2)
    k_match(QueryPlanT<Q> q, MatchGraph G, const int32_t *__restrict__ rows, int t, int64_t n,
            unsigned long long *__restrict__ cursor, unsigned long long *__restrict__ out, unsigned long long limit,
            unsigned long long *found, int32_t *__restrict__ emb_out) {
  __shared__ int32_t sbuf[kMatchWarps][Q <= kNarrowQ ? Q : 1][32];
  int32_t(*buf)[32] = warp_rows<Q>(sbuf[threadIdx.x >> 5]);
  const unsigned lane = lane_id();
  unsigned long long c = 0;
  while (true) {
    unsigned long long r = 0;
    if (lane == 0) r = atomicAdd(cursor, 1ull);
    r = __shfl_sync(0xffffffffu, r, 0);
    if (r >= (unsigned long long)n) break;
    if (TRACK && *(volatile unsigned long long *)found >= limit) break;
    c += match_task<TRACK, Q>(q, G, rows + (int64_t)r * t, t, -1, 0, buf, limit, found, emb_out);
  }
  if (TRACK) return;
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}

// One position more for a list of partial embeddings (rows of t ids,
// positions 0 .. t-1 mapped): every candidate of position t that passes
// match_task's filters (its label segment of the mapped query-neighbour with
// the shortest one, degree bound, injectivity, the other back-edges) makes a
// row of t + 1 ids.  A warp per row; survivors are counted into *cnt and
// written to out while their slot is below cap (out == nullptr: counted only).
__global__ void k_extend_rows(WidePlan q, MatchGraph G, const int32_t *__restrict__ rows, int64_t nrows, int t,
                              int32_t *__restrict__ out, unsigned long long cap,
                              unsigned long long *__restrict__ cnt) {
  const int64_t *__restrict__ off = G.off;
  const int32_t *__restrict__ ladj = G.ladj;
  const int32_t *__restrict__ loff = G.loff;
  const int L = G.L;
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lab = q.label[t];
  for (int64_t r = warp; r < nrows; r += nw) {
    const int32_t *row = rows + r * t;
    int src = q.parent_pos[t];
    int64_t s, e;
    seg_range(off, loff, L, row[src], lab, &s, &e);
    if (L > 0)
      for (unsigned long long bm = q.back_pos[t]; bm; bm &= bm - 1) {
        const int j = low_bit(bm);
        int64_t sj, ej;
        seg_range(off, loff, L, row[j], lab, &sj, &ej);
        if (ej - sj < e - s) {
          src = j;
          s = sj;
          e = ej;
        }
      }
    const unsigned long long chk = (q.back_pos[t] | (1ull << q.parent_pos[t])) & ~(1ull << src);
    const int64_t base = off[row[src]];
    for (int64_t i0 = base + s; i0 < base + e; i0 += 32) {
      const int64_t i = i0 + lane;
      bool ok = false;
      int32_t x = 0;
      if (i < base + e) {
        x = __ldg(ladj + i);
        ok = (L > 0 || G.labels[x] == lab) && off[x + 1] - off[x] >= q.mindeg[t];
        for (int j = 0; ok && j < t; ++j) ok = row[j] != x;
        for (unsigned long long bm = chk; ok && bm; bm &= bm - 1)
          ok = adjacent(G.hub, off, G.adj, ladj, loff, L, row[low_bit(bm)], lab, x);
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (!m) continue;
      unsigned long long at = 0;
      if (lane == 0) at = atomicAdd(cnt, (unsigned long long)__popc(m));
      at = __shfl_sync(0xffffffffu, at, 0);
      const unsigned long long slot = at + __popc(m & ((1u << lane) - 1u));
      if (out && ok && slot < cap) {
        int32_t *o = out + slot * (unsigned long long)(t + 1);
        for (int j = 0; j < t; ++j) o[j] = row[j];
        o[t] = x;
      }
    }
  }
}

// Embeddings of a one- or two-vertex query into emb_out (slots below
// limit): roots with the query root's label, or the materialised pairs.
__global__ void k_list_small(WidePlan q, int64_t n, const int32_t *__restrict__ labels, const int64_t *__restrict__ off,
                             const int2 *__restrict__ pairs, int64_t npairs, unsigned long long limit,
                             unsigned long long *__restrict__ found, int32_t *__restrict__ emb_out) {
  const int64_t tot = q.n == 1 ? n : npairs;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    if (q.n == 1) {
      if (labels[i] != q.label[0]) continue;
      const unsigned long long slot = atomicAdd(found, 1ull);
      if (slot < limit) emb_out[slot] = (int32_t)i;
    } else {
      const unsigned long long slot = atomicAdd(found, 1ull);
      if (slot < limit) {
        emb_out[slot * 2 + q.order[0]] = pairs[i].x;
        emb_out[slot * 2 + q.order[1]] = pairs[i].y;
      }
    }
  }
}

// (root, second) pairs: a warp per root with the query root's label; the
// second vertex comes from the root's segment of the second query vertex's
// label.  count_only: the query has two vertices, so the pairs are the answer.
__global__ void k_match_pairs(WidePlan q, int64_t n, const int64_t *__restrict__ off,
                              const int32_t *__restrict__ ladj, const int32_t *__restrict__ loff, int L,
                              const int32_t *__restrict__ labels, int count_only, int2 *__restrict__ pairs,
                              unsigned long long *__restrict__ npairs) {
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = warp; v < n; v += nw) {
    if (labels[v] != q.label[0] || off[v + 1] - off[v] < q.mindeg[0]) continue;
    const int32_t *seg = ladj + off[v];
    int64_t s, e;
    seg_range(off, loff, L, (int32_t)v, q.label[1], &s, &e);
    for (int64_t base = s; base < e; base += 32) {
      int64_t i = base + lane;
      int32_t x = 0;
      bool ok = false;
      if (i < e) {
        x = __ldg(seg + i);
        ok = labels[x] == q.label[1] && off[x + 1] - off[x] >= q.mindeg[1];
      }
      unsigned m = __ballot_sync(0xffffffffu, ok);
      if (!m) continue;
      unsigned long long at = 0;
      if (lane == 0) at = atomicAdd(npairs, (unsigned long long)__popc(m));
      at = __shfl_sync(0xffffffffu, at, 0);
      if (!count_only && ok) pairs[at + __popc(m & ((1u << lane) - 1u))] = make_int2((int32_t)v, x);
    }
  }
}

// Label-partitioned copy of the lists: neighbours sorted by (label, id); loff
// holds, per vertex, the L + 1 segment starts relative to off[v].
__global__ void k_label_keys(int64_t nnz, const int32_t *__restrict__ adj, const int32_t *__restrict__ labels, int L,
                             uint64_t *__restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t w = adj[i];
    uint32_t l = L > 1 ? (uint32_t)labels[w] : 0u;
    keys[i] = ((uint64_t)l << 32) | (uint32_t)w;
  }
}
__global__ void k_label_offsets(int64_t n, const int64_t *__restrict__ off, const uint64_t *__restrict__ keys, int L,
                                int32_t *__restrict__ ladj, int32_t *__restrict__ loff) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = lane_id();
  for (int64_t v = warp; v < n; v += nw) {
    const int64_t s = off[v], e = off[v + 1];
    // segment start of label l = number of entries with label < l (sorted)
    for (int l = lane; l <= L; l += 32) {
      int64_t lo = s, hi = e;
      while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((int64_t)(keys[mid] >> 32) < l) lo = mid + 1; else hi = mid;
      }
      loff[v * (L + 1) + l] = (int32_t)(lo - s);
    }
    for (int64_t k = s + lane; k < e; k += 32) ladj[k] = (int32_t)(keys[k] & 0xffffffffu);
  }
}

static int plan_query(const gpm_query *q, const std::vector<int64_t> &label_freq, WidePlan *p) {
  const int n = q->n;
  memset(p, 0, sizeof *p);
  p->n = n;
  bool placed[kMaxQ] = {false};
  int best = 0;
  auto freq = [&](int u) -> int64_t {
    int32_t l = q->labels[u];
    return (l >= 0 && (size_t)l < label_freq.size()) ? label_freq[l] : 0;
  };
  for (int u = 1; u < n; ++u)
    if (freq(u) < freq(best) || (freq(u) == freq(best) && q->deg[u] > q->deg[best])) best = u;
  p->order[0] = best;
  placed[best] = true;
  for (int k = 1; k < n; ++k) {
    int b = -1, bs = -1, bd = -1;
    for (int u = 0; u < n; ++u) {
      if (placed[u]) continue;
      int s = 0;
      for (int w = 0; w < n; ++w) s += placed[w] && ((q->adjmask[u] >> w) & 1u);
      if (s > bs || (s == bs && q->deg[u] > bd)) {
        b = u;
        bs = s;
        bd = q->deg[u];
      }
    }
    if (bs <= 0) return fail(GPM_EUNSUPPORTED, "query graph must be connected");
    p->order[k] = b;
    placed[b] = true;
  }
  for (int k = 0; k < n; ++k) {
    int u = p->order[k];
    p->label[k] = q->labels[u];
    p->mindeg[k] = q->deg[u];
    p->parent_pos[k] = -1;
    p->back_pos[k] = 0;
    for (int j = 0; j < k; ++j) {
      if (!((q->adjmask[u] >> p->order[j]) & 1u)) continue;
      if (p->parent_pos[k] < 0) p->parent_pos[k] = j;
      else p->back_pos[k] |= 1ull << j;
    }
  }
  return GPM_OK;
}

// Label-partitioned copy of a labelled graph's lists (cached per graph).
struct LabelCsr {
  int L = 0;  // partitions (max label + 1); 0: labels too wide, lists copied as they are
  DevBuf<int32_t> ladj, loff;
  // adjacency bitmaps of the vertices with at least hub_min neighbours
  DevBuf<int32_t> hub_slot;
  DevBuf<uint32_t> hub_bm;
  int64_t hub_words = 0;
  int hubs = 0, hub_min = 0;
};
void free_label_csr(LabelCsr *p) { delete p; }

__global__ void k_label_range(int64_t n, const int32_t *__restrict__ labels, int *__restrict__ mm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    atomicMax(&mm[0], labels[i]);
    atomicMin(&mm[1], labels[i]);
  }
}

__global__ void k_deg_hist(int64_t n, const int64_t *__restrict__ off, unsigned long long *__restrict__ h) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = off[v + 1] - off[v];
    atomicAdd(&h[d > 0 ? 64 - __clzll((unsigned long long)d) : 0], 1ull);  // bin b: 2^(b-1) <= d < 2^b
  }
}
__global__ void k_hub_slots(int64_t n, const int64_t *__restrict__ off, int64_t dmin, int32_t *__restrict__ slot,
                            int *__restrict__ cnt) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    slot[v] = off[v + 1] - off[v] >= dmin ? atomicAdd(cnt, 1) : -1;
}
__global__ void k_hub_fill(int64_t n, const int64_t *__restrict__ off, const int32_t *__restrict__ adj,
                           const int32_t *__restrict__ slot, int64_t words, uint32_t *__restrict__ bm) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = warp; v < n; v += nw) {
    const int32_t hs = slot[v];
    if (hs < 0) continue;
    uint32_t *row = bm + hs * words;
    for (int64_t k = off[v] + lane_id(); k < off[v + 1]; k += 32) {
      const int32_t x = adj[k];
      atomicOr(row + (x >> 5), 1u << (x & 31));
    }
  }
}

// Adjacency bitmaps for the highest-degree vertices: the smallest power-of-two
// degree bound (at least kHubMinDegree) whose bitmaps fit the byte budget
// (GPM_HUB_BITMAP_BYTES, default 8 GiB, at most a quarter of the free memory).
constexpr int64_t kHubMinDegree = 256;
static int build_hub_index(gpm_graph *g, LabelCsr *lc) {
  const int64_t n = g->n, words = (n + 31) / 32;
  GPM_TRY(lc->hub_slot.reserve(std::max<int64_t>(n, 1)));
  lc->hub_words = words;
  if (n == 0) return GPM_OK;
  DevBuf<unsigned long long> h;
  GPM_TRY(h.reserve(65));
  GPM_CUDA(cudaMemset(h.p, 0, 65 * sizeof(unsigned long long)));
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16);
  k_deg_hist<<<blocks, 256>>>(n, g->off.p, h.p);
  unsigned long long hist[65];
  GPM_CUDA(cudaMemcpy(hist, h.p, sizeof hist, cudaMemcpyDeviceToHost));
  size_t free_b = 0, total_b = 0;
  GPM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  int64_t budget = (int64_t)8 << 30;
  if (const char *e = getenv("GPM_HUB_BITMAP_BYTES")) budget = atoll(e);
  budget = std::min<int64_t>(budget, (int64_t)(free_b / 4));
  // vertices with degree >= 2^(b-1) are those in bins b .. 64
  int64_t dmin = 0, count = 0;
  for (int b = 1; b <= 64; ++b) {
    unsigned long long above = 0;
    for (int k = b; k <= 64; ++k) above += hist[k];
    const int64_t d = (int64_t)1 << (b - 1);
    if (d < kHubMinDegree) continue;
    if ((int64_t)above * words * 4 <= budget) {
      dmin = d;
      count = (int64_t)above;
      break;
    }
  }
  DevBuf<int> cnt;
  GPM_TRY(cnt.reserve(1));
  GPM_CUDA(cudaMemset(cnt.p, 0, sizeof(int)));
  if (count == 0) {
    GPM_CUDA(cudaMemset(lc->hub_slot.p, 0xff, sizeof(int32_t) * n));
    lc->hubs = 0;
    lc->hub_min = 0;
    GPM_TRY(lc->hub_bm.reserve(1));
    return GPM_OK;
  }
  GPM_TRY(lc->hub_bm.reserve((size_t)(count * words)));
  GPM_CUDA(cudaMemset(lc->hub_bm.p, 0, sizeof(uint32_t) * count * words));
  k_hub_slots<<<blocks, 256>>>(n, g->off.p, dmin, lc->hub_slot.p, cnt.p);
  k_hub_fill<<<(int)std::min<int64_t>((n * 32 + 255) / 256, (int64_t)num_sms() * 16), 256>>>(
      n, g->off.p, g->adj.p, lc->hub_slot.p, words, lc->hub_bm.p);
  GPM_LAUNCH_CHECK();
  lc->hubs = (int)count;
  lc->hub_min = (int)dmin;
  return GPM_OK;
}

static int ensure_label_csr(gpm_graph *g) {
  if (g->lcsr) return GPM_OK;
  const int64_t n = g->n, nnz = g->nnz;
  LabelCsr *lc = new LabelCsr();
  auto bail = [&](int s) {
    delete lc;
    return s;
  };
  int s;
  DevBuf<int> mm;
  if ((s = mm.reserve(2)) || (s = lc->ladj.reserve(nnz))) return bail(s);
  int init[2] = {INT32_MIN, INT32_MAX}, h[2] = {0, 0};
  cudaMemcpy(mm.p, init, sizeof init, cudaMemcpyHostToDevice);
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16);
  if (n > 0) k_label_range<<<std::max(1, blocks), 256>>>(n, g->labels.p, mm.p);
  cudaMemcpy(h, mm.p, sizeof h, cudaMemcpyDeviceToHost);
  const int L = (n > 0 && h[1] >= 0 && h[0] < 64) ? h[0] + 1 : 0;
  lc->L = L;
  if (L == 0) {
    if ((s = lc->loff.reserve(1))) return bail(s);
    if (nnz > 0) cudaMemcpy(lc->ladj.p, g->adj.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice);
  } else {
    DevBuf<uint64_t> keys, sorted;
    if ((s = lc->loff.reserve((size_t)n * (L + 1))) || (s = keys.reserve(nnz)) || (s = sorted.reserve(nnz)))
      return bail(s);
    if (nnz > 0) {
      k_label_keys<<<(int)std::min<int64_t>((nnz + 255) / 256, num_sms() * 16), 256>>>(nnz, g->adj.p, g->labels.p, L,
                                                                                      keys.p);
      size_t tmp = 0;
      cub::DeviceSegmentedSort::SortKeys(nullptr, tmp, keys.p, sorted.p, (int)nnz, (int)n, g->off.p, g->off.p + 1);
      DevBuf<char> t;
      if ((s = t.reserve(tmp))) return bail(s);
      cub::DeviceSegmentedSort::SortKeys(t.p, tmp, keys.p, sorted.p, (int)nnz, (int)n, g->off.p, g->off.p + 1);
    }
    k_label_offsets<<<(int)std::min<int64_t>((n * 32 + 255) / 256, num_sms() * 16), 256>>>(n, g->off.p, sorted.p, L,
                                                                                          lc->ladj.p, lc->loff.p);
  }
  if ((s = build_hub_index(g, lc))) return bail(s);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("label partition: ") + cudaGetErrorString(e)));
  g->lcsr = lc;
  return GPM_OK;
}

__global__ void k_label_hist(int64_t n, const int32_t *__restrict__ labels, int nl, unsigned long long *__restrict__ h) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t l = labels[i];
    if (l >= 0 && l < nl) atomicAdd(&h[l], 1ull);
  }
}

}  // namespace gpm

using namespace gpm;

extern "C" {

int gpm_query_create(int64_t n, int64_t m, const int32_t *src, const int32_t *dst, const int32_t *labels,
                     gpm_query **out) {
  if (!out || !labels || n < 1 || m < 0 || (m > 0 && (!src || !dst)))
    return fail(GPM_EINVAL, "gpm_query_create: bad argument");
  if (n > kMaxQ) return fail(GPM_EUNSUPPORTED, "query graphs are limited to 64 vertices");
  gpm_query *q = new gpm_query();
  q->n = (int)n;
  for (int i = 0; i < n; ++i) {
    q->labels[i] = labels[i];
    q->adjmask[i] = 0;
  }
  for (int64_t e = 0; e < m; ++e) {
    int a = src[e], b = dst[e];
    if (a < 0 || b < 0 || a >= n || b >= n) {
      delete q;
      return fail(GPM_EINVAL, "query edge out of range");
    }
    if (a == b) continue;
    q->adjmask[a] |= 1ull << b;
    q->adjmask[b] |= 1ull << a;
  }
  for (int i = 0; i < n; ++i) q->deg[i] = __builtin_popcountll(q->adjmask[i]);
  *out = q;
  return GPM_OK;
}

int gpm_query_destroy(gpm_query *q) {
  delete q;
  return GPM_OK;
}

}  // extern "C"

namespace gpm {

// One k_match launch over the (root, second vertex) pairs on a persistent
// grid (occupancy x SMs, per device and plan width).
template <int Q>
static int launch_match(const QueryPlanT<Q> &plan, const MatchGraph &G, const int32_t *rows, int t, int64_t nrows,
                        unsigned long long *cursor, unsigned long long *out, bool track, unsigned long long limit,
                        unsigned long long *found, int32_t *emb) {
  constexpr int smem = match_dyn_smem<Q>();
  static PerDevice match_grid;
  const int grid = match_grid.get([] {
    if (smem > 0) {
      cudaFuncSetAttribute(k_match<false, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      cudaFuncSetAttribute(k_match<true, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match<false, Q>, kMatchWarps * 32, smem);
    return std::max(1, per_sm) * num_sms();
  });
  if (track)
    k_match<true, Q><<<grid, kMatchWarps * 32, smem>>>(plan, G, rows, t, nrows, cursor, out, limit, found, emb);
  else
    k_match<false, Q><<<grid, kMatchWarps * 32, smem>>>(plan, G, rows, t, nrows, cursor, out, limit, found, nullptr);
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

// Rows to aim for before the depth-first kernels start: about five per
// resident warp (48 per SM).
static int64_t row_target() { return (int64_t)num_sms() * 256; }

// Breadth-first extension of a query's partial embeddings while they are
// too few to fill the grid (small data graphs, rare labels, deep queries):
// the rows of depth t (the (root, second vertex) pairs at t = 2) are extended
// one position per step until there are at least `target` rows, t reaches
// n - 1, or the next level would pass 2 GiB (or an eighth of the free
// memory).  On return *rows, *nrows and *t describe the last level, held by
// *store unless it is still the caller's; *nrows == 0: no embedding.
static int extend_rows(const WidePlan &plan, const MatchGraph &G, DevBuf<int32_t> *store, const int32_t **rows,
                       int64_t *nrows, int *t, int64_t target) {
  if (*nrows == 0 || *nrows >= target || *t >= plan.n - 1) return GPM_OK;
  size_t free_b = 0, total_b = 0;
  GPM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const unsigned long long budget = std::min<unsigned long long>(2ull << 30, free_b / 8);
  DevBuf<unsigned long long> cnt;
  GPM_TRY(cnt.reserve(1));
  const int blocks = num_sms() * 8;
  while (*nrows > 0 && *nrows < target && *t < plan.n - 1) {
    GPM_CUDA(cudaMemset(cnt.p, 0, 8));
    k_extend_rows<<<blocks, 256>>>(plan, G, *rows, *nrows, *t, nullptr, 0, cnt.p);
    GPM_LAUNCH_CHECK();
    unsigned long long nn = 0;
    GPM_CUDA(cudaMemcpy(&nn, cnt.p, 8, cudaMemcpyDeviceToHost));
    if (nn * (unsigned long long)(*t + 1) * sizeof(int32_t) > budget) break;
    DevBuf<int32_t> next;
    if (nn) {
      GPM_TRY(next.reserve((size_t)nn * (*t + 1)));
      GPM_CUDA(cudaMemset(cnt.p, 0, 8));
      k_extend_rows<<<blocks, 256>>>(plan, G, *rows, *nrows, *t, next.p, nn, cnt.p);
      GPM_LAUNCH_CHECK();
      GPM_CUDA(cudaDeviceSynchronize());  // the previous level is released below
    }
    *store = std::move(next);
    *rows = store->p;
    *nrows = (int64_t)nn;
    ++*t;
  }
  return GPM_OK;
}

// The embeddings of q in g: counted (limit = ~0, emb = nullptr), counted up
// to `limit`, or listed (emb: host array of limit * q->n ids).  *out = the
// count, min(total, limit).
static int match_run(gpm_graph *g, const gpm_query *q, unsigned long long limit, int32_t *emb, uint64_t *out) {
  if (!g || !q || !out) return fail(GPM_EINVAL, "gpm_match: NULL argument");
  if (!g->labels.p) return fail(GPM_EINVAL, "the data graph carries no labels");
  if (g->oriented) return fail(GPM_EINVAL, "matching needs the symmetric (unoriented) data graph");
  const bool track = limit != ~0ull || emb;
  *out = 0;
  if (limit == 0) return GPM_OK;
  // label frequencies pick the root
  int maxl = 0;
  for (int i = 0; i < q->n; ++i) maxl = std::max(maxl, q->labels[i] + 1);
  std::vector<int64_t> freq(maxl, 0);
  {
    DevBuf<unsigned long long> h;
    GPM_TRY(h.reserve(maxl));
    GPM_CUDA(cudaMemset(h.p, 0, sizeof(unsigned long long) * maxl));
    if (g->n > 0) k_label_hist<<<(int)std::min<int64_t>((g->n + 255) / 256, num_sms() * 8), 256>>>(g->n, g->labels.p, maxl, h.p);
    std::vector<unsigned long long> hh(maxl);
    GPM_CUDA(cudaMemcpy(hh.data(), h.p, sizeof(unsigned long long) * maxl, cudaMemcpyDeviceToHost));
    for (int i = 0; i < maxl; ++i) freq[i] = (int64_t)hh[i];
  }
  WidePlan plan;
  GPM_TRY(plan_query(q, freq, &plan));
  DevBuf<unsigned long long> found;
  DevBuf<int32_t> demb;
  GPM_TRY(found.reserve(1));
  GPM_CUDA(cudaMemset(found.p, 0, 8));
  auto finish = [&](unsigned long long total) -> int {
    const unsigned long long got = std::min<unsigned long long>(total, limit);
    if (emb && got) GPM_CUDA(cudaMemcpy(emb, demb.p, sizeof(int32_t) * got * q->n, cudaMemcpyDeviceToHost));
    *out = got;
    return GPM_OK;
  };
  if (emb) GPM_TRY(demb.reserve(std::max<unsigned long long>(1, limit) * q->n));
  const int sblocks = (int)std::min<int64_t>((g->n + 255) / 256 + 1, (int64_t)num_sms() * 8);
  if (q->n == 1) {
    const unsigned long long total =
        (unsigned long long)(plan.label[0] >= 0 && plan.label[0] < maxl ? freq[plan.label[0]] : 0);
    if (emb && total) {
      k_list_small<<<sblocks, 256>>>(plan, g->n, g->labels.p, g->off.p, nullptr, 0, limit, found.p, demb.p);
      GPM_LAUNCH_CHECK();
    }
    return finish(total);
  }
  GPM_TRY(ensure_label_csr(g));
  LabelCsr *lc = g->lcsr;
  const int blocks = (int)std::min<int64_t>((g->n * 32 + 255) / 256, (int64_t)num_sms() * 16);
  DevBuf<unsigned long long> d, npairs;
  GPM_TRY(d.reserve(1));
  GPM_TRY(npairs.reserve(1));
  GPM_CUDA(cudaMemset(npairs.p, 0, 8));
  // (root, second vertex) pairs: counted, then materialised
  k_match_pairs<<<blocks, 256>>>(plan, g->n, g->off.p, lc->ladj.p, lc->loff.p, lc->L, g->labels.p, 1, nullptr,
                                 npairs.p);
  GPM_LAUNCH_CHECK();
  unsigned long long np = 0;
  GPM_CUDA(cudaMemcpy(&np, npairs.p, 8, cudaMemcpyDeviceToHost));
  if (np == 0 || (q->n == 2 && !emb)) return finish(np);
  DevBuf<int2> pairs;
  GPM_TRY(pairs.reserve(np));
  GPM_CUDA(cudaMemset(npairs.p, 0, 8));
  k_match_pairs<<<blocks, 256>>>(plan, g->n, g->off.p, lc->ladj.p, lc->loff.p, lc->L, g->labels.p, 0, pairs.p,
                                 npairs.p);
  GPM_LAUNCH_CHECK();
  if (q->n == 2) {
    k_list_small<<<sblocks, 256>>>(plan, g->n, g->labels.p, g->off.p, pairs.p, (int64_t)np, limit, found.p, demb.p);
    GPM_LAUNCH_CHECK();
    return finish(np);
  }
  const HubIndex hub{lc->hub_slot.p, lc->hub_bm.p, lc->hub_words};
  const MatchGraph G{g->off.p, g->adj.p, lc->ladj.p, lc->loff.p, g->labels.p, lc->L, hub};
  // the pairs are rows of two ids; too few of them are extended first
  const int32_t *rows = reinterpret_cast<const int32_t *>(pairs.p);
  int64_t nrows = (int64_t)np;
  int t = 2;
  DevBuf<int32_t> store;
  GPM_TRY(extend_rows(plan, G, &store, &rows, &nrows, &t, row_target()));
  if (nrows == 0) return finish(0);
  DevBuf<unsigned long long> cursor;
  GPM_TRY(cursor.reserve(1));
  GPM_CUDA(cudaMemset(cursor.p, 0, 8));
  GPM_CUDA(cudaMemset(d.p, 0, 8));
  if (plan.n <= kNarrowQ) {
    QueryPlan p16;
    narrow_plan(plan, &p16);
    GPM_TRY(launch_match(p16, G, rows, t, nrows, cursor.p, d.p, track, limit, found.p, emb ? demb.p : nullptr));
  } else {
    GPM_TRY(launch_match(plan, G, rows, t, nrows, cursor.p, d.p, track, limit, found.p, emb ? demb.p : nullptr));
  }
  unsigned long long h = 0;
  GPM_CUDA(cudaMemcpy(&h, track ? found.p : d.p, 8, cudaMemcpyDeviceToHost));
  return finish(h);
}

}  // namespace gpm

extern "C" {

int gpm_match(gpm_graph *g, const gpm_query *q, uint64_t *out) { return match_run(g, q, ~0ull, nullptr, out); }

int gpm_match_limit(gpm_graph *g, const gpm_query *q, uint64_t limit, uint64_t *out) {
  return match_run(g, q, limit, nullptr, out);
}

int gpm_match_list(gpm_graph *g, const gpm_query *q, uint64_t limit, int32_t *emb, uint64_t *written) {
  if (!emb && limit > 0) return fail(GPM_EINVAL, "gpm_match_list: NULL output");
  return match_run(g, q, limit, emb, written);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Many labelled queries on one data graph in one persistent launch.
//
// The reference runs one kernel per pattern and synchronises after each
// (src/PatternSolver.cuh:177-246).  Here the (root, second vertex) pairs of
// every query become one task list, each task carrying its query; a warp
// loads its task's plan into shared memory and walks the task with the same
// depth-first code as gpm_match, so the GPU stays busy across query
// boundaries and no query waits for another's tail.  Tasks of 4+ vertex
// queries can be split over chunks of position 2's candidates (the span
// chosen by gpm_match_batch_autotune) so hub tasks do not form the tail.
// With a member id per vertex (many graphs as one disjoint union), each
// embedding is counted for its root's member.  The launch (cursor reset,
// count reset, kernel) is captured into a CUDA graph and replayed.
// ---------------------------------------------------------------------------
struct gpm_match_batch {
  gpm_graph *g = nullptr;
  int nq = 0, nm = 1;
  int qcap = 16;  // plan width of the launch: 16, or 64 when a query has more than 16 vertices
  std::vector<gpm::WidePlan> plans;
  std::vector<gpm::DevBuf<int2>> pairs;  // per query (empty for 1- and 2-vertex queries)
  std::vector<int64_t> npairs;
  // per query: its task rows (the pairs, or their breadth-first extension
  // held in ext), their count and depth
  std::vector<gpm::DevBuf<int32_t>> ext;
  std::vector<const int32_t *> rows;
  std::vector<int64_t> nrows;
  std::vector<int> depth;
  gpm::DevBuf<int4> drows;               // nq x (rows pointer lo, hi, depth, -)
  gpm::DevBuf<char> dplans;              // nq plans of width qcap
  gpm::DevBuf<int32_t> member;           // n (nm > 1 only)
  gpm::DevBuf<unsigned long long> base;  // counts of 1- and 2-vertex queries, nq * nm
  gpm::DevBuf<unsigned long long> out, cursor;
  gpm::DevBuf<int4> tasks;               // (row index lo, hi, query, chunk or -1)
  int64_t ntasks = 0, span = 0;
  int grid = 0;  // persistent grid of k_match_batch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~gpm_match_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

namespace gpm {

template <int Q>
__global__ void __launch_bounds__(kMatchWarps * 32, Q <= kNarrowQ ? GPM_MATCH_MIN_BLOCKS : 2)
    k_match_batch(const QueryPlanT<Q> *__restrict__ plans, const int4 *__restrict__ qrows, MatchGraph G,
                  const int4 *__restrict__ tasks, int64_t ntasks, int64_t span, const int32_t *__restrict__ member,
                  int nm, unsigned long long *__restrict__ cursor, unsigned long long *__restrict__ out) {
  __shared__ int32_t sbuf[kMatchWarps][Q <= kNarrowQ ? Q : 1][32];
  __shared__ QueryPlanT<Q> splan[kMatchWarps];
  static_assert(sizeof(QueryPlanT<Q>) % 4 == 0, "plan copied as words");
  const int w = threadIdx.x >> 5;
  int32_t(*buf)[32] = warp_rows<Q>(sbuf[w]);
  const unsigned lane = lane_id();
  int cur = -1;
  while (true) {
    unsigned long long r = 0;
    if (lane == 0) r = atomicAdd(cursor, 1ull);
    r = __shfl_sync(0xffffffffu, r, 0);
    if (r >= (unsigned long long)ntasks) break;
    const int4 t = tasks[r];
    if (t.z != cur) {
      __syncwarp();
      const int32_t *src = reinterpret_cast<const int32_t *>(plans + t.z);
      int32_t *dst = reinterpret_cast<int32_t *>(&splan[w]);
      for (int i = lane; i < (int)(sizeof(QueryPlanT<Q>) / 4); i += 32) dst[i] = src[i];
      __syncwarp();
      cur = t.z;
    }
    const int4 qr = qrows[t.z];
    const int32_t *rows = reinterpret_cast<const int32_t *>(((unsigned long long)(unsigned)qr.y << 32) |
                                                             (unsigned)qr.x);
    const int32_t *row = rows + (((int64_t)t.y << 32) | (unsigned)t.x) * qr.z;
    const unsigned long long c = match_task<false, Q>(splan[w], G, row, qr.z, t.w < 0 ? -1 : (int64_t)t.w * span,
                                                      span, buf, ~0ull, nullptr, nullptr);
    if (lane == 0 && c) atomicAdd(&out[(int64_t)t.z * nm + (member ? member[row[0]] : 0)], c);
  }
}

// Position t's candidate count of each row (the segment match_task opens:
// the parent's label segment, or a shorter one of another mapped
// query-neighbour when the lists are label-partitioned), as the task count of
// the row: ceil(len / span), at least 1.
__global__ void k_row_tasks(WidePlan q, const int32_t *__restrict__ rows, int64_t nrows, int t,
                            const int64_t *__restrict__ off, const int32_t *__restrict__ loff, int L, int64_t span,
                            int64_t *__restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t *row = rows + i * t;
    const int lab = q.label[t];
    int64_t s, e;
    seg_range(off, loff, L, row[q.parent_pos[t]], lab, &s, &e);
    int64_t best = e - s;
    if (L > 0)
      for (unsigned long long bm = q.back_pos[t]; bm; bm &= bm - 1) {
        seg_range(off, loff, L, row[low_bit(bm)], lab, &s, &e);
        best = min(best, e - s);
      }
    cnt[i] = span > 0 ? max((int64_t)1, (best + span - 1) / span) : 1;
  }
}
__global__ void k_expand_tasks(int64_t nrows, const int64_t *__restrict__ first, const int64_t *__restrict__ cnt,
                               int query, int split, int4 *__restrict__ tasks) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x)
    for (int64_t c = 0; c < cnt[i]; ++c)
      tasks[first[i] + c] = make_int4((int)(uint32_t)i, (int)(i >> 32), query, split ? (int)c : -1);
}
// per-member counts of a one-vertex query (vertices with its label) or of a
// two-vertex query (its pairs, by the root's member)
__global__ void k_small_counts(int64_t n, const int32_t *__restrict__ labels, int label, const int2 *__restrict__ pairs,
                               int64_t np, const int32_t *__restrict__ member, unsigned long long *__restrict__ dst) {
  const int64_t tot = pairs ? np : n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    if (pairs) atomicAdd(&dst[member ? member[pairs[i].x] : 0], 1ull);
    else if (labels[i] == label) atomicAdd(&dst[member ? member[i] : 0], 1ull);
  }
}

static int label_freq(gpm_graph *g, int maxl, std::vector<int64_t> &freq) {
  freq.assign(maxl, 0);
  DevBuf<unsigned long long> h;
  GPM_TRY(h.reserve(maxl));
  GPM_CUDA(cudaMemset(h.p, 0, sizeof(unsigned long long) * maxl));
  if (g->n > 0)
    k_label_hist<<<(int)std::min<int64_t>((g->n + 255) / 256, num_sms() * 8), 256>>>(g->n, g->labels.p, maxl, h.p);
  std::vector<unsigned long long> hh(maxl);
  GPM_CUDA(cudaMemcpy(hh.data(), h.p, sizeof(unsigned long long) * maxl, cudaMemcpyDeviceToHost));
  for (int i = 0; i < maxl; ++i) freq[i] = (int64_t)hh[i];
  return GPM_OK;
}

static void drop_batch_graph(gpm_match_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// The task list for a given split span (0: one task per pair).
static int batch_tasks(gpm_match_batch *b, int64_t span) {
  gpm_graph *g = b->g;
  LabelCsr *lc = g->lcsr;
  std::vector<int64_t> cnt_total(b->nq, 0);
  std::vector<DevBuf<int64_t>> cnt(b->nq), first(b->nq);
  int64_t total = 0;
  const int blocks = num_sms() * 8;
  // position t of a row is split into chunks only when the depth-first walk
  // takes it (t <= n - 2; a row of depth n - 1 is closed at once)
  auto splits = [&](int k) { return span > 0 && b->depth[k] <= b->plans[k].n - 2; };
  for (int k = 0; k < b->nq; ++k) {
    const int64_t np = b->nrows[k];
    if (b->plans[k].n < 3 || np == 0) continue;
    GPM_TRY(cnt[k].reserve(np));
    GPM_TRY(first[k].reserve(np + 1));
    k_row_tasks<<<blocks, 256>>>(b->plans[k], b->rows[k], np, b->depth[k], g->off.p, lc->loff.p, lc->L,
                                 splits(k) ? span : 0, cnt[k].p);
    GPM_LAUNCH_CHECK();
    size_t tmp = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tmp, cnt[k].p, first[k].p + 1, (int)np);
    DevBuf<char> t;
    GPM_TRY(t.reserve(tmp));
    GPM_CUDA(cudaMemset(first[k].p, 0, sizeof(int64_t)));
    cub::DeviceScan::InclusiveSum(t.p, tmp, cnt[k].p, first[k].p + 1, (int)np);
    int64_t c = 0;
    GPM_CUDA(cudaMemcpy(&c, first[k].p + np, sizeof(int64_t), cudaMemcpyDeviceToHost));
    cnt_total[k] = c;
    total += c;
  }
  GPM_TRY(b->tasks.reserve(std::max<int64_t>(total, 1)));
  int64_t at = 0;
  for (int k = 0; k < b->nq; ++k) {
    if (!cnt_total[k]) continue;
    // each query's tasks at its own offset: shift the scan by `at`
    k_expand_tasks<<<blocks, 256>>>(b->nrows[k], first[k].p, cnt[k].p, k, splits(k), b->tasks.p + at);
    GPM_LAUNCH_CHECK();
    at += cnt_total[k];
  }
  GPM_CUDA(cudaDeviceSynchronize());
  b->ntasks = total;
  b->span = span;
  drop_batch_graph(b);
  return GPM_OK;
}

template <int Q>
static int batch_grid() {
  static PerDevice grid;
  return grid.get([] {
    constexpr int smem = match_dyn_smem<Q>();
    if (smem > 0) cudaFuncSetAttribute(k_match_batch<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match_batch<Q>, kMatchWarps * 32, smem);
    return std::max(1, per_sm) * num_sms();
  });
}

static int batch_launch(gpm_match_batch *b, cudaStream_t st) {
  gpm_graph *g = b->g;
  LabelCsr *lc = g->lcsr;
  const size_t bytes = sizeof(unsigned long long) * b->nq * b->nm;
  GPM_CUDA(cudaMemcpyAsync(b->out.p, b->base.p, bytes, cudaMemcpyDeviceToDevice, st));
  GPM_CUDA(cudaMemsetAsync(b->cursor.p, 0, 8, st));
  if (b->ntasks == 0) return GPM_OK;
  const MatchGraph G{g->off.p, g->adj.p, lc->ladj.p, lc->loff.p, g->labels.p, lc->L,
                     HubIndex{lc->hub_slot.p, lc->hub_bm.p, lc->hub_words}};
  const int32_t *member = b->nm > 1 ? b->member.p : nullptr;
  if (b->qcap <= kNarrowQ)
    k_match_batch<kNarrowQ><<<b->grid, kMatchWarps * 32, 0, st>>>(
        reinterpret_cast<const QueryPlan *>(b->dplans.p), b->drows.p, G, b->tasks.p, b->ntasks, b->span, member,
        b->nm, b->cursor.p, b->out.p);
  else
    k_match_batch<kMaxQ><<<b->grid, kMatchWarps * 32, match_dyn_smem<kMaxQ>(), st>>>(
        reinterpret_cast<const WidePlan *>(b->dplans.p), b->drows.p, G, b->tasks.p, b->ntasks, b->span, member,
        b->nm, b->cursor.p, b->out.p);
  GPM_LAUNCH_CHECK();
  return GPM_OK;
}

static int batch_run(gpm_match_batch *b, int use_graph, cudaStream_t st) {
  if (!use_graph) return batch_launch(b, st);
  if (!b->exec) {
    // capture on a private stream so the caller's stream may be the legacy one
    cudaStream_t cs;
    GPM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int s = e == cudaSuccess ? batch_launch(b, cs) : fail(GPM_ECUDA, cudaGetErrorString(e));
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (s != GPM_OK) {
      if (graph) cudaGraphDestroy(graph);
      return s;
    }
    if (e != cudaSuccess) return fail(GPM_ECUDA, std::string("match batch capture: ") + cudaGetErrorString(e));
    b->graph = graph;
    GPM_CUDA(cudaGraphInstantiate(&b->exec, graph, 0));
  }
  GPM_CUDA(cudaGraphLaunch(b->exec, st));
  return GPM_OK;
}

}  // namespace gpm

extern "C" {

int gpm_match_batch_create(gpm_graph *g, int nq, const gpm_query *const *queries, const int32_t *member,
                           int nmembers, gpm_match_batch **out) {
  if (!g || !out || nq < 1 || !queries || (member && nmembers < 1))
    return fail(GPM_EINVAL, "gpm_match_batch_create: bad argument");
  if (!g->labels.p) return fail(GPM_EINVAL, "the data graph carries no labels");
  if (g->oriented) return fail(GPM_EINVAL, "matching needs the symmetric (unoriented) data graph");
  for (int k = 0; k < nq; ++k)
    if (!queries[k]) return fail(GPM_EINVAL, "gpm_match_batch_create: NULL query");
  auto *b = new gpm_match_batch();
  b->g = g;
  b->nq = nq;
  b->nm = member ? nmembers : 1;
  auto bail = [&](int s) {
    delete b;
    return s;
  };
  int s;
  if (member) {
    for (int64_t v = 0; v < g->n; ++v)
      if (member[v] < 0 || member[v] >= nmembers) return bail(fail(GPM_EINVAL, "member id out of range"));
    if ((s = b->member.reserve(std::max<int64_t>(g->n, 1)))) return bail(s);
    if (g->n && cudaMemcpy(b->member.p, member, sizeof(int32_t) * g->n, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(GPM_ECUDA, "member upload"));
  }
  int maxl = 1;
  for (int k = 0; k < nq; ++k)
    for (int i = 0; i < queries[k]->n; ++i) maxl = std::max(maxl, queries[k]->labels[i] + 1);
  std::vector<int64_t> freq;
  if ((s = label_freq(g, maxl, freq))) return bail(s);
  if ((s = ensure_label_csr(g))) return bail(s);
  LabelCsr *lc = g->lcsr;
  const size_t cells = (size_t)nq * b->nm;
  for (int k = 0; k < nq; ++k)
    if (queries[k]->n > kNarrowQ) b->qcap = kMaxQ;
  const size_t plan_bytes = b->qcap <= kNarrowQ ? sizeof(QueryPlan) : sizeof(WidePlan);
  if ((s = b->base.reserve(cells)) || (s = b->out.reserve(cells)) || (s = b->cursor.reserve(1)) ||
      (s = b->dplans.reserve(plan_bytes * nq)))
    return bail(s);
  GPM_CUDA(cudaMemset(b->base.p, 0, sizeof(unsigned long long) * cells));
  b->plans.resize(nq);
  b->pairs.resize(nq);
  b->npairs.assign(nq, 0);
  b->ext.resize(nq);
  b->rows.assign(nq, nullptr);
  b->nrows.assign(nq, 0);
  b->depth.assign(nq, 2);
  const MatchGraph G{g->off.p, g->adj.p, lc->ladj.p, lc->loff.p, g->labels.p, lc->L,
                     HubIndex{lc->hub_slot.p, lc->hub_bm.p, lc->hub_words}};
  DevBuf<unsigned long long> np;
  if ((s = np.reserve(1))) return bail(s);
  const int blocks = (int)std::min<int64_t>((g->n * 32 + 255) / 256, (int64_t)num_sms() * 16);
  const int sblocks = (int)std::min<int64_t>((g->n + 255) / 256 + 1, (int64_t)num_sms() * 8);
  for (int k = 0; k < nq; ++k) {
    WidePlan &p = b->plans[k];
    if ((s = plan_query(queries[k], freq, &p))) return bail(s);
    if (p.n == 1) {
      if (g->n) k_small_counts<<<sblocks, 256>>>(g->n, g->labels.p, p.label[0], nullptr, 0,
                                                  b->nm > 1 ? b->member.p : nullptr, b->base.p + (size_t)k * b->nm);
      continue;
    }
    GPM_CUDA(cudaMemset(np.p, 0, 8));
    k_match_pairs<<<blocks, 256>>>(p, g->n, g->off.p, lc->ladj.p, lc->loff.p, lc->L, g->labels.p, 1, nullptr, np.p);
    unsigned long long h = 0;
    GPM_CUDA(cudaMemcpy(&h, np.p, 8, cudaMemcpyDeviceToHost));
    b->npairs[k] = (int64_t)h;
    if (h == 0) continue;
    if ((s = b->pairs[k].reserve(h))) return bail(s);
    GPM_CUDA(cudaMemset(np.p, 0, 8));
    k_match_pairs<<<blocks, 256>>>(p, g->n, g->off.p, lc->ladj.p, lc->loff.p, lc->L, g->labels.p, 0, b->pairs[k].p,
                                   np.p);
    if (p.n == 2) {
      k_small_counts<<<sblocks, 256>>>(0, nullptr, 0, b->pairs[k].p, (int64_t)h, b->nm > 1 ? b->member.p : nullptr,
                                       b->base.p + (size_t)k * b->nm);
      continue;
    }
    // the pairs are rows of two ids; too few of them are extended first
    b->rows[k] = reinterpret_cast<const int32_t *>(b->pairs[k].p);
    b->nrows[k] = (int64_t)h;
    if ((s = extend_rows(p, G, &b->ext[k], &b->rows[k], &b->nrows[k], &b->depth[k], row_target()))) return bail(s);
  }
  {
    std::vector<int4> qr(nq);
    for (int k = 0; k < nq; ++k) {
      const unsigned long long a = (unsigned long long)(uintptr_t)b->rows[k];
      qr[k] = make_int4((int)(uint32_t)a, (int)(uint32_t)(a >> 32), b->depth[k], 0);
    }
    if ((s = b->drows.reserve(nq))) return bail(s);
    GPM_CUDA(cudaMemcpy(b->drows.p, qr.data(), sizeof(int4) * nq, cudaMemcpyHostToDevice));
  }
  if (b->qcap <= kNarrowQ) {
    std::vector<QueryPlan> narrow(nq);
    for (int k = 0; k < nq; ++k) narrow_plan(b->plans[k], &narrow[k]);
    GPM_CUDA(cudaMemcpy(b->dplans.p, narrow.data(), plan_bytes * nq, cudaMemcpyHostToDevice));
    b->grid = batch_grid<kNarrowQ>();
  } else {
    GPM_CUDA(cudaMemcpy(b->dplans.p, b->plans.data(), plan_bytes * nq, cudaMemcpyHostToDevice));
    b->grid = batch_grid<kMaxQ>();
  }
  if ((s = batch_tasks(b, 0))) return bail(s);
  *out = b;
  return GPM_OK;
}

int gpm_match_batch_autotune(gpm_match_batch *b, int64_t *span) {
  if (!b) return fail(GPM_EINVAL, "NULL batch");
  static const int64_t cand[] = {0, 16384, 2048, 256};
  cudaEvent_t e0, e1;
  GPM_CUDA(cudaEventCreate(&e0));
  GPM_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int64_t best_span = b->span;
  for (int64_t c : cand) {
    GPM_TRY(batch_tasks(b, c));
    GPM_TRY(batch_launch(b, 0));  // warm-up
    GPM_CUDA(cudaEventRecord(e0, 0));
    GPM_TRY(batch_launch(b, 0));
    GPM_CUDA(cudaEventRecord(e1, 0));
    GPM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    GPM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_span = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  GPM_TRY(batch_tasks(b, best_span));
  if (span) *span = best_span;
  return GPM_OK;
}

int gpm_match_batch_run_async(gpm_match_batch *b, int use_graph, void *stream, uint64_t *d_out) {
  if (!b || !d_out) return fail(GPM_EINVAL, "gpm_match_batch_run_async: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  GPM_TRY(batch_run(b, use_graph, st));
  GPM_CUDA(cudaMemcpyAsync(d_out, b->out.p, sizeof(unsigned long long) * b->nq * b->nm, cudaMemcpyDeviceToDevice, st));
  return GPM_OK;
}

int gpm_match_batch_run(gpm_match_batch *b, int use_graph, void *stream, uint64_t *out) {
  if (!b || !out) return fail(GPM_EINVAL, "gpm_match_batch_run: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  GPM_TRY(batch_run(b, use_graph, st));
  GPM_CUDA(cudaMemcpyAsync(out, b->out.p, sizeof(unsigned long long) * b->nq * b->nm, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

int gpm_match_batch_info(const gpm_match_batch *b, int64_t *tasks, int64_t *span) {
  if (!b) return fail(GPM_EINVAL, "NULL batch");
  if (tasks) *tasks = b->ntasks;
  if (span) *span = b->span;
  return GPM_OK;
}

int gpm_match_batch_destroy(gpm_match_batch *b) {
  delete b;
  return GPM_OK;
}

}  // extern "C"
