// tc_rank.cu -- the B200 triangle-count path (variant GPM_TC_BITMAP).
//
// Same sum as every TCSolver variant, T = sum over stored u->v of
// |N(u) & N(v)|, reorganised five ways:
//
// 1. Rank relabel.  Vertices are renumbered by (in+out degree, id), the
//    order the degree orientation (graph.h:128-129) is built on, so a DAG
//    edge always points to a larger id and the out-list of a high-degree
//    vertex is a short run of large ids.
// 2. Smaller side probes.  Each stored edge is owned by the endpoint with
//    the longer list ("owner"); the other endpoint is its "partner".  An
//    owner task loads N(owner) once and streams the lists N(partner) of all
//    its partners.  The streamed work is sum over edges of
//    min(d(u), d(v)) instead of sum d(v) (2.3x less on R-MAT).
// 3. Clipped segments.  Only the part of N(partner) inside
//    [min N(owner), max N(owner)] can meet N(owner); the plan stores that
//    range of radj per edge (two binary searches at plan time), which drops
//    another 30 % of the streamed keys on R-MAT and every range check.
// 4. Direct-mapped membership.  After the relabel nearly every large owner
//    list spans few ids, so membership is one shared-memory byte load (span
//    within the byte map) or bit test (within the bitmap): no hashing, no
//    probe loops, no divergence.  Wider owners use an open-addressing table.
// 5. Dense core.  The top 16,384 ranks are dense among themselves: an owner
//    there meets partners whose clipped lists hold many keys per 32 ids of
//    its span.  Such a partner's core keys are kept as a bitmap row, and the
//    segment is counted as popc(row & N(owner)) over the owner's span by
//    k_tc_dense (one 32-bit word per 32 ids instead of one key per id) on a
//    side stream beside the count kernel (R-MAT 22: 4.2 G of the 8.15 G
//    streamed keys become 1.7 G words).
//
// Long segments (48 keys or more in the fixed schedule) are streamed by
// half-warps, one coalesced 256-byte row of 64 keys per step; short ones by
// 4-lane groups.  Owners with more than `cta_min` keys are CTA tasks, the
// rest warp tasks; both queues are sorted heaviest first and drained by a
// persistent grid.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "tc.cuh"
#include "tc_rank.cuh"

namespace gpm {

namespace cg = cooperative_groups;

constexpr int kRWarps = 8;
constexpr int kCtaWords = kRankCtaWords;
constexpr int kWarpWords = kCtaWords / kRWarps;
static_assert(kWarpWords >= 64 && kWarpWords * kRWarps == kCtaWords, "warp regions tile the CTA region");
constexpr size_t kRankSmem = kCtaWords * 4;

static int grid_for(int64_t work, int block = 256) {
  int64_t g = (work + block - 1) / block;
  int64_t cap = (int64_t)num_sms() * 16;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}

// ------------------------------------------------------------ membership
// Keys handed to a table come from aligned 16-byte rows of the padded lists
// (radj4): the clipped segment's own keys lie in [min N(owner), max
// N(owner)], and the other keys of its first and last rows lie below that
// range (earlier keys of the sorted partner list) or above it (later keys,
// the INT32_MAX padding).  The byte map and bitmap clamp the key's offset to
// the span, where a guard entry is zero; the hash table finds no such key.
struct ByteTable {
  const uint8_t *bm;  // span + 1 bytes, bm[span] = 0
  int32_t base;
  uint32_t span;
  __device__ __forceinline__ unsigned hit(int32_t w) const { return bm[min((uint32_t)(w - base), span)]; }
};
struct BitTable {
  const uint32_t *bm;  // span + 1 bits, bit span = 0
  int32_t base;
  uint32_t span;
  __device__ __forceinline__ unsigned hit(int32_t w) const {
    const uint32_t o = min((uint32_t)(w - base), span);
    return (bm[o >> 5] >> (o & 31)) & 1u;
  }
};
struct HashTable {
  const int32_t *tab;
  int logcap;
  __device__ __forceinline__ unsigned hit(int32_t w) const {
    uint32_t mask = (1u << logcap) - 1u;
    uint32_t h = ((uint32_t)w * 2654435769u) >> (32 - logcap);
    while (true) {
      int32_t k = tab[h];
      if (k == w) return 1u;
      if (k < 0) return 0u;
      h = (h + 1) & mask;
    }
  }
};

#ifndef GPM_RANK_SHORT_LANES
#define GPM_RANK_SHORT_LANES 4  // lanes per short segment (2, 4, 8 or 16)
#endif
#ifndef GPM_RANK_BYTEMAP
#define GPM_RANK_BYTEMAP 1  // 0: owners whose span fits a byte map use the bitmap
#endif
#ifndef GPM_RANK_UNROLL
#define GPM_RANK_UNROLL 1
#endif
constexpr int kRankUnroll = GPM_RANK_UNROLL;  // 16-byte rows in flight per lane
template <class T>
__device__ __forceinline__ unsigned hit4(const T &t, int4 v) {
  return t.hit(v.x) + t.hit(v.y) + t.hit(v.z) + t.hit(v.w);
}

// Segments of one owner, read as aligned 16-byte rows of radj4 (four keys
// per lane and load; the rows' keys outside the segment miss, see above):
// the long ones [l0, l1): each half-warp streams one, 64 keys per step (one
// 256-byte row), so the per-segment work of a warp is shared by two
// segments; the short ones [s0, s1): groups of GPM_RANK_SHORT_LANES lanes,
// eight segments per warp at 4 lanes.
// `wid`/`nw` spread segments over the warps of the executing group (1 warp
// for warp tasks, the CTA's warps for CTA tasks).
// Dense long segments ({-1 - i, keys}, owners in the dense core) are counted
// by k_tc_dense and skipped here.
template <class T>
__device__ __forceinline__ unsigned long long scan_segments(const int32_t *__restrict__ radj4,
                                                            const Seg *__restrict__ pseg, int64_t l0,
                                                            int64_t l1, int64_t s0, int64_t s1, const T &t,
                                                            int wid, int nw, unsigned lane) {
  const int4 *__restrict__ rows = reinterpret_cast<const int4 *>(radj4);
  unsigned long long c = 0;
  int64_t j;
  const unsigned half = lane >> 4, hl = lane & 15;
  for (j = l0 + wid * 2 + half; j < l1; j += nw * 2) {
    const Seg sg = pseg[j];
    const int4 *__restrict__ q = rows + max(sg.x, 0);
    const int nr = sg.x < 0 ? 0 : seg_rows(sg);  // dense: none
    unsigned cs = 0;
#pragma unroll kRankUnroll
    for (int i = (int)hl; i < nr; i += 16) cs += hit4(t, __ldg(q + i));
    c += cs;
  }
  constexpr int S = GPM_RANK_SHORT_LANES, G = 32 / S;
  const unsigned grp = lane / S, gl = lane % S;
  for (j = s0 + wid * G + grp; j < s1; j += nw * G) {
    const Seg sg = pseg[j];
    unsigned cs = 0;
    const int64_t k1 = (int64_t)sg.x + seg_rows(sg);
    for (int64_t k = (int64_t)sg.x + gl; k < k1; k += S) cs += hit4(t, __ldg(rows + k));
    c += cs;
  }
  return c;
}

// ------------------------------------------------------------ tasks
template <bool CTA>
__device__ __forceinline__ void group_sync() {
  if (CTA)
    __syncthreads();
  else
    __syncwarp();
}

// One owner task: the membership structure of N(x) in `words` (nwords
// 32-bit words of shared memory), built by the group's threads (the CTA, or
// one warp), then the owner's segments streamed against it.  By the span S of
// N(x): S <= 4 * nwords -> byte map; S <= 32 * nwords -> bitmap; else
// open-addressing tables of the largest power-of-two size that fits, built
// over chunks of at most half that many keys.  REC: each warp adds the
// cycles it was busy on the task (to just before the closing barrier) to
// *rec, so a task's logged cost is its active warp-cycles.
template <bool CTA, bool REC>
__device__ __forceinline__ unsigned long long owner_task(int32_t x, const int64_t *__restrict__ roff,
                                                         const int32_t *__restrict__ radj,
                                                         const int32_t *__restrict__ radj4,
                                                         const int64_t *__restrict__ poff,
                                                         const Seg *__restrict__ pseg,
                                                         const int32_t *__restrict__ plong,
                                                         const int32_t *__restrict__ pshort, uint32_t *words,
                                                         int nwords, unsigned long long *rec) {
  const long long t0 = REC ? clock64() : 0;
  const int tid = CTA ? (int)threadIdx.x : (int)lane_id(), nthr = CTA ? (int)blockDim.x : 32;
  const int wid = CTA ? tid >> 5 : 0, nw = CTA ? nthr >> 5 : 1;
  const unsigned lane = lane_id();
  const int64_t s0 = roff[x];
  const int d = (int)(roff[x + 1] - s0);
  const int64_t l0 = poff[x], l1 = l0 + plong[x], h1 = poff[x + 1], h0 = h1 - pshort[x];
  const int32_t kmin = radj[s0], kmax = radj[s0 + d - 1];
  const int64_t span = (int64_t)kmax - kmin + 1;
  unsigned long long c = 0;
  if (GPM_RANK_BYTEMAP && span < (int64_t)nwords * 4) {
    // byte map / bitmap: span + 1 entries, the last the zero guard
    const int nclear = (int)((span + 4) >> 2);
    for (int i = tid; i < nclear; i += nthr) words[i] = 0u;
    group_sync<CTA>();
    uint8_t *bytes = reinterpret_cast<uint8_t *>(words);
    for (int i = tid; i < d; i += nthr) bytes[radj[s0 + i] - kmin] = 1;
    group_sync<CTA>();
    c = scan_segments(radj4, pseg, l0, l1, h0, h1, ByteTable{bytes, kmin, (uint32_t)span}, wid, nw, lane);
  } else if (span < (int64_t)nwords * 32) {
    const int nclear = (int)((span + 32) >> 5);
    for (int i = tid; i < nclear; i += nthr) words[i] = 0u;
    group_sync<CTA>();
    for (int i = tid; i < d; i += nthr) {
      uint32_t o = (uint32_t)(radj[s0 + i] - kmin);
      atomicOr(&words[o >> 5], 1u << (o & 31));
    }
    group_sync<CTA>();
    c = scan_segments(radj4, pseg, l0, l1, h0, h1, BitTable{words, kmin, (uint32_t)span}, wid, nw, lane);
  } else {
    int32_t *tab = reinterpret_cast<int32_t *>(words);
    const int logcap = 31 - __clz(nwords);
    const int chunk = 1 << (logcap - 1);
    const uint32_t mask = (1u << logcap) - 1u;
    for (int t0 = 0; t0 < d; t0 += chunk) {
      const int tk = min(chunk, d - t0);
      group_sync<CTA>();
      for (int i = tid; i < (1 << logcap); i += nthr) tab[i] = -1;
      group_sync<CTA>();
      for (int i = tid; i < tk; i += nthr) {
        int32_t key = radj[s0 + t0 + i];
        uint32_t h = ((uint32_t)key * 2654435769u) >> (32 - logcap);
        while (atomicCAS(&tab[h], -1, key) != -1) h = (h + 1) & mask;
      }
      group_sync<CTA>();
      c += scan_segments(radj4, pseg, l0, l1, h0, h1, HashTable{tab, logcap}, wid, nw, lane);
    }
  }
  if (REC && lane == 0) atomicAdd(rec, (unsigned long long)(clock64() - t0));
  group_sync<CTA>();
  return c;
}

#ifndef GPM_TC_RANK_MIN_BLOCKS
// CTAs per SM the register budget is sized for: 8 (32 registers) measured
// 23.5 ms on R-MAT 22 against 25.5 ms at 6 and 29.3 ms at 4 (59 registers)
#define GPM_TC_RANK_MIN_BLOCKS 8
#endif
// REC = true is the instrumented build the learned scheduler trains on: it
// adds each task's active warp-cycles (per warp, the SM clock cycles it spent
// on the task outside the closing barrier) into rec[owner], which the caller
// zeroes first.
template <bool REC>
__global__ void __launch_bounds__(256, GPM_TC_RANK_MIN_BLOCKS)
    k_tc_rank_t(const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                const int32_t *__restrict__ radj4, const int64_t *__restrict__ poff,
                const Seg *__restrict__ pseg,
                const int32_t *__restrict__ plong, const int32_t *__restrict__ pshort,
                const int32_t *__restrict__ cta_tasks, int n_cta,
                const int32_t *__restrict__ warp_tasks, int n_warp, int *__restrict__ counters,
                unsigned long long *__restrict__ out, unsigned long long *__restrict__ rec) {
  extern __shared__ __align__(16) uint32_t rsm[];
  __shared__ int s_task;
  unsigned long long c = 0;
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(&counters[0], 1);
    __syncthreads();
    int t = s_task;
    __syncthreads();
    if (t >= n_cta) break;
    const int32_t x = cta_tasks[t];
    c += owner_task<true, REC>(x, roff, radj, radj4, poff, pseg, plong, pshort, rsm, kCtaWords,
                               REC ? rec + x : nullptr);
  }
  const int wid = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31;
  uint32_t *region = rsm + wid * kWarpWords;
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&counters[1], 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_warp) break;
    const int32_t x = warp_tasks[t];
    c += owner_task<false, REC>(x, roff, radj, radj4, poff, pseg, plong, pshort, region, kWarpWords,
                                REC ? rec + x : nullptr);
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(out, c);
}
#define k_tc_rank k_tc_rank_t<false>

// Dense segments of the core owners, one owner per CTA task (heaviest
// first): N(x) as a bitmap from base = min N(x) rounded down to 128 in shared
// memory (core_clear_words, at most row_words + 4), then every dense
// segment {-1 - i, keys} of x (dseg[doff[x] .. doff[x+1])) by a group of kDenseLanes lanes: the partner's
// core row words from base on (rows4[i] ..), ANDed 16 bytes per lane with the
// bitmap over core_and_words(x) / 4 loads.  Its own launch, so that its
// register budget (64 at 4 CTAs of 256 per SM) allows several 16-byte loads
// in flight per lane; the owners' other segments run in k_tc_rank.
#ifndef GPM_RANK_DENSE_LANES
// lanes per dense segment: 8 (R-MAT 22 5.88 ms at unroll 2) against 4 (5.79)
// and 16 (6.27); 8 kept with unroll 1 (5.50 against 5.69 at 4 lanes)
#define GPM_RANK_DENSE_LANES 8
#endif
constexpr int kDenseLanes = GPM_RANK_DENSE_LANES;
#ifndef GPM_RANK_DENSE_UNROLL
// 16-byte loads unrolled per lane: 1 (28 registers) ran R-MAT 22 in 5.78 ms
// against 5.88 at 2 (40 registers) and 6.16 at 4 (56 registers): the kernel
// shares the SMs with the count kernel, and fewer registers leave it more room
#define GPM_RANK_DENSE_UNROLL 1
#endif
constexpr int kDenseUnroll = GPM_RANK_DENSE_UNROLL;
__global__ void __launch_bounds__(256, 4)
    k_tc_dense(const int64_t *__restrict__ roff, const int32_t *__restrict__ radj, const int64_t *__restrict__ doff,
               const Seg *__restrict__ dseg, const int32_t *__restrict__ tasks, int ntasks,
               const uint4 *__restrict__ rows4, int *__restrict__ counter, unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t dsm[];
  __shared__ int s_task;
  const int grp = threadIdx.x / kDenseLanes, gl = threadIdx.x % kDenseLanes, ngrp = blockDim.x / kDenseLanes;
  const uint4 *b = reinterpret_cast<const uint4 *>(dsm);
  unsigned long long c = 0;
  while (true) {
    if (threadIdx.x == 0) s_task = atomicAdd(counter, 1);
    __syncthreads();
    const int t = s_task;
    __syncthreads();
    if (t >= ntasks) break;
    const int32_t x = tasks[t];
    const int64_t s0 = roff[x], s1 = roff[x + 1];
    const int32_t kmin = radj[s0], kmax = radj[s1 - 1], base = kmin & ~127;
    const int nclear = core_clear_words(kmin, kmax), nq = core_and_words(kmin, kmax) >> 2;
    for (int i = threadIdx.x; i < nclear; i += blockDim.x) dsm[i] = 0u;
    __syncthreads();
    for (int64_t k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
      const uint32_t o = (uint32_t)(radj[k] - base);
      atomicOr(&dsm[o >> 5], 1u << (o & 31));
    }
    __syncthreads();
    const int64_t d1 = doff[x + 1];
    for (int64_t j = doff[x] + grp; j < d1; j += ngrp) {
      const uint4 *__restrict__ r = rows4 + (-1 - dseg[j].x);
      unsigned cs = 0;
#pragma unroll kDenseUnroll
      for (int i = gl; i < nq; i += kDenseLanes) {
        const uint4 a = __ldg(r + i), m = b[i];
        cs += __popc(a.x & m.x) + __popc(a.y & m.y) + __popc(a.z & m.z) + __popc(a.w & m.w);
      }
      c += cs;
    }
    __syncthreads();
  }
  c = warp_sum(c);
  if (lane_id() == 0 && c) atomicAdd(out, c);
}

// ------------------------------------------------------------ plan build
__global__ void k_indeg(int64_t nnz, const int32_t *__restrict__ adj, int32_t *__restrict__ indeg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&indeg[adj[i]], 1);
}
// sort key: (graph id, in + out degree); the stable sort breaks ties by id.
// indeg == nullptr: the stored graph is symmetric, out-degree orders alike
__global__ void k_rank_keys(int64_t n, const int64_t *__restrict__ off, const int32_t *__restrict__ indeg,
                            const int32_t *__restrict__ gid, uint64_t *__restrict__ key, int32_t *__restrict__ val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t d = (uint64_t)(uint32_t)((off[i + 1] - off[i]) + (indeg ? indeg[i] : 0));
    key[i] = gid ? ((uint64_t)(uint32_t)gid[i] << 32) | d : d;
    val[i] = (int32_t)i;
  }
}
__global__ void k_rank_inverse(int64_t n, const int32_t *__restrict__ order, const int64_t *__restrict__ off,
                               int32_t *__restrict__ rank, int64_t *__restrict__ rdeg) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = order[r];
    rank[v] = (int32_t)r;
    rdeg[r] = off[v + 1] - off[v];
  }
}
// Relabelled lists, gathered and sorted in one pass (one warp per rank r):
// the neighbours of order[r] as ranks are collected in the warp's shared
// buffer, sorted there -- a register bitonic network up to 32 keys, a
// shared-memory one up to kSortCap -- and written to out[roff[r] ..].
// Longer lists are written unsorted and their rank appended to big[] for a
// segmented sort afterwards.
constexpr int kSortCap = 1024;
constexpr int kGatherWarps = 8;

__device__ __forceinline__ int32_t warp_bitonic32(int32_t key, unsigned lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int32_t other = __shfl_xor_sync(0xffffffffu, key, j);
      const bool asc = (lane & k) == 0, low = (lane & j) == 0;
      key = (low == asc) ? min(key, other) : max(key, other);
    }
  return key;
}

__global__ void __launch_bounds__(kGatherWarps * 32)
    k_rank_gather_sort(int64_t n, const int32_t *__restrict__ order, const int32_t *__restrict__ rank,
                       const int64_t *__restrict__ off, const int32_t *__restrict__ adj,
                       const int64_t *__restrict__ roff, int32_t *__restrict__ out, int32_t *__restrict__ big,
                       int *__restrict__ nbig) {
  __shared__ int32_t sbuf[kGatherWarps][kSortCap];
  int32_t *buf = sbuf[threadIdx.x >> 5];
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < n; r += nw) {
    const int32_t v = order[r];
    const int64_t s = off[v], e = off[v + 1], o = roff[r];
    const int64_t len = roff[r + 1] - o;
    if (len == 0) continue;
    const bool fits = len <= kSortCap;
    int32_t *dst = fits ? buf : out + o;
    int64_t filled = 0;
    for (int64_t base = s; base < e && filled < len; base += 32) {
      const int64_t k = base + lane;
      const int32_t x = k < e ? rank[adj[k]] : -1;
      const bool keep = k < e;
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) dst[filled + __popc(m & ((1u << lane) - 1u))] = x;
      filled += __popc(m);
    }
    __syncwarp();
    if (!fits) {
      if (lane == 0) big[atomicAdd(nbig, 1)] = (int32_t)r;
      continue;
    }
    if (len <= 32) {
      const int32_t key = warp_bitonic32((int64_t)lane < len ? buf[lane] : INT_MAX, lane);
      if ((int64_t)lane < len) out[o + lane] = key;
    } else {
      int p = 64;
      while (p < len) p <<= 1;
      for (int i = (int)len + lane; i < p; i += 32) buf[i] = INT_MAX;
      __syncwarp();
      for (int k = 2; k <= p; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = lane; i < p; i += 32) {
            const int ixj = i ^ j;
            if (ixj > i) {
              const int32_t a = buf[i], b = buf[ixj];
              if ((a > b) == ((i & k) == 0)) {
                buf[i] = b;
                buf[ixj] = a;
              }
            }
          }
          __syncwarp();
        }
      for (int64_t i = lane; i < len; i += 32) out[o + i] = buf[i];
    }
    __syncwarp();
  }
}

// incident edges of rank r: its out-degree plus the in-degree of order[r]
__global__ void k_incident(int64_t n, const int32_t *__restrict__ order, const int64_t *__restrict__ rdeg,
                           const int32_t *__restrict__ indeg, int64_t *__restrict__ inc) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    inc[r] = rdeg[r] + indeg[order[r]];
}

__global__ void k_big_bounds(int nbig, const int32_t *__restrict__ big, const int64_t *__restrict__ roff,
                             int64_t *__restrict__ bb, int64_t *__restrict__ be) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x) {
    bb[i] = roff[big[i]];
    be[i] = roff[big[i] + 1];
  }
}
__global__ void k_big_copy(int nbig, const int64_t *__restrict__ bb, const int64_t *__restrict__ be,
                           const int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  for (int i = blockIdx.x; i < nbig; i += gridDim.x)
    for (int64_t k = bb[i] + threadIdx.x; k < be[i]; k += blockDim.x) dst[k] = src[k];
}

// Per-owner task configuration (learned scheduler): queue = cfg / 3
// (0 warp, 1 CTA), long-segment threshold = kCfgLong[cfg % 3].
__device__ __constant__ int kCfgLong[3] = {16, 64, 256};
__device__ __forceinline__ int owner_long_min(const uint8_t *cfg, int32_t owner, int long_min) {
  return cfg ? kCfgLong[cfg[owner] % 3] : long_min;
}

__device__ __forceinline__ int64_t lower_bound_key(const int32_t *__restrict__ a, int64_t lo, int64_t hi,
                                                   int32_t key) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}
__device__ __forceinline__ int64_t upper_bound_key(const int32_t *__restrict__ a, int64_t lo, int64_t hi,
                                                   int32_t key) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Every stored edge k = (u, radj[k]) placed in one pass: the endpoint with
// the longer list owns it (ties to u), the other is its partner; the segment
// is the part of the partner's list inside [min, max] of the owner's list
// (empty, hence left out, also when the owner has fewer than 2 keys and so
// closes no triangle through the edge).  It goes into the owner's room
// [poff[x], poff[x+1]) -- one slot per incident edge, so it always fits --
// long segments from the front (cursor plong[x]), short ones from the back
// (cursor pshort[x]), as ranges of radj4.  With radj4 non-null the pass also
// copies each list u into it (with its INT32_MAX padding).  upward: every list holds only ids above its vertex,
// so when u owns the edge, min N(u) <= v < every id of N(v) and the lower
// search is skipped.  The lanes of a warp that share an (owner, class) take
// their slots with one atomic (hub owners get most of theirs from their own
// list, i.e. from one warp).
__global__ void k_partner_place(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                                const int64_t *__restrict__ roff4, int32_t *__restrict__ radj4, int upward,
                                int long_min, const uint8_t *__restrict__ cfg,
                                const int64_t *__restrict__ poff, int32_t *__restrict__ plong,
                                int32_t *__restrict__ pshort, Seg *__restrict__ pseg,
                                unsigned long long *__restrict__ work, int32_t core_base,
                                const int32_t *__restrict__ rowid, int row_words, int dense_pct,
                                int32_t *__restrict__ pdense, int *__restrict__ too_long) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t u = warp; u < n; u += nw) {
    int64_t s = roff[u], e = roff[u + 1], du = e - s;
    if (radj4) {  // u's list into radj4 with its padding, one 16-byte row per lane
      int4 *row = reinterpret_cast<int4 *>(radj4 + roff4[u]);
      for (int64_t r = lane_id(); 4 * r < du; r += 32) {
        const int64_t b = s + 4 * r;
        row[r] = make_int4(radj[b], b + 1 < e ? radj[b + 1] : INT32_MAX, b + 2 < e ? radj[b + 2] : INT32_MAX,
                           b + 3 < e ? radj[b + 3] : INT32_MAX);
      }
    }
    for (int64_t k = s + lane_id(); k < e; k += 32) {
      int32_t v = radj[k];
      int64_t vs = roff[v], ve = roff[v + 1], dv = ve - vs;
      bool own_u = dv <= du;
      int32_t owner = own_u ? (int32_t)u : v;
      int64_t os = own_u ? s : vs, oe = own_u ? e : ve;
      int64_t ps = own_u ? vs : s, pe = own_u ? ve : e;
      if (oe - os < 2) continue;
      // upward: when v owns the edge, every id of N(u) up to v sits at or
      // before slot k, and min N(v) > v, so the search starts past k
      const int64_t lo = upward ? (own_u ? ps : lower_bound_key(radj, k + 1, pe, radj[os]))
                                : lower_bound_key(radj, ps, pe, radj[os]);
      const int64_t len = upper_bound_key(radj, lo, pe, radj[oe - 1]) - lo;
      if (len == 0) continue;
      const int32_t partner = own_u ? v : (int32_t)u;
      // dense: a core owner and a partner with a core row, the keys at least
      // dense_pct % of the owner's words to AND (k_tc_dense counts it; the
      // count kernel only skips its descriptor)
      int64_t row = -1;  // dense: the uint4 index of the partner's row words from the owner's base
      if (rowid && radj[os] >= core_base) {
        const int32_t kmin = radj[os], r = rowid[partner];
        if (r >= 0 && 100 * len >= (int64_t)dense_pct * core_and_words(kmin, radj[oe - 1]))
          row = (int64_t)r * (row_words >> 2) + (((kmin & ~127) - core_base) >> 7);
      }
      const int64_t units = row >= 0 ? 0 : len;
      const bool lng = row >= 0 || len >= owner_long_min(cfg, owner, long_min);
      cg::coalesced_group grp =
          cg::labeled_partition(cg::coalesced_threads(), ((unsigned long long)(uint32_t)owner << 1) | lng);
      int base = 0;
      if (grp.thread_rank() == 0) base = atomicAdd(lng ? &plong[owner] : &pshort[owner], (int)grp.size());
      const int64_t slot = grp.shfl(base, 0) + (int64_t)grp.thread_rank();
      const int64_t pos = lng ? poff[owner] + slot : poff[owner + 1] - 1 - slot;
      const int64_t lo4 = lo - roff[partner] + roff4[partner];  // the same keys in radj4
      if (len >= (1 << 29)) *too_long = 1;  // no 8-byte descriptor for it
      pseg[pos] = row >= 0 ? make_int2((int)(-1 - row), (int)(len << 2))
                           : make_int2((int)(lo4 >> 2), (int)((len << 2) | (lo4 & 3)));
      const unsigned long long w = cg::reduce(grp, (unsigned long long)units + 1ull, cg::plus<unsigned long long>());
      if (grp.thread_rank() == 0) atomicAdd(&work[owner], w);
      if (rowid) {
        const int nd = __popc(grp.ballot(row >= 0));
        if (nd && grp.thread_rank() == 0) atomicAdd(&pdense[owner], nd);
      }
    }
  }
}
// Dense core rows: rowid[v] = a row number when v has at least min_keys
// keys >= core_base, else -1 (*nrows counts the rows)
__global__ void k_core_rowid(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                             int32_t core_base, int min_keys, int32_t *__restrict__ rowid, int *__restrict__ nrows) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = roff[v + 1];
    rowid[v] = e - lower_bound_key(radj, roff[v], e, core_base) >= min_keys ? atomicAdd(nrows, 1) : -1;
  }
}
// row rowid[v] = v's keys >= core_base as bits from core_base (one warp per
// vertex; rows zeroed first)
__global__ void k_core_rows(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                            int32_t core_base, const int32_t *__restrict__ rowid, int row_words,
                            uint32_t *__restrict__ rows) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = warp; v < n; v += nw) {
    const int32_t r = rowid[v];
    if (r < 0) continue;
    uint32_t *row = rows + (int64_t)r * row_words;
    const int64_t e = roff[v + 1];
    for (int64_t k = lower_bound_key(radj, roff[v], e, core_base) + lane_id(); k < e; k += 32) {
      const uint32_t o = (uint32_t)(radj[k] - core_base);
      atomicOr(&row[o >> 5], 1u << (o & 31));
    }
  }
}

// The dense segments of owner x (pdense[x] > 0, one warp each) moved out of
// its long segments into dseg[doff[x] ..); the others closed up at the
// front of the long region and plong[x] set to their number.  A chunk of 32
// is read whole before any lane writes, and a write never passes the chunk.
__global__ void k_split_dense(int64_t n, const int64_t *__restrict__ poff, int32_t *__restrict__ plong,
                              const int32_t *__restrict__ pdense, const int64_t *__restrict__ doff,
                              Seg *__restrict__ pseg, Seg *__restrict__ dseg) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = lane_id(), below = (1u << lane) - 1u;
  for (int64_t x = warp; x < n; x += nw) {
    if (pdense[x] == 0) continue;
    Seg *lg = pseg + poff[x];
    const int nl = plong[x];
    int64_t wd = doff[x];
    int wn = 0;
    for (int b = 0; b < nl; b += 32) {
      const bool valid = b + (int)lane < nl;
      const Seg sg = valid ? lg[b + lane] : make_int2(0, 0);
      const bool dense = valid && sg.x < 0;
      const unsigned md = __ballot_sync(0xffffffffu, dense), mn = __ballot_sync(0xffffffffu, valid && !dense);
      if (dense) dseg[wd + __popc(md & below)] = sg;
      if (valid && !dense) lg[wn + __popc(mn & below)] = sg;
      wd += __popc(md);
      wn += __popc(mn);
      __syncwarp();
    }
    if (lane == 0) plong[x] = wn;
  }
}
__global__ void k_widen(int64_t n, const int32_t *__restrict__ a, int64_t *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

// roff4: list lengths rounded up to a multiple of four, for the scan that
// places every list of radj4 at a multiple of four keys
__global__ void k_padded_len(int64_t n, const int64_t *__restrict__ roff, int64_t *__restrict__ len4) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    len4[v] = (roff[v + 1] - roff[v] + 3) & ~(int64_t)3;
}

// dense tasks: owners with dense segments, key = ~(their words to AND)
__global__ void k_dense_tasks(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                              const int32_t *__restrict__ pdense, unsigned long long *__restrict__ key,
                              int32_t *__restrict__ val, int *__restrict__ size) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    if (pdense[x] == 0) continue;
    const int i = atomicAdd(size, 1);
    key[i] = ~((unsigned long long)pdense[x] * (unsigned long long)core_and_words(radj[roff[x]], radj[roff[x + 1] - 1]));
    val[i] = (int32_t)x;
  }
}

// tasks: owners with partners; key = ~work so an ascending sort puts heavy first
__global__ void k_rank_tasks(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ plong,
                             const int32_t *__restrict__ pshort,
                             const unsigned long long *__restrict__ work, int cta_min,
                             const uint8_t *__restrict__ cfg, const int32_t *__restrict__ pdense,
                             int32_t *__restrict__ donly, unsigned long long *__restrict__ ckey,
                             int32_t *__restrict__ cval, unsigned long long *__restrict__ wkey,
                             int32_t *__restrict__ wval, int *__restrict__ sizes) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    if (plong[x] + pshort[x] == 0) {  // nothing to stream
      if (pdense && pdense[x]) donly[atomicAdd(&sizes[3], 1)] = (int32_t)x;  // dense segments only
      continue;
    }
    int64_t d = roff[x + 1] - roff[x];
    if (cfg ? cfg[x] / 3 == 1 : d > cta_min) {
      int i = atomicAdd(&sizes[0], 1);
      ckey[i] = ~work[x];
      cval[i] = (int32_t)x;
    } else {
      int i = atomicAdd(&sizes[1], 1);
      wkey[i] = ~work[x];
      wval[i] = (int32_t)x;
    }
  }
}

void free_rank_plan(RankPlan *p) { delete p; }

static int sort_pairs_u64(DevBuf<unsigned long long> &k, DevBuf<int32_t> &v, int count, DevBuf<int32_t> &out,
                          cudaStream_t st) {
  if (count <= 0) return GPM_OK;
  DevBuf<unsigned long long> k2;
  GPM_TRY(k2.reserve(count));
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k.p, k2.p, v.p, out.p, count, 0, 64, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, k.p, k2.p, v.p, out.p, count, 0, 64, st));
  return GPM_OK;
}

static int scan_i64(int64_t n, const int64_t *cnt, int64_t *off, cudaStream_t st) {
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, cnt, off + 1, (int)n, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cudaMemsetAsync(off, 0, sizeof(int64_t), st));
  if (n > 0) GPM_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, cnt, off + 1, (int)n, st));
  return GPM_OK;
}

__global__ void k_count_down(int64_t n, const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                             int *__restrict__ down) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
    if (roff[u + 1] > roff[u] && radj[roff[u]] <= (int32_t)u) atomicAdd(down, 1);
}

void free_rank_graph(RankGraph *r) { delete r; }

// Renumber the stored graph by (in + out degree, id) rank; lists re-sorted.
// With a per-vertex graph id (a disjoint union of graphs whose vertices are
// contiguous id ranges) the key is (graph id, degree), so every member graph
// keeps its id range and is ranked within itself.
// Lists of the ranks in big[0..nbig) sorted in place by a segmented sort,
// then r->upward set by checking every list against its rank.
static int finish_rank_graph(RankGraph *r, int64_t n, int64_t nnz, const int32_t *big, int hbig, cudaStream_t st) {
  int s;
  if (hbig > 0) {
    DevBuf<int64_t> bb, be;
    DevBuf<int32_t> sorted;
    if ((s = bb.reserve(hbig)) || (s = be.reserve(hbig)) || (s = sorted.reserve(nnz))) return s;
    k_big_bounds<<<grid_for(hbig), 256, 0, st>>>(hbig, big, r->roff.p, bb.p, be.p);
    size_t tmp = 0;
    GPM_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp, r->radj.p, sorted.p, (int)nnz, hbig, bb.p, be.p, st));
    DevBuf<char> t;
    if ((s = t.reserve(tmp))) return s;
    GPM_CUDA(cub::DeviceSegmentedSort::SortKeys(t.p, tmp, r->radj.p, sorted.p, (int)nnz, hbig, bb.p, be.p, st));
    k_big_copy<<<std::min(hbig, num_sms() * 8), 256, 0, st>>>(hbig, bb.p, be.p, sorted.p, r->radj.p);
  }
  // does every stored edge point to a larger rank? (true for a degree-oriented DAG)
  DevBuf<int> down;
  if ((s = down.reserve(1))) return s;
  cudaMemsetAsync(down.p, 0, sizeof(int), st);
  k_count_down<<<grid_for(n), 256, 0, st>>>(n, r->roff.p, r->radj.p, down.p);
  int hdown = 0;
  cudaMemcpyAsync(&hdown, down.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(GPM_ECUDA, std::string("rank relabel: ") + cudaGetErrorString(e));
  r->upward = hdown == 0;
  return GPM_OK;
}

// Rank keys of the stored graph sorted: order[rank] = vertex, rank[vertex].
// indeg == nullptr: a symmetric graph (out-degree orders like in + out).
static int rank_order(gpm_graph *g, const int32_t *indeg, const int32_t *gid, int ngraphs, int32_t *order,
                      int32_t *rank, int64_t *rdeg, cudaStream_t st) {
  const int64_t n = g->n;
  int s;
  DevBuf<int32_t> val;
  DevBuf<uint64_t> key, key2;
  if ((s = val.reserve(n)) || (s = key.reserve(n)) || (s = key2.reserve(n))) return s;
  int end_bit = 32;
  if (gid)
    while (end_bit < 64 && (1ll << (end_bit - 32)) < ngraphs) ++end_bit;
  k_rank_keys<<<grid_for(n), 256, 0, st>>>(n, g->off.p, indeg, gid, key.p, val.p);
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key2.p, val.p, order, (int)n, 0, end_bit, st));
  DevBuf<char> t;
  if ((s = t.reserve(tmp))) return s;
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, key2.p, val.p, order, (int)n, 0, end_bit, st));
  k_rank_inverse<<<grid_for(n), 256, 0, st>>>(n, order, g->off.p, rank, rdeg);
  return GPM_OK;
}

// dst[0 .. len) sorted in place by one warp (len <= kSortCap): a register
// bitonic network up to 32 ids, else a shared-memory network in buf.
__device__ __forceinline__ void warp_sort_list(int32_t *dst, int64_t len, int32_t *buf, unsigned lane) {
  if (len <= 1) return;
  if (len <= 32) {
    const int32_t key = warp_bitonic32((int64_t)lane < len ? dst[lane] : INT_MAX, lane);
    if ((int64_t)lane < len) dst[lane] = key;
    return;
  }
  int p = 64;
  while (p < len) p <<= 1;
  for (int i = lane; i < p; i += 32) buf[i] = i < len ? dst[i] : INT_MAX;
  __syncwarp();
  for (int k = 2; k <= p; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < p; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int32_t a = buf[i], b = buf[ixj];
          if ((a > b) == ((i & k) == 0)) {
            buf[i] = b;
            buf[ixj] = a;
          }
        }
      }
      __syncwarp();
    }
  for (int64_t i = lane; i < len; i += 32) dst[i] = buf[i];
  __syncwarp();
}

// Upward lists of a symmetric graph, gathered chunk by chunk: for source
// vertex v, the ranks of its neighbours above rank[v], appended (unsorted)
// into tmp at v's own symmetric offset -- room for all of v's neighbours, so
// no count pass is needed first.  A vertex with at most kHubBlock neighbours
// is one warp's task; a longer list is cut into kHubBlock-entry block tasks
// (queued here, run by k_up_gather_hub) so that no warp scans a hub's whole
// list alone.
constexpr int kHubBlock = 1024;
static_assert(kHubBlock <= kSortCap, "a non-hub list must fit the sort buffer");

__device__ __forceinline__ int64_t gather_upward(int32_t r, int64_t s, int64_t e, const int32_t *__restrict__ rank,
                                                 const int32_t *__restrict__ adj, int32_t *dst,
                                                 unsigned long long *cursor, unsigned lane) {
  int64_t len = 0;
  for (int64_t base = s; base < e; base += 32) {
    const int64_t k = base + lane;
    const int32_t x = k < e ? rank[adj[k]] : -1;
    const bool keep = k < e && x > r;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (m == 0) continue;
    int64_t at = len;
    if (cursor) {  // shared with the hub's other block tasks
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(cursor, (unsigned long long)__popc(m));
      at = (int64_t)__shfl_sync(0xffffffffu, b, 0);
    }
    if (keep) dst[at + __popc(m & ((1u << lane) - 1u))] = x;
    len += __popc(m);
  }
  return len;
}

__global__ void __launch_bounds__(kGatherWarps * 32)
    k_up_gather(int64_t v0, int64_t v1, const int32_t *__restrict__ rank, const int64_t *__restrict__ off,
                const int32_t *__restrict__ adj, int32_t *__restrict__ tmp, int64_t *__restrict__ kept,
                unsigned long long *__restrict__ hubcnt, int2 *__restrict__ hubq, int *__restrict__ nhubq) {
  __shared__ int32_t sbuf[kGatherWarps][kSortCap];
  int32_t *buf = sbuf[threadIdx.x >> 5];
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = v0 + warp; v < v1; v += nw) {
    const int64_t s = off[v], e = off[v + 1];
    if (e - s > kHubBlock) {
      const int nb = (int)((e - s + kHubBlock - 1) / kHubBlock);
      if (lane == 0) {
        hubcnt[v] = 0;
        const int at = atomicAdd(nhubq, nb);
        for (int b = 0; b < nb; ++b) hubq[at + b] = make_int2((int)v, b);
      }
      continue;
    }
    const int32_t r = rank[v];
    const int64_t len = gather_upward(r, s, e, rank, adj, tmp + s, nullptr, lane);
    if (lane == 0) kept[r] = len;
    __syncwarp();
    warp_sort_list(tmp + s, len, buf, lane);  // len <= kHubBlock = kSortCap
  }
}

__global__ void k_up_gather_hub(const int2 *__restrict__ hubq, const int *__restrict__ nhubq,
                                const int32_t *__restrict__ rank, const int64_t *__restrict__ off,
                                const int32_t *__restrict__ adj, int32_t *__restrict__ tmp,
                                unsigned long long *__restrict__ hubcnt) {
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int nt = *nhubq;
  for (int64_t t = warp; t < nt; t += nw) {
    const int2 task = hubq[t];
    const int64_t s = off[task.x], e = off[task.x + 1];
    const int64_t b0 = s + (int64_t)task.y * kHubBlock, b1 = min(e, b0 + kHubBlock);
    gather_upward(rank[task.x], b0, b1, rank, adj, tmp + s, &hubcnt[task.x], lane);
  }
}

// kept[rank[v]] of the hubs queued at [q0, nhubq) (one entry per hub: b = 0)
__global__ void k_up_hub_kept(const int2 *__restrict__ hubq, int q0, const int *__restrict__ nhubq,
                              const int32_t *__restrict__ rank, const unsigned long long *__restrict__ hubcnt,
                              int64_t *__restrict__ kept) {
  const int nt = *nhubq;
  for (int64_t t = q0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x)
    if (hubq[t].y == 0) kept[rank[hubq[t].x]] = (int64_t)hubcnt[hubq[t].x];
}

// radj[roff[r] ..] = tmp[off[order[r]] ..], one warp per rank.  Lists of
// small vertices arrive sorted; a hub's list (assembled by block tasks) is
// sorted here, or, beyond kSortCap ids, copied and its rank appended to big[].
__global__ void __launch_bounds__(kGatherWarps * 32)
    k_up_compact(int64_t n, const int32_t *__restrict__ order, const int64_t *__restrict__ off,
                 int32_t *__restrict__ tmp, const int64_t *__restrict__ roff, int32_t *__restrict__ radj,
                 int32_t *__restrict__ big, int *__restrict__ nbig) {
  __shared__ int32_t sbuf[kGatherWarps][kSortCap];
  int32_t *buf = sbuf[threadIdx.x >> 5];
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < n; r += nw) {
    const int32_t v = order[r];
    int32_t *src = tmp + off[v];
    const int64_t o = roff[r], len = roff[r + 1] - o;
    if (off[v + 1] - off[v] > kHubBlock) {
      if (len > kSortCap) {
        if (lane == 0) big[atomicAdd(nbig, 1)] = (int32_t)r;
      } else {
        warp_sort_list(src, len, buf, lane);
      }
    }
    for (int64_t i = lane; i < len; i += 32) radj[o + i] = src[i];
  }
}

int build_upward_rank_graph(gpm_graph *g, cudaStream_t st, const int64_t *h_off, const int32_t *h_adj) {
  if (g->rg) return GPM_OK;
  const int64_t n = g->n, nsym = g->nnz;
  RankGraph *r = new RankGraph();
  cudaStream_t cs = nullptr;
  std::vector<cudaEvent_t> evs;
  auto bail = [&](int s) {
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    delete r;
    return s;
  };
  int s;
  DevBuf<int32_t> rank, tmp, big;
  DevBuf<int64_t> kept, inc;
  DevBuf<int> nbig, nhubq;
  DevBuf<unsigned long long> hubcnt;
  DevBuf<int2> hubq;
  // hub block tasks: at most nsym / kHubBlock + (number of hubs) of them
  const int64_t maxq = nsym / kHubBlock + nsym / (kHubBlock + 1) + 1;
  if ((s = r->order.reserve(n)) || (s = rank.reserve(n)) || (s = kept.reserve(n)) || (s = r->roff.reserve(n + 1)) ||
      (s = inc.reserve(n)) || (s = r->rinc.reserve(n + 1)) || (s = tmp.reserve(std::max<int64_t>(nsym, 1))) ||
      (s = big.reserve(n)) || (s = nbig.reserve(1)) ||
      (s = nhubq.reserve(1)) || (s = hubcnt.reserve(n)) || (s = hubq.reserve(maxq)))
    return bail(s);
  // vertex ranges of the adjacency chunks (about nsym / 16 edges each)
  std::vector<int64_t> cut{0};
  if (h_adj && nsym > 0) {
    const int chunks = 16;
    for (int c = 1; c < chunks; ++c) {
      const int64_t want = nsym * c / chunks;
      int64_t v = std::lower_bound(h_off, h_off + n + 1, want) - h_off;
      if (v > cut.back() && v < n) cut.push_back(v);
    }
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
      cs = nullptr;
      return bail(fail(GPM_ECUDA, "copy stream"));
    }
  }
  cut.push_back(n);
  // 1. the adjacency upload, chunk by chunk on its own stream
  if (h_adj)
    for (size_t c = 0; c + 1 < cut.size(); ++c) {
      const int64_t e0 = h_off[cut[c]], e1 = h_off[cut[c + 1]];
      cudaEvent_t ev;
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(GPM_ECUDA, "event"));
      evs.push_back(ev);
      if (e1 > e0 && cudaMemcpyAsync(g->adj.p + e0, h_adj + e0, sizeof(int32_t) * (e1 - e0),
                                     cudaMemcpyHostToDevice, cs) != cudaSuccess)
        return bail(fail(GPM_ECUDA, "adjacency upload"));
      cudaEventRecord(ev, cs);
    }
  // 2. ranks from the degrees alone (symmetric input), meanwhile; a
  // vertex's symmetric degree is its incident-edge count in the DAG
  if ((s = rank_order(g, nullptr, nullptr, 1, r->order.p, rank.p, inc.p, st))) return bail(s);
  if ((s = scan_i64(n, inc.p, r->rinc.p, st))) return bail(s);
  // 3. each chunk gathered as soon as it has landed: small lists one warp
  // each, hub lists as block tasks over the whole grid
  cudaMemsetAsync(nbig.p, 0, sizeof(int), st);
  cudaMemsetAsync(nhubq.p, 0, sizeof(int), st);
  const int qgrid = num_sms() * 8;
  for (size_t c = 0; c + 1 < cut.size(); ++c) {
    if (h_adj) cudaStreamWaitEvent(st, evs[c], 0);
    const int64_t nv = cut[c + 1] - cut[c];
    if (nv == 0) continue;
    // the queue is drained by this chunk's hub launch, so each chunk starts it at 0
    cudaMemsetAsync(nhubq.p, 0, sizeof(int), st);
    k_up_gather<<<grid_for(nv * 32), 256, 0, st>>>(cut[c], cut[c + 1], rank.p, g->off.p, g->adj.p, tmp.p, kept.p,
                                                   hubcnt.p, hubq.p, nhubq.p);
    k_up_gather_hub<<<qgrid, 256, 0, st>>>(hubq.p, nhubq.p, rank.p, g->off.p, g->adj.p, tmp.p, hubcnt.p);
    k_up_hub_kept<<<qgrid, 256, 0, st>>>(hubq.p, 0, nhubq.p, rank.p, hubcnt.p, kept.p);
  }
  // 4. list offsets, then the lists moved to them
  if ((s = scan_i64(n, kept.p, r->roff.p, st))) return bail(s);
  int64_t nnz = 0;
  int hbig = 0;
  cudaMemcpyAsync(&nnz, r->roff.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&r->nin, r->rinc.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank relabel: ") + cudaGetErrorString(e)));
  if ((s = r->radj.reserve(std::max<int64_t>(nnz, 1)))) return bail(s);
  k_up_compact<<<grid_for(n * 32, kGatherWarps * 32), kGatherWarps * 32, 0, st>>>(
      n, r->order.p, g->off.p, tmp.p, r->roff.p, r->radj.p, big.p, nbig.p);
  cudaMemcpyAsync(&hbig, nbig.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank relabel: ") + cudaGetErrorString(e)));
  if ((s = finish_rank_graph(r, n, nnz, big.p, hbig, st))) return bail(s);
  if (cs) cudaStreamDestroy(cs);
  cs = nullptr;
  for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
  evs.clear();
  g->rg = r;
  return GPM_OK;
}

int ensure_rank_graph(gpm_graph *g, cudaStream_t st, const int32_t *gid, int ngraphs, bool upward_only) {
  if (g->rg) return GPM_OK;
  if (upward_only) return build_upward_rank_graph(g, st, nullptr, nullptr);
  const int64_t n = g->n, nnz = g->nnz;
  RankGraph *r = new RankGraph();
  auto bail = [&](int s) {
    delete r;
    return s;
  };
  int s;
  DevBuf<int32_t> indeg, rank, big;
  DevBuf<int64_t> rdeg, inc;
  DevBuf<int> nbig;
  if ((s = indeg.reserve(n)) || (s = r->order.reserve(n)) || (s = rank.reserve(n)) || (s = rdeg.reserve(n)) ||
      (s = inc.reserve(n)) || (s = r->roff.reserve(n + 1)) || (s = r->rinc.reserve(n + 1)) ||
      (s = r->radj.reserve(std::max<int64_t>(nnz, 1))) || (s = big.reserve(n)) || (s = nbig.reserve(1)))
    return bail(s);
  cudaMemsetAsync(indeg.p, 0, sizeof(int32_t) * n, st);
  k_indeg<<<grid_for(nnz), 256, 0, st>>>(nnz, g->adj.p, indeg.p);
  if ((s = rank_order(g, indeg.p, gid, ngraphs, r->order.p, rank.p, rdeg.p, st))) return bail(s);
  if ((s = scan_i64(n, rdeg.p, r->roff.p, st))) return bail(s);
  k_incident<<<grid_for(n), 256, 0, st>>>(n, r->order.p, rdeg.p, indeg.p, inc.p);
  if ((s = scan_i64(n, inc.p, r->rinc.p, st))) return bail(s);
  cudaMemcpyAsync(&r->nin, r->rinc.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  // gather + sort in one pass; lists longer than kSortCap get a segmented
  // sort of their own afterwards
  cudaMemsetAsync(nbig.p, 0, sizeof(int), st);
  k_rank_gather_sort<<<grid_for(n * 32, kGatherWarps * 32), kGatherWarps * 32, 0, st>>>(
      n, r->order.p, rank.p, g->off.p, g->adj.p, r->roff.p, r->radj.p, big.p, nbig.p);
  int hbig = 0;
  cudaMemcpyAsync(&hbig, nbig.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank relabel: ") + cudaGetErrorString(e)));
  if ((s = finish_rank_graph(r, n, nnz, big.p, hbig, st))) return bail(s);
  g->rg = r;
  return GPM_OK;
}

int rank_build_plan(gpm_graph *g, int cta_min, int long_min, cudaStream_t st) {
  if (g->rank && g->rank->cta_min == cta_min && g->rank->long_min == long_min) return GPM_OK;
  free_rank_plan(g->rank);
  g->rank = nullptr;
  RankPlan *p = nullptr;
  GPM_TRY(rank_plan_new(g, cta_min, long_min, nullptr, st, &p));
  g->rank = p;
  return GPM_OK;
}

// roff4 of the rank graph and room for radj4 (kept with it); *fill: radj4
// is still empty and the next placement pass writes it.  radj4 takes at
// most nnz + 3n keys, so no count is read back.
static int ensure_padded_lists(gpm_graph *g, cudaStream_t st, bool *fill) {
  RankGraph *r = g->rg;
  *fill = false;
  if (r->padded) return GPM_OK;
  const int64_t n = g->n;
  DevBuf<int64_t> len4;
  GPM_TRY(len4.reserve(std::max<int64_t>(n, 1)));
  GPM_TRY(r->roff4.reserve(n + 1));
  GPM_TRY(r->radj4.reserve(r->radj.n + 3 * (size_t)n + 4));  // radj.n: the rank graph's stored keys
  k_padded_len<<<grid_for(n), 256, 0, st>>>(n, r->roff.p, len4.p);
  GPM_LAUNCH_CHECK();
  GPM_TRY(scan_i64(n, len4.p, r->roff4.p, st));
  *fill = true;
  return GPM_OK;
}

// Resident CTAs of k_tc_dense x SMs (its largest shared-memory size, rows
// of kRankCtaWords words, does not limit its occupancy).
static int dense_grid() {
  static PerDevice grid;
  return grid.get([] {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_dense, 256, (kRankCtaWords + 4) * sizeof(uint32_t));
    return std::max(1, per_sm) * num_sms();
  });
}

// The side stream of the current device that k_tc_dense runs on (created on
// first use, kept until the process exits; every plan of the device shares it).
static cudaStream_t dense_stream(int *status) {
  static std::mutex mu;
  static cudaStream_t side[64];
  int dev = 0;
  *status = GPM_OK;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    *status = fail(GPM_ECUDA, "dense kernel: no current device below index 64");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!side[dev] && cudaStreamCreateWithFlags(&side[dev], cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    side[dev] = nullptr;
    *status = fail(GPM_ECUDA, "dense kernel: side stream");
  }
  return side[dev];
}

static int64_t env_or(const char *name, int64_t dflt) {
  const char *e = getenv(name);
  return e && *e ? atoll(e) : dflt;
}

// The dense core of a plan: core_base, the rows and rowid (see
// RankPlan).  GPM_TC_CORE, GPM_TC_CORE_MIN and GPM_TC_DENSE_PCT override
// GPM_RANK_CORE, GPM_RANK_CORE_MIN and GPM_RANK_DENSE_PCT.  The rows are left
// out (p->n_rows = 0) when none qualifies or they would take more than 1 GiB
// and more than four times the bytes of the rank graph's lists (R-MAT 22:
// 176 MB of rows against 257 MB of lists).
static int build_core_rows(gpm_graph *g, RankPlan *p, DevBuf<int32_t> &rowid, int *dense_pct, cudaStream_t st) {
  const int64_t n = g->n;
  const int64_t K = env_or("GPM_TC_CORE", GPM_RANK_CORE);
  const int64_t min_keys = std::max<int64_t>(1, env_or("GPM_TC_CORE_MIN", GPM_RANK_CORE_MIN));
  *dense_pct = (int)std::max<int64_t>(0, env_or("GPM_TC_DENSE_PCT", GPM_RANK_DENSE_PCT));
  if (K <= 0 || n <= 0 || n > INT32_MAX - 128) return GPM_OK;
  const int32_t core_base = (int32_t)(std::max<int64_t>(0, n - K) & ~(int64_t)127);
  const int64_t row_words = ((n - core_base + 127) >> 7) << 2;
  // k_tc_dense holds an owner's bitmap of up to row_words + 4 words in shared
  // memory, sized (and its occupancy taken) for kRankCtaWords + 4
  if (row_words > (int64_t)kRankCtaWords) return GPM_OK;
  DevBuf<int> nrows;
  GPM_TRY(rowid.reserve(n));
  GPM_TRY(nrows.reserve(1));
  GPM_CUDA(cudaMemsetAsync(nrows.p, 0, sizeof(int), st));
  k_core_rowid<<<grid_for(n), 256, 0, st>>>(n, g->rg->roff.p, g->rg->radj.p, core_base, (int)min_keys, rowid.p,
                                            nrows.p);
  GPM_LAUNCH_CHECK();
  int h = 0;
  GPM_CUDA(cudaMemcpyAsync(&h, nrows.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  if (h <= 0) return GPM_OK;
  const size_t bytes = (size_t)h * (size_t)row_words * 4;
  if (bytes > std::max<size_t>((size_t)1 << 30, 16 * (size_t)g->rg->radj.n)) return GPM_OK;
  if (bytes / 16 >= ((size_t)1 << 31)) return GPM_OK;  // a dense descriptor indexes the rows' uint4 in 31 bits
  GPM_TRY(p->rows.reserve((size_t)h * (size_t)row_words));
  GPM_CUDA(cudaMemsetAsync(p->rows.p, 0, bytes, st));
  k_core_rows<<<grid_for(n * 32), 256, 0, st>>>(n, g->rg->roff.p, g->rg->radj.p, core_base, rowid.p,
                                                (int)row_words, p->rows.p);
  GPM_LAUNCH_CHECK();
  p->core_base = core_base;
  p->row_words = (int)row_words;
  p->n_rows = h;
  return GPM_OK;
}

int rank_plan_new(gpm_graph *g, int cta_min, int long_min, const uint8_t *cfg, cudaStream_t st, RankPlan **out) {
  GPM_TRY(ensure_rank_graph(g, st));
  bool fill = false;
  GPM_TRY(ensure_padded_lists(g, st, &fill));
  const int64_t n = g->n;
  RankPlan *p = new RankPlan();
  p->cta_min = cta_min;
  p->long_min = long_min;
  auto bail = [&](int s) {
    delete p;
    return s;
  };
  int s;
  const int64_t nin = g->rg->nin;
  if ((s = p->poff.reserve(n + 1)) || (s = p->pseg.reserve(std::max<int64_t>(nin, 1))) ||
      (s = p->plong.reserve(n)) || (s = p->pshort.reserve(n)) || (s = p->counters.reserve(4)))
    return bail(s);
  const int64_t *roff = g->rg->roff.p;
  const int32_t *radj = g->rg->radj.p;
  // 2. segments placed in their owners' rooms, one pass
  DevBuf<unsigned long long> work;
  if ((s = work.reserve(n))) return bail(s);
  cudaMemcpyAsync(p->poff.p, g->rg->rinc.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(p->plong.p, 0, sizeof(int32_t) * n, st);
  cudaMemsetAsync(p->pshort.p, 0, sizeof(int32_t) * n, st);
  cudaMemsetAsync(work.p, 0, sizeof(unsigned long long) * n, st);
  // 8-byte segment descriptors address radj4 by 16-byte rows in 31 bits
  if ((int64_t)(g->rg->radj4.n / 4) >= ((int64_t)1 << 31))
    return bail(fail(GPM_EUNSUPPORTED, "triangle plan: more than 2^33 padded keys"));
  DevBuf<int32_t> rowid;
  int dense_pct = 0;
  // the dense core does not depend on the schedule: every plan has it
  if ((s = build_core_rows(g, p, rowid, &dense_pct, st))) return bail(s);
  if (p->n_rows) {
    if ((s = p->pdense.reserve(n))) return bail(s);
    cudaMemsetAsync(p->pdense.p, 0, sizeof(int32_t) * n, st);
  }
  // sizes: [0] CTA tasks, [1] warp tasks, [2] dense tasks, [3] dense-only
  // owners, [4] a segment too long for its descriptor
  DevBuf<int> sizes;
  if ((s = sizes.reserve(5))) return bail(s);
  cudaMemsetAsync(sizes.p, 0, 5 * sizeof(int), st);
  k_partner_place<<<grid_for(n * 32), 256, 0, st>>>(n, roff, radj, g->rg->roff4.p, fill ? g->rg->radj4.p : nullptr,
                                                     g->rg->upward, long_min, cfg, p->poff.p, p->plong.p, p->pshort.p,
                                                     p->pseg.p, work.p, p->core_base, p->n_rows ? rowid.p : nullptr,
                                                     p->row_words, dense_pct, p->pdense.p, sizes.p + 4);
  GPM_LAUNCH_CHECK();
  if (p->n_rows) {  // the dense segments moved out of the long ones
    DevBuf<int64_t> cnt;
    if ((s = cnt.reserve(n)) || (s = p->doff.reserve(n + 1))) return bail(s);
    k_widen<<<grid_for(n), 256, 0, st>>>(n, p->pdense.p, cnt.p);
    if ((s = scan_i64(n, cnt.p, p->doff.p, st))) return bail(s);
    int64_t total = 0;
    cudaMemcpyAsync(&total, p->doff.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    cudaError_t e0 = cudaStreamSynchronize(st);
    if (e0 != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank plan: ") + cudaGetErrorString(e0)));
    if ((s = p->dseg.reserve(std::max<int64_t>(total, 1)))) return bail(s);
    k_split_dense<<<grid_for(n * 32), 256, 0, st>>>(n, p->poff.p, p->plong.p, p->pdense.p, p->doff.p, p->pseg.p,
                                                    p->dseg.p);
    GPM_LAUNCH_CHECK();
  }
  if (fill) g->rg->padded = 1;
  // 3. task queues, heaviest first
  DevBuf<unsigned long long> ckey, wkey;
  DevBuf<int32_t> cval, wval;
  DevBuf<unsigned long long> dkey;
  DevBuf<int32_t> dval;
  if ((s = ckey.reserve(n)) || (s = wkey.reserve(n)) || (s = cval.reserve(n)) || (s = wval.reserve(n)) ||
      (s = p->cta_tasks.reserve(n)) || (s = p->warp_tasks.reserve(n)))
    return bail(s);
  const int32_t *pdense = p->n_rows ? p->pdense.p : nullptr;
  if (pdense && (s = p->dense_only.reserve(n))) return bail(s);
  k_rank_tasks<<<grid_for(n), 256, 0, st>>>(n, roff, p->plong.p, p->pshort.p, work.p, cta_min, cfg, pdense,
                                            p->dense_only.p, ckey.p, cval.p, wkey.p, wval.p, sizes.p);
  if (pdense) {
    if ((s = dkey.reserve(n)) || (s = dval.reserve(n))) return bail(s);
    k_dense_tasks<<<grid_for(n), 256, 0, st>>>(n, roff, radj, pdense, dkey.p, dval.p, sizes.p + 2);
  }
  int h[5] = {0, 0, 0, 0, 0};
  cudaMemcpyAsync(h, sizes.p, sizeof h, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank plan: ") + cudaGetErrorString(e)));
  if (h[4]) return bail(fail(GPM_EUNSUPPORTED, "triangle plan: a partner segment of 2^29 keys or more"));
  p->n_cta = h[0];
  p->n_warp = h[1];
  p->n_dense = h[2];
  p->n_dense_only = h[3];
  if (p->n_dense && (s = p->dense_tasks.reserve(p->n_dense))) return bail(s);
  if ((s = sort_pairs_u64(ckey, cval, h[0], p->cta_tasks, st)) || (s = sort_pairs_u64(wkey, wval, h[1], p->warp_tasks, st)) ||
      (s = sort_pairs_u64(dkey, dval, h[2], p->dense_tasks, st)))
    return bail(s);
  if (p->n_dense) {
    p->dense_smem = (size_t)(p->row_words + 4) * sizeof(uint32_t);
    p->dense_grid = std::max(1, std::min(dense_grid(), p->n_dense));
    if (cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(GPM_ECUDA, "rank plan: events for the dense kernel"));
    }
  }
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(fail(GPM_ECUDA, std::string("rank plan: ") + cudaGetErrorString(e)));
  *out = p;
  return GPM_OK;
}

static int rank_grid() {
  static PerDevice grid;
  return grid.get([] {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_rank, 256, kRankSmem);
    return std::max(1, per_sm) * num_sms();
  });
}

// Launch of a given plan; rec != nullptr selects the instrumented build.
int rank_plan_launch(gpm_graph *g, RankPlan *p, cudaStream_t st, unsigned long long *d_out,
                     unsigned long long *rec) {
  GPM_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
  if (g->nnz == 0) return GPM_OK;
  GPM_CUDA(cudaMemsetAsync(p->counters.p, 0, 4 * sizeof(int), st));
  if (p->n_dense) {  // forked onto the device's side stream, joined after the count kernel
    int s = GPM_OK;
    cudaStream_t side = dense_stream(&s);
    if (s != GPM_OK) return s;
    GPM_CUDA(cudaEventRecord(p->fork, st));
    GPM_CUDA(cudaStreamWaitEvent(side, p->fork, 0));
    k_tc_dense<<<p->dense_grid, 256, p->dense_smem, side>>>(g->rg->roff.p, g->rg->radj.p, p->doff.p, p->dseg.p,
                                                             p->dense_tasks.p, p->n_dense,
                                                             reinterpret_cast<const uint4 *>(p->rows.p),
                                                             p->counters.p + 2, d_out);
    GPM_LAUNCH_CHECK();
    GPM_CUDA(cudaEventRecord(p->join, side));
  }
  if (rec)
    k_tc_rank_t<true><<<rank_grid(), 256, kRankSmem, st>>>(
        g->rg->roff.p, g->rg->radj.p, g->rg->radj4.p, p->poff.p, p->pseg.p, p->plong.p, p->pshort.p, p->cta_tasks.p,
        p->n_cta, p->warp_tasks.p, p->n_warp, p->counters.p, d_out, rec);
  else
    k_tc_rank<<<rank_grid(), 256, kRankSmem, st>>>(g->rg->roff.p, g->rg->radj.p, g->rg->radj4.p, p->poff.p,
                                                   p->pseg.p, p->plong.p, p->pshort.p, p->cta_tasks.p, p->n_cta,
                                                   p->warp_tasks.p, p->n_warp, p->counters.p, d_out, nullptr);
  GPM_LAUNCH_CHECK();
  if (p->n_dense) GPM_CUDA(cudaStreamWaitEvent(st, p->join, 0));
  return GPM_OK;
}

int rank_launch(gpm_graph *g, cudaStream_t st, unsigned long long *d_out) {
  if (g->nnz == 0) return cudaMemsetAsync(d_out, 0, 8, st) == cudaSuccess ? GPM_OK : GPM_ECUDA;
  // fixed schedule: owners with > kRankCtaMin keys go to a CTA, segments of
  // >= kRankLongMin keys are streamed by a half-warp
  GPM_TRY(rank_build_plan(g, kRankCtaMin, kRankLongMin, st));
  return rank_plan_launch(g, g->rank, st, d_out, nullptr);
}

// out[0] segments, out[1] keys in them, out[2] keys of the owners' lists
__global__ void k_plan_stats(const int32_t *__restrict__ tasks, int ntasks, const int64_t *__restrict__ roff,
                             const int64_t *__restrict__ poff, const Seg *__restrict__ pseg,
                             const int32_t *__restrict__ plong, const int32_t *__restrict__ pshort,
                             const int32_t *__restrict__ pdense, const int32_t *__restrict__ radj,
                             unsigned long long *__restrict__ out) {
  unsigned long long segs = 0, keys = 0, okeys = 0, dsegs = 0, dwords = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntasks; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t x = tasks[t];
    const int nd = pdense ? pdense[x] : 0;
    okeys += (unsigned long long)(roff[x + 1] - roff[x]);
    segs += (unsigned long long)(plong[x] + pshort[x] + nd);
    if (nd) {  // dense: the owner's bitmap words each
      dsegs += (unsigned long long)nd;
      dwords += (unsigned long long)nd * (unsigned long long)core_and_words(radj[roff[x]], radj[roff[x + 1] - 1]);
    }
    for (int64_t j = poff[x]; j < poff[x] + plong[x]; ++j) keys += (unsigned long long)seg_keys(pseg[j]);
    for (int64_t j = poff[x + 1] - pshort[x]; j < poff[x + 1]; ++j) keys += (unsigned long long)seg_keys(pseg[j]);
  }
  segs = warp_sum(segs);
  keys = warp_sum(keys);
  okeys = warp_sum(okeys);
  dsegs = warp_sum(dsegs);
  dwords = warp_sum(dwords);
  if (lane_id() == 0) {
    atomicAdd(&out[0], segs);
    atomicAdd(&out[1], keys);
    atomicAdd(&out[2], okeys);
    atomicAdd(&out[3], dsegs);
    atomicAdd(&out[4], dwords);
  }
}

int rank_plan_stats(gpm_graph *g, uint64_t *out) {
  for (int i = 0; i < 6; ++i) out[i] = 0;
  if (g->nnz == 0) return GPM_OK;
  GPM_TRY(rank_build_plan(g, kRankCtaMin, kRankLongMin, 0));
  RankPlan *p = g->rank;
  DevBuf<unsigned long long> o;
  GPM_TRY(o.reserve(5));
  GPM_CUDA(cudaMemset(o.p, 0, 40));
  const int grid = num_sms() * 8;
  const int32_t *pdense = p->n_rows ? p->pdense.p : nullptr;
  k_plan_stats<<<grid, 256>>>(p->cta_tasks.p, p->n_cta, g->rg->roff.p, p->poff.p, p->pseg.p, p->plong.p,
                              p->pshort.p, pdense, g->rg->radj.p, o.p);
  k_plan_stats<<<grid, 256>>>(p->warp_tasks.p, p->n_warp, g->rg->roff.p, p->poff.p, p->pseg.p, p->plong.p,
                              p->pshort.p, pdense, g->rg->radj.p, o.p);
  if (p->n_dense_only)
    k_plan_stats<<<grid, 256>>>(p->dense_only.p, p->n_dense_only, g->rg->roff.p, p->poff.p, p->pseg.p, p->plong.p,
                                p->pshort.p, pdense, g->rg->radj.p, o.p);
  GPM_LAUNCH_CHECK();
  unsigned long long h[5];
  GPM_CUDA(cudaMemcpy(h, o.p, sizeof h, cudaMemcpyDeviceToHost));
  out[0] = h[0];
  out[1] = h[1];
  out[2] = h[2];
  out[3] = (uint64_t)(p->n_cta + p->n_warp + p->n_dense_only);
  out[4] = h[3];
  out[5] = h[4];
  return GPM_OK;
}

}  // namespace gpm

extern "C" int gpm_tc_plan_stats(gpm_graph *g, uint64_t *stats) {
  if (!g || !stats) return gpm::fail(GPM_EINVAL, "gpm_tc_plan_stats: NULL argument");
  return gpm::rank_plan_stats(g, stats);
}
