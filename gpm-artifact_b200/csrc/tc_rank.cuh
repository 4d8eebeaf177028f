// tc_rank.cuh -- rank-relabelled copy of a graph and the plan of the
// smaller-side triangle count built on it.
#pragma once
#include "common.cuh"

namespace gpm {

#ifndef GPM_RANK_CTA_WORDS
// 24 KB of shared memory per CTA of the count kernel (8 CTAs = 192 KB of an
// SM's 228 KB): a byte map of 24,576 ids, a bitmap of 196,608 ids or a
// 4096-slot hash table; a warp task gets an eighth (3,072 ids / 24,576 ids /
// 512 slots)
#define GPM_RANK_CTA_WORDS 6144
#endif
constexpr int kRankCtaWords = GPM_RANK_CTA_WORDS;
#ifndef GPM_RANK_CTA_MIN
// fixed schedule: owners with more keys than this are CTA tasks.  With the
// dense core segments in their own kernel, R-MAT 20 / 21 / 22 (ms): 100 ->
// 1.030 / 2.210 / 5.349, 80 -> 1.002 / - / 5.472, 128 -> 1.269 / 2.212 /
// 5.367, 160 -> 1.349 / 2.800 / 5.370 (long threshold 48); before the dense
// core the best was 50 (R-MAT 22 6.49 ms, against 6.55 at 128)
#define GPM_RANK_CTA_MIN 100
#endif
constexpr int kRankCtaMin = GPM_RANK_CTA_MIN;
// fixed schedule: partner segments of at least this many keys are streamed
// by a half-warp, shorter ones by 4-lane groups (16-byte rows).  With the
// dense core (CTA threshold 100), R-MAT 20 / 21 / 22 (ms): 48 -> 1.030 /
// 2.210 / 5.349, 64 -> 1.023 / 2.211 / 5.441, 96 -> 1.011 / 2.194 / 5.424,
// 32 -> 1.048 / - / 5.404 (CTA threshold 80: 24 -> 5.580, 32 -> 5.498, 48 ->
// 5.472 at R-MAT 22); before the dense core 16 was best (R-MAT 22: 6.47-6.49
// ms at 16, 6.53 at 8, 6.51-6.57 at 24; every segment to 8-lane groups 7.17)
#ifndef GPM_RANK_LONG_MIN
#define GPM_RANK_LONG_MIN 48
#endif
constexpr int kRankLongMin = GPM_RANK_LONG_MIN;

// The stored graph renumbered by (in + out degree, id) rank, lists sorted.
// upward == 1 when every stored edge points to a larger rank, which holds
// for a degree-oriented DAG (orientation rule of graph.h:128-129); then
// every out-list holds only ids above its owner.
struct RankGraph {
  DevBuf<int64_t> roff;   // n + 1
  DevBuf<int32_t> radj;   // nnz
  DevBuf<int32_t> order;  // rank -> original id
  // rinc[r] .. rinc[r+1]: one slot per stored edge incident to rank r (out
  // or in); the triangle plan's segment room, nin = rinc[n]
  DevBuf<int64_t> rinc;
  int64_t nin = 0;
  int upward = 0;
  // The lists again, each padded with INT32_MAX to a multiple of four keys
  // and starting at a multiple of four (roff4), for the count kernel's
  // 16-byte loads: an aligned 16-byte row of a clipped partner segment then
  // stays inside its list, and the keys it holds outside the segment lie
  // below the owner's smallest key or above its largest (built with the
  // first triangle plan)
  DevBuf<int64_t> roff4;
  DevBuf<int32_t> radj4;
  int padded = 0;  // radj4 written
};

#ifndef GPM_RANK_CORE
// dense core of the fixed plan: the top this-many ranks (0: none).  R-MAT 22
// holds 64 % of its streamed keys in owners of the top 16,384 ranks
#define GPM_RANK_CORE 16384
#endif
#ifndef GPM_RANK_CORE_MIN
// a vertex gets a core bitmap row when at least this many of its keys lie
// in the core (R-MAT 22: 86,115 rows of 2 KB)
#define GPM_RANK_CORE_MIN 128
#endif
#ifndef GPM_RANK_DENSE_PCT
// a core owner's segment with a row is ANDed as bitmap words when its key
// count is at least this percentage of the words to AND
#define GPM_RANK_DENSE_PCT 100
#endif

// A partner segment in 8 bytes.  A segment read as keys: x = its first
// 16-byte row of radj4 (>= 0), y = keys << 2 | the position of its first key
// in that row; dense: x = -1 - (uint4 index of its core row words), y =
// keys << 2.  Plans stop with GPM_EUNSUPPORTED where radj4 holds 2^31 rows or
// more, or a segment 2^29 keys or more.
using Seg = int2;
__host__ __device__ __forceinline__ int seg_keys(Seg s) { return (int)((uint32_t)s.y >> 2); }
__host__ __device__ __forceinline__ int seg_rows(Seg s) { return (int)(((s.y & 3) + ((uint32_t)s.y >> 2) + 3) >> 2); }

// Core bitmaps of an owner x whose keys all lie in the core (min N(x) >=
// core_base): N(x) as bits from base = min N(x) rounded down to 128, so
// bitmap word i lines up with word (base - core_base) / 32 + i of every core
// row and 16-byte loads of both stay aligned.  and_words: the words that can
// hold keys of N(x) (a multiple of four); clear_words: those plus the word of
// the zero guard bit at max N(x) - base + 1 (a multiple of four).
__host__ __device__ __forceinline__ int core_and_words(int32_t kmin, int32_t kmax) {
  return (((kmax - (kmin & ~127)) >> 5) + 4) & ~3;
}
__host__ __device__ __forceinline__ int core_clear_words(int32_t kmin, int32_t kmax) {
  return (((kmax - (kmin & ~127) + 1) >> 5) + 4) & ~3;
}

// Per-graph schedule of GPM_TC_BITMAP (device arrays):
//   poff/pseg   partner segments: owner x has the room pseg[poff[x] ..
//               poff[x+1]) (poff = rinc, one slot per incident edge); its
//               plong[x] long segments fill the room from the front, its
//               pshort[x] short ones from the back.  A segment (a Seg,
//               above) names the 16-byte rows of radj4 holding the part of
//               one partner's list inside [min N(x), max N(x)] (no key
//               outside that range can be in N(x)); empty ranges are left out
//   cta_tasks / warp_tasks  owners by size class, heaviest first
//   rows        dense core: ranks [core_base, n) with
//               core_base a multiple of 128; row r holds, as row_words bits
//               from core_base, the core keys of one vertex that has at
//               least GPM_RANK_CORE_MIN of them.  A long segment
//               {-1 - i, keys} is dense: its owner lies in the core and the
//               count is popc(row & N(owner)) over the owner's words, with
//               the partner's row words from the owner's base on starting at
//               uint4 index i of rows, instead of streaming the partner's
//               keys; placed among the long segments, then moved to dseg
//               (below); k_tc_dense counts them (tasks: dense_tasks)
struct RankPlan {
  int cta_min = 0, long_min = 0;
  int n_cta = 0, n_warp = 0;
  int32_t core_base = INT32_MAX;  // INT32_MAX: no dense core
  int row_words = 0;              // multiple of 4
  int64_t n_rows = 0;
  DevBuf<uint32_t> rows;
  DevBuf<int32_t> pdense;       // dense segments per owner
  // the dense segments, apart from pseg: owner x's are dseg[doff[x] ..
  // doff[x+1]); plong[x] counts only x's other long segments
  DevBuf<int64_t> doff;         // n + 1
  DevBuf<Seg> dseg;
  DevBuf<int32_t> dense_tasks;  // owners with dense segments, most words first
  DevBuf<int32_t> dense_only;   // owners with dense segments only (in neither task queue)
  int n_dense = 0, n_dense_only = 0, dense_grid = 0;
  size_t dense_smem = 0;
  // k_tc_dense runs on the device's side stream (one per device, kept until
  // exit), forked from and joined back into the caller's stream by the two
  // events, so that it overlaps the count kernel
  cudaEvent_t fork = nullptr, join = nullptr;
  RankPlan() = default;
  RankPlan(const RankPlan &) = delete;
  RankPlan &operator=(const RankPlan &) = delete;
  ~RankPlan() {
    if (join) cudaEventSynchronize(join);  // the side stream's last use of the buffers
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
  }
  DevBuf<int64_t> poff;
  DevBuf<Seg> pseg;
  DevBuf<int32_t> plong, pshort;
  DevBuf<int32_t> cta_tasks, warp_tasks;
  DevBuf<int> counters;
};

// upward_only: keep only neighbours of larger rank, i.e. orient a symmetric
// graph and relabel it in one pass (the DAG's own id order is lost).
int ensure_rank_graph(gpm_graph *g, cudaStream_t st, const int32_t *gid = nullptr, int ngraphs = 1,
                      bool upward_only = false);
// The upward rank graph of a symmetric graph (orientation folded into the
// relabel).  g->off must be on the device; with h_off/h_adj (host arrays,
// pinned for overlap) the adjacency is uploaded into g->adj in chunks on a
// copy stream, each chunk relabelled as soon as it lands; with nullptr,
// g->adj is already on the device.
int build_upward_rank_graph(gpm_graph *g, cudaStream_t st, const int64_t *h_off, const int32_t *h_adj);
int rank_build_plan(gpm_graph *g, int cta_min, int long_min, cudaStream_t st);
int rank_launch(gpm_graph *g, cudaStream_t st, unsigned long long *d_out);
// out[0..5]: segments, keys streamed from the key segments, owner-list keys,
// owner tasks, dense segments, bitmap words ANDed for them (fixed plan)
int rank_plan_stats(gpm_graph *g, uint64_t *out);
// An uncached plan; cfg (device, one byte per vertex, may be nullptr) gives
// each owner its queue (cfg / 3: 0 warp, 1 CTA) and long-segment threshold
// ({16, 64, 256}[cfg % 3]) instead of the fixed thresholds.
int rank_plan_new(gpm_graph *g, int cta_min, int long_min, const uint8_t *cfg, cudaStream_t st, RankPlan **out);
// rec != nullptr: instrumented run adding each owner's cost (active warp-cycles)
// to rec[owner]; rec must be zeroed first
int rank_plan_launch(gpm_graph *g, RankPlan *p, cudaStream_t st, unsigned long long *d_out,
                     unsigned long long *rec);

}  // namespace gpm
