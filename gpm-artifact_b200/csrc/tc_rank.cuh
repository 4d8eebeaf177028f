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
// fixed schedule: owners with more keys than this are CTA tasks (R-MAT 22:
// 7.65 ms at 50 against 8.0 ms at the reference's USE_CTA = 100 and 7.67 ms
// at 70; smaller owners rarely fit a warp's bitmap and hash instead)
#define GPM_RANK_CTA_MIN 50
#endif
constexpr int kRankCtaMin = GPM_RANK_CTA_MIN;
// fixed schedule: partner segments of at least this many keys are streamed
// by a half-warp, shorter ones by 4-lane groups (16-byte rows, R-MAT 22:
// 6.47-6.49 ms at 16, 6.53 at 8, 6.51-6.57 at 24; with 8-lane groups 6.63 ms
// at 32, 6.66 at 24 and 128, 6.72 at 64; 2-lane groups 6.52 ms at 8 or 16;
// every segment to 8-lane groups 7.17 ms)
#ifndef GPM_RANK_LONG_MIN
#define GPM_RANK_LONG_MIN 16
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

// Per-graph schedule of GPM_TC_BITMAP (device arrays):
//   poff/pseg   partner segments: owner x has the room pseg[poff[x] ..
//               poff[x+1]) (poff = rinc, one slot per incident edge); its
//               plong[x] long segments fill the room from the front, its
//               pshort[x] short ones from the back.  A segment is the
//               [start, end) range of radj4 holding the part of one
//               partner's list inside [min N(x), max N(x)] (no key outside
//               that range can be in N(x)); empty ranges are left out
//   cta_tasks / warp_tasks  owners by size class, heaviest first
struct RankPlan {
  int cta_min = 0, long_min = 0;
  int n_cta = 0, n_warp = 0;
  DevBuf<int64_t> poff;
  DevBuf<longlong2> pseg;
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
// out[0..3]: segments, keys in them, owner-list keys, owner tasks of the fixed plan
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
