// pattern.cu -- named patterns P1..P8 and Motif4 (G2MinerSolver,
// src/G2MinerSolver.cuh:17-176, and PatternSolver, src/PatternSolver.cuh:16-265).
//
// Both reference families compute, per stored edge (v0, v1) of the symmetric
// graph, the same nested set algebra (G2Miner with materialised lists,
// PatternSolver with frequency products minus corrections); on sorted
// duplicate-free lists they give the same counts:
//   P1, Motif4[0]  induced 3-stars            (motif pipeline, motif.cu)
//   P4, Motif4[1]  induced 4-paths            (motif pipeline)
//   Motif4[2..5]   tailed triangle, 4-cycle, diamond, 4-clique (motif pipeline)
//   P2 P3 P5 P6 P7 P8  enumerated here: one warp per stored edge, lists
//   materialised in per-warp global scratch with ballot compaction (order
//   preserved), membership by binary search in the longer list.
// The per-edge programs restate G2Miner_kernels.cuh:52-435.
#include <algorithm>
#include <string>

#include "common.cuh"
#include "motif.cuh"
#include "tc_rank.cuh"

namespace gpm {

constexpr int32_t kNoUb = 0x7fffffff;

__device__ __forceinline__ bool member(const int32_t *__restrict__ b, int nb, int32_t key) {
  int lo = 0, hi = nb - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int32_t x = __ldg(b + mid);
    if (x == key) return true;
    if (x < key) lo = mid + 1; else hi = mid - 1;
  }
  return false;
}

// out = {x in a : x < ub, (x in b) == keep_in}; returns |out| (warp-uniform).
// out == nullptr: count only.
__device__ int wset(const int32_t *a, int na, const int32_t *b, int nb, int32_t ub, bool keep_in, int32_t *out,
                    unsigned lane) {
  int cnt = 0;
  for (int base = 0; base < na; base += 32) {
    int i = base + lane;
    bool below = false, take = false;
    int32_t key = 0;
    if (i < na) {
      key = a[i];
      below = key < ub;
      take = below && (member(b, nb, key) == keep_in);
    }
    unsigned m = __ballot_sync(0xffffffffu, take);
    if (out && take) out[cnt + __popc(m & ((1u << lane) - 1u))] = key;
    cnt += __popc(m);
    if (__ballot_sync(0xffffffffu, i < na && !below)) break;  // sorted: the rest is >= ub
  }
  __syncwarp();
  return cnt;
}

__device__ __forceinline__ int wdiff(const int32_t *a, int na, const int32_t *b, int nb, int32_t ub, int32_t *out,
                                     unsigned lane) {
  return wset(a, na, b, nb, ub, false, out, lane);
}
__device__ __forceinline__ int wisect(const int32_t *a, int na, const int32_t *b, int nb, int32_t ub, int32_t *out,
                                      unsigned lane) {
  return wset(a, na, b, nb, ub, true, out, lane);
}
// NBR(v) expands to the (pointer, length) pair of v's sorted list
#define NBR(v) (adj + off[v]), (int)(off[(v) + 1] - off[v])
#define DIFF(...) wdiff(__VA_ARGS__, lane)
#define ISECT(...) wisect(__VA_ARGS__, lane)

__global__ void __launch_bounds__(256) k_pattern(int p, int64_t nnz, const int64_t *__restrict__ off,
                                                 const int32_t *__restrict__ adj, const int32_t *__restrict__ src,
                                                 int32_t *__restrict__ scratch, int64_t maxd,
                                                 unsigned long long *__restrict__ out) {
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int32_t *A = scratch + warp * maxd * 5, *B = A + maxd, *C = B + maxd, *D = C + maxd, *E = D + maxd;
  unsigned long long c = 0;
  for (int64_t e = warp; e < nnz; e += nw) {
    const int32_t v0 = src[e], v1 = adj[e];
    int nA, nB, nC, nD, nE;
    switch (p) {
      case 2:  // G2Miner_kernels.cuh:68-103
        nA = DIFF(NBR(v0), NBR(v1), kNoUb, A);
        nB = DIFF(NBR(v1), NBR(v0), kNoUb, B);
        for (int i = 0; i < nB; ++i) {
          nC = DIFF(A, nA, NBR(B[i]), kNoUb, C);
          for (int j = 0; j < nC; ++j) c += DIFF(C, nC, NBR(C[j]), C[j], nullptr);
        }
        break;
      case 3:  // :126-157
        nA = DIFF(NBR(v0), NBR(v1), kNoUb, A);
        for (int i = 0; i < nA; ++i) {
          nB = DIFF(A, nA, NBR(A[i]), A[i], B);
          for (int j = 0; j < nB; ++j) c += DIFF(B, nB, NBR(B[j]), B[j], nullptr);
        }
        break;
      case 5:  // :219-261
        nA = DIFF(NBR(v0), NBR(v1), kNoUb, A);
        nB = DIFF(NBR(v1), NBR(v0), kNoUb, B);
        nC = ISECT(NBR(v0), NBR(v1), kNoUb, C);
        for (int i = 0; i < nC; ++i) {
          nD = DIFF(A, nA, NBR(C[i]), kNoUb, D);
          nE = DIFF(B, nB, NBR(C[i]), kNoUb, E);
          for (int j = 0; j < nD; ++j) c += DIFF(E, nE, NBR(D[j]), kNoUb, nullptr);
        }
        break;
      case 6:  // :281-318
        nC = ISECT(NBR(v0), NBR(v1), kNoUb, C);
        nB = DIFF(NBR(v1), NBR(v0), kNoUb, B);
        for (int i = 0; i < nC; ++i) {
          nD = DIFF(C, nC, NBR(C[i]), kNoUb, D);
          nE = DIFF(B, nB, NBR(C[i]), kNoUb, E);
          for (int j = 0; j < nD; ++j) c += DIFF(E, nE, NBR(D[j]), kNoUb, nullptr);
        }
        break;
      case 7:  // :339-371
        nC = ISECT(NBR(v0), NBR(v1), kNoUb, C);
        for (int i = 0; i < nC; ++i) {
          nD = DIFF(C, nC, NBR(C[i]), C[i], D);
          for (int j = 0; j < nD; ++j) c += DIFF(D, nD, NBR(D[j]), D[j], nullptr);
        }
        break;
      case 8:  // :394-430
        nC = ISECT(NBR(v0), NBR(v1), kNoUb, C);
        nB = DIFF(NBR(v1), NBR(v0), kNoUb, B);
        for (int i = 0; i < nB; ++i) {
          nD = DIFF(C, nC, NBR(B[i]), kNoUb, D);
          for (int j = 0; j < nD; ++j) c += ISECT(D, nD, NBR(D[j]), D[j], nullptr);
        }
        break;
      default:
        break;
    }
  }
  if (lane == 0 && c) atomicAdd(out, c);
}

// Enumerated count of pattern p in {2,3,5,6,7,8} on the symmetric graph.
int pattern_enumerate(gpm_graph *g, int p, cudaStream_t st, uint64_t *result) {
  GPM_TRY(ensure_src(g, st));
  DevBuf<unsigned long long> d;
  GPM_TRY(d.reserve(1));
  GPM_CUDA(cudaMemsetAsync(d.p, 0, 8, st));
  const int64_t maxd = std::max(1, g->max_deg);
  // scratch: 5 lists of max degree per warp, capped at ~8 GB
  int64_t warps = (int64_t)num_sms() * 4 * 8;
  const int64_t cap_words = (int64_t)2 << 30;
  while (warps > 32 && warps * maxd * 5 > cap_words) warps >>= 1;
  DevBuf<int32_t> scratch;
  GPM_TRY(scratch.reserve((size_t)(warps * maxd * 5)));
  if (g->nnz > 0) {
    k_pattern<<<(int)(warps / 8), 256, 0, st>>>(p, g->nnz, g->off.p, g->adj.p, g->src.p, scratch.p, maxd, d.p);
    GPM_LAUNCH_CHECK();
  }
  unsigned long long h = 0;
  GPM_CUDA(cudaMemcpyAsync(&h, d.p, 8, cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  *result = h;
  return GPM_OK;
}

}  // namespace gpm

using namespace gpm;

extern "C" int gpm_pattern(gpm_graph *g, const char *name, int family, uint64_t *counters, uint64_t *result) {
  if (!g || !name || !result) return fail(GPM_EINVAL, "gpm_pattern: NULL argument");
  if (family != GPM_G2MINER && family != GPM_PATTERN_SOLVER) return fail(GPM_EINVAL, "unknown pattern family");
  if (g->oriented) return fail(GPM_EINVAL, "pattern counting runs on the symmetric (unoriented) graph");
  const std::string nm(name);
  uint64_t h[6] = {0, 0, 0, 0, 0, 0};
  uint64_t res = 0;
  int p = -1;
  if (nm == "Motif4") p = 0;
  else if (nm.size() == 2 && nm[0] == 'P' && nm[1] >= '1' && nm[1] <= '8') p = nm[1] - '0';
  if (p < 0) return fail(GPM_EINVAL, nm + " not support!");  // G2MinerSolver.cuh:157
  uint64_t m4[6];
  if (p == 0 || p == 1 || p == 4) {
    GPM_TRY(gpm_motif(g, 4, m4));
  }
  if (p == 0) {
    for (int i = 0; i < 6; ++i) h[i] = m4[i];
    // G2MinerSolver returns h_total[0]; PatternSolver h_total[1] - h_total[2]
    res = family == GPM_G2MINER ? h[0] : h[1] - h[2];
  } else {
    uint64_t cnt = 0;
    if (p == 1) cnt = m4[0];
    else if (p == 4) cnt = m4[1];
    else GPM_TRY(pattern_enumerate(g, p, 0, &cnt));
    res = cnt;
    // G2Miner accumulates into counters[0]; PatternSolver reports counters[1]
    // (minus the correction it keeps in counters[2], folded in here).
    if (family == GPM_G2MINER) h[0] = cnt;
    else h[1] = cnt;
  }
  if (counters)
    for (int i = 0; i < 6; ++i) counters[i] = h[i];
  *result = res;
  return GPM_OK;
}
