/*
 * gpm_oracle.c -- CPU restatement of the AntiRF count algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker used by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline / --impl reference legs of
 * bench.py.  The CUDA engine never links or calls it.
 *
 * Every set operation below is a merge over sorted, duplicate-free int32
 * lists.  The reference computes the same sets with warp binary searches
 * (src/graph/set_intersection.cuh, src/graph/set_difference.cuh); on sorted
 * unique lists those return exactly:
 *   intersect(a,b)            = a & b
 *   intersect(a,b,ub)         = {x in a & b : x < ub}
 *   difference_set(a,b)       = a - b
 *   difference_set(a,b,ub)    = {x in a - b : x < ub}
 * (the "ub" variants stop at the first warp chunk holding a key >= ub, which
 * on a sorted list drops exactly the keys >= ub).
 */
#include "gpm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UNUSED(x) (void)(x)

static void set_threads(int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  UNUSED(threads);
#endif
}

/* ------------------------------------------------------------------ */
/* sorted-list set algebra                                             */
/* ------------------------------------------------------------------ */
static int64_t s_isect(const int32_t *a, int64_t na, const int32_t *b, int64_t nb,
                       int32_t ub, int32_t *out) {
  int64_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) {
    int32_t x = a[i], y = b[j];
    if (x >= ub || y >= ub) break;
    if (x < y) i++;
    else if (y < x) j++;
    else { if (out) out[k] = x; k++; i++; j++; }
  }
  return k;
}

static int64_t s_diff(const int32_t *a, int64_t na, const int32_t *b, int64_t nb,
                      int32_t ub, int32_t *out) {
  int64_t i = 0, j = 0, k = 0;
  while (i < na) {
    int32_t x = a[i];
    if (x >= ub) break;
    while (j < nb && b[j] < x) j++;
    if (j < nb && b[j] == x) { i++; continue; }
    if (out) out[k] = x;
    k++; i++;
  }
  return k;
}

static int s_has(const int32_t *a, int64_t na, int32_t key) {
  int64_t lo = 0, hi = na - 1;
  while (lo <= hi) {
    int64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] == key) return 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return 0;
}

#define NOUB 0x7fffffff
#define NB(v) (idx + off[v]), (off[(v) + 1] - off[v])

/* ------------------------------------------------------------------ */
/* CSR construction and orientation                                    */
/* ------------------------------------------------------------------ */
static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y);
}

int64_t orc_build_csr(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                      int symmetrize, int64_t *offsets, int32_t *indices, int64_t cap) {
  int64_t cnt = 0, i;
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(m * 2 + 1));
  if (!keys) return -1;
  for (i = 0; i < m; i++) {
    int32_t u = src[i], v = dst[i];
    if (u == v || u < 0 || v < 0 || u >= n || v >= n) continue;
    keys[cnt++] = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
    if (symmetrize) keys[cnt++] = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
  }
  qsort(keys, (size_t)cnt, sizeof(uint64_t), cmp_u64);
  int64_t w = 0;
  for (i = 0; i < cnt; i++)
    if (i == 0 || keys[i] != keys[i - 1]) keys[w++] = keys[i];
  if (w > cap) { free(keys); return -1; }
  memset(offsets, 0, sizeof(int64_t) * (size_t)(n + 1));
  for (i = 0; i < w; i++) {
    offsets[(keys[i] >> 32) + 1]++;
    indices[i] = (int32_t)(keys[i] & 0xffffffffu);
  }
  for (i = 0; i < n; i++) offsets[i + 1] += offsets[i];
  free(keys);
  return w;
}

int64_t orc_orient(int64_t n, const int64_t *off, const int32_t *idx,
                   int64_t *doff, int32_t *didx) {
  int64_t u, k = 0;
  doff[0] = 0;
  for (u = 0; u < n; u++) {
    int64_t du = off[u + 1] - off[u], e;
    for (e = off[u]; e < off[u + 1]; e++) {
      int32_t v = idx[e];
      int64_t dv = off[v + 1] - off[v];
      if (dv > du || (dv == du && v > u)) didx[k++] = v;
    }
    doff[u + 1] = k;
  }
  return k;
}

/* ------------------------------------------------------------------ */
/* triangle counting (src/TCSolver.cuh:40-54)                          */
/* ------------------------------------------------------------------ */
uint64_t orc_tc_merge(int64_t n, const int64_t *doff, const int32_t *didx) {
  const int64_t *off = doff;
  const int32_t *idx = didx;
  uint64_t total = 0;
  int64_t u, e;
  for (u = 0; u < n; u++)
    for (e = off[u]; e < off[u + 1]; e++) {
      int32_t v = idx[e];
      total += (uint64_t)s_isect(NB(u), NB(v), NOUB, NULL);
    }
  return total;
}

uint64_t orc_tc(int64_t n, const int64_t *doff, const int32_t *didx, int threads) {
  uint64_t total = 0;
  set_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int64_t u;
    for (u = 0; u < n; u++) mark[u] = -1;
#pragma omp for schedule(dynamic, 256)
    for (u = 0; u < n; u++) {
      int64_t e, f;
      if (doff[u + 1] - doff[u] < 2) continue;
      for (e = doff[u]; e < doff[u + 1]; e++) mark[didx[e]] = (int32_t)u;
      for (e = doff[u]; e < doff[u + 1]; e++) {
        int32_t v = didx[e];
        for (f = doff[v]; f < doff[v + 1]; f++) total += (mark[didx[f]] == (int32_t)u);
      }
    }
    free(mark);
  }
  return total;
}

/* ------------------------------------------------------------------ */
/* k-clique (src/CFSolver.cuh:15-97)                                   */
/* ------------------------------------------------------------------ */
static uint64_t clique_rec(const int64_t *off, const int32_t *idx, const int32_t *w,
                           int64_t nw, int level, int k, int32_t *buf, int64_t maxd) {
  /* w holds the common DAG out-neighbours of the first `level` vertices. */
  uint64_t c = 0;
  int64_t i;
  if (level == k - 1) return (uint64_t)nw;
  if (level == k - 2) {
    for (i = 0; i < nw; i++) c += (uint64_t)s_isect(w, nw, NB(w[i]), NOUB, NULL);
    return c;
  }
  for (i = 0; i < nw; i++) {
    int64_t nn = s_isect(w, nw, NB(w[i]), NOUB, buf);
    c += clique_rec(off, idx, buf, nn, level + 1, k, buf + maxd, maxd);
  }
  return c;
}

uint64_t orc_clique(int64_t n, const int64_t *doff, const int32_t *didx, int k, int threads) {
  return orc_clique_tasks(n, doff, didx, k, NULL, threads);
}

/* orc_clique over the tasks (first DAG vertices) u with keep[u] != 0, or all
 * of them when keep is NULL: a bounded sample for the CPU baseline. */
uint64_t orc_clique_tasks(int64_t n, const int64_t *doff, const int32_t *didx, int k, const uint8_t *keep,
                          int threads) {
  const int64_t *off = doff;
  const int32_t *idx = didx;
  uint64_t total = 0;
  int64_t maxd = 1, u;
  if (k < 3) return 0;
  for (u = 0; u < n; u++)
    if (off[u + 1] - off[u] > maxd) maxd = off[u + 1] - off[u];
  set_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxd * (k + 1)));
#pragma omp for schedule(dynamic, 64)
    for (u = 0; u < n; u++) {
      int64_t e;
      if (keep && !keep[u]) continue;
      for (e = off[u]; e < off[u + 1]; e++) {
        int32_t v = idx[e];
        /* level-2 list W = N+(u) & N+(v), as clique_4_edge_warp does */
        int64_t nw = s_isect(NB(u), NB(v), NOUB, buf);
        total += clique_rec(off, idx, buf, nw, 2, k, buf + maxd, maxd);
      }
    }
    free(buf);
  }
  return total;
}

/* ------------------------------------------------------------------ */
/* Motif4_G2Miner (src/gpu_kernels/G2Miner_kernels.cuh:438-552)        */
/* ------------------------------------------------------------------ */
static int64_t max_degree(int64_t n, const int64_t *off) {
  int64_t m = 1, u;
  for (u = 0; u < n; u++)
    if (off[u + 1] - off[u] > m) m = off[u + 1] - off[u];
  return m;
}

void orc_motif4_g2miner(int64_t n, const int64_t *off, const int32_t *idx,
                        uint64_t *out, int threads) {
  orc_motif4_tasks(n, off, idx, NULL, out, threads);
}

/* orc_motif4_g2miner over the edge tasks of the vertices v0 with keep[v0] != 0
 * (all when keep is NULL): a bounded sample for the CPU baseline. */
void orc_motif4_tasks(int64_t n, const int64_t *off, const int32_t *idx, const uint8_t *keep,
                      uint64_t *out, int threads) {
  uint64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;
  int64_t maxd = max_degree(n, off), v0;
  set_threads(threads);
#pragma omp parallel reduction(+ : c0, c1, c2, c3, c4, c5)
  {
    int32_t *L0 = (int32_t *)malloc(sizeof(int32_t) * (size_t)maxd);
    int32_t *L1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)maxd);
#pragma omp for schedule(dynamic, 64)
    for (v0 = 0; v0 < n; v0++) {
      int64_t e, i, j;
      if (keep && !keep[v0]) continue;
      for (e = off[v0]; e < off[v0 + 1]; e++) {
        int32_t v1 = idx[e];
        int64_t n0, n1;
        if (v1 == v0) continue;
        /* 3-star: L0 = {x in N(v0)-N(v1) : x < v1}; sum |{y in L0-N(v2): y < v2}| */
        n0 = s_diff(NB(v0), NB(v1), v1, L0);
        for (i = 0; i < n0; i++) c0 += (uint64_t)s_diff(L0, n0, NB(L0[i]), L0[i], NULL);
        if (v1 > v0) continue;
        /* diamond + tailed triangle over W = N(v0) & N(v1) */
        n0 = s_isect(NB(v0), NB(v1), NOUB, L0);
        for (j = 0; j < n0; j++) {
          int32_t v2 = L0[j];
          c4 += (uint64_t)s_diff(L0, n0, NB(v2), v2, NULL);
          n1 = s_diff(NB(v2), NB(v0), NOUB, L1);
          c2 += (uint64_t)s_diff(L1, n1, NB(v1), NOUB, NULL);
        }
        /* 4-clique: {x in N(v0) & N(v1): x < v1}, pairs joined with y < v2 */
        n0 = s_isect(NB(v0), NB(v1), v1, L0);
        for (i = 0; i < n0; i++) c5 += (uint64_t)s_isect(L0, n0, NB(L0[i]), L0[i], NULL);
        /* 4-path: sum over v2 in N(v0)-N(v1) of |(N(v1)-N(v0)) - N(v2)| */
        n0 = s_diff(NB(v0), NB(v1), NOUB, L0);
        n1 = s_diff(NB(v1), NB(v0), NOUB, L1);
        for (j = 0; j < n0; j++) c1 += (uint64_t)s_diff(L1, n1, NB(L0[j]), NOUB, NULL);
        /* 4-cycle: L0 = {x in N(v1)-N(v0): x < v0}, L1 = {x in N(v0)-N(v1): x < v1} */
        n0 = s_diff(NB(v1), NB(v0), (int32_t)v0, L0);
        n1 = s_diff(NB(v0), NB(v1), v1, L1);
        for (j = 0; j < n1; j++) c3 += (uint64_t)s_isect(L0, n0, NB(L1[j]), (int32_t)v0, NULL);
      }
    }
    free(L0);
    free(L1);
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3; out[4] = c4; out[5] = c5;
}

/* ------------------------------------------------------------------ */
/* P1..P8_G2Miner (src/gpu_kernels/G2Miner_kernels.cuh:6-435)          */
/* ------------------------------------------------------------------ */
static uint64_t pattern_edge(const int64_t *off, const int32_t *idx, int p, int32_t v0,
                             int32_t v1, int32_t **L) {
  uint64_t c = 0;
  int64_t nA, nB, nC, nD, nE, i, j;
  int32_t *A = L[0], *B = L[1], *C = L[2], *D = L[3], *E = L[4];
  switch (p) {
    case 1: /* :22-42 */
      if (v1 == v0) break;
      nA = s_diff(NB(v0), NB(v1), v1, A);
      for (i = 0; i < nA; i++) c += (uint64_t)s_diff(A, nA, NB(A[i]), A[i], NULL);
      break;
    case 2: /* :68-103 */
      nA = s_diff(NB(v0), NB(v1), NOUB, A);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      for (i = 0; i < nB; i++) {
        nC = s_diff(A, nA, NB(B[i]), NOUB, C);
        for (j = 0; j < nC; j++) c += (uint64_t)s_diff(C, nC, NB(C[j]), C[j], NULL);
      }
      break;
    case 3: /* :126-157 */
      nA = s_diff(NB(v0), NB(v1), NOUB, A);
      for (i = 0; i < nA; i++) {
        nB = s_diff(A, nA, NB(A[i]), A[i], B);
        for (j = 0; j < nB; j++) c += (uint64_t)s_diff(B, nB, NB(B[j]), B[j], NULL);
      }
      break;
    case 4: /* :174-198 */
      if (v1 >= v0) break;
      nA = s_diff(NB(v0), NB(v1), NOUB, A);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      for (j = 0; j < nA; j++) c += (uint64_t)s_diff(B, nB, NB(A[j]), NOUB, NULL);
      break;
    case 5: /* :219-261 */
      nA = s_diff(NB(v0), NB(v1), NOUB, A);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      nC = s_isect(NB(v0), NB(v1), NOUB, C);
      for (i = 0; i < nC; i++) {
        nD = s_diff(A, nA, NB(C[i]), NOUB, D);
        nE = s_diff(B, nB, NB(C[i]), NOUB, E);
        for (j = 0; j < nD; j++) c += (uint64_t)s_diff(E, nE, NB(D[j]), NOUB, NULL);
      }
      break;
    case 6: /* :281-318 */
      nC = s_isect(NB(v0), NB(v1), NOUB, C);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      for (i = 0; i < nC; i++) {
        nD = s_diff(C, nC, NB(C[i]), NOUB, D);
        nE = s_diff(B, nB, NB(C[i]), NOUB, E);
        for (j = 0; j < nD; j++) c += (uint64_t)s_diff(E, nE, NB(D[j]), NOUB, NULL);
      }
      break;
    case 7: /* :339-371 */
      nC = s_isect(NB(v0), NB(v1), NOUB, C);
      for (i = 0; i < nC; i++) {
        nD = s_diff(C, nC, NB(C[i]), C[i], D);
        for (j = 0; j < nD; j++) c += (uint64_t)s_diff(D, nD, NB(D[j]), D[j], NULL);
      }
      break;
    case 8: /* :394-430 */
      nC = s_isect(NB(v0), NB(v1), NOUB, C);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      for (i = 0; i < nB; i++) {
        nD = s_diff(C, nC, NB(B[i]), NOUB, D);
        for (j = 0; j < nD; j++) c += (uint64_t)s_isect(D, nD, NB(D[j]), D[j], NULL);
      }
      break;
    default:
      break;
  }
  return c;
}

uint64_t orc_pattern_g2miner(int64_t n, const int64_t *off, const int32_t *idx,
                             int p, int threads) {
  uint64_t total = 0;
  int64_t maxd = max_degree(n, off), v0;
  if (p < 1 || p > 8) return 0;
  set_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxd * 5));
    int32_t *L[5];
    int t;
    for (t = 0; t < 5; t++) L[t] = buf + t * maxd;
#pragma omp for schedule(dynamic, 64)
    for (v0 = 0; v0 < n; v0++) {
      int64_t e;
      for (e = off[v0]; e < off[v0 + 1]; e++)
        total += pattern_edge(off, idx, p, (int32_t)v0, idx[e], L);
    }
    free(buf);
  }
  return total;
}

/* ------------------------------------------------------------------ */
/* PatternSolver (src/gpu_kernels/new_edge_warp.cuh)                    */
/* The frequency/correction kernels compute, per edge, a product sum    */
/* minus a correction that equals the G2Miner nested loops; the        */
/* restatement below follows the new_edge_warp.cuh formulas directly.  */
/* ------------------------------------------------------------------ */
static void solver_edge(const int64_t *off, const int32_t *idx, int p, int32_t v0, int32_t v1,
                        int32_t **L, uint64_t *cnt) {
  int64_t nA, nB, nC, nD, i, j, k;
  int32_t *A = L[0], *B = L[1], *D1 = L[2], *D2 = L[3];
  int32_t *F = L[4];
  switch (p) {
    case 2: /* :171-249 */
    case 8: /* :488-566 */ {
      if (p == 2) nA = s_diff(NB(v0), NB(v1), NOUB, A);
      else nA = s_isect(NB(v0), NB(v1), NOUB, A);
      nB = s_diff(NB(v1), NB(v0), NOUB, B);
      for (j = 0; j < nA; j++) {
        F[j] = 0;
        for (i = 0; i < nB; i++) F[j] += !s_has(NB(B[i]), A[j]);
      }
      for (i = 0; i < nA; i++) {
        uint64_t t = p == 2 ? (uint64_t)s_diff(A, nA, NB(A[i]), A[i], NULL)
                            : (uint64_t)s_isect(A, nA, NB(A[i]), A[i], NULL);
        cnt[1] += t * (uint64_t)F[i];
      }
      for (i = 0; i < nB; i++) {
        nC = s_diff(A, nA, NB(B[i]), NOUB, D1);
        nD = s_isect(A, nA, NB(B[i]), NOUB, D2);
        for (k = 0; k < nD; k++)
          for (j = 0; j < nC; j++) {
            int32_t key = D1[j], x = D2[k];
            int adj = s_has(NB(key), x);
            if (key > x && (p == 2 ? !adj : adj)) cnt[2]++;
          }
      }
      break;
    }
    case 3: /* :276-345 */
    case 7: /* :373-452 */ {
      if (p == 3) nA = s_diff(NB(v0), NB(v1), NOUB, A);
      else nA = s_isect(NB(v0), NB(v1), NOUB, A);
      for (j = 0; j < nA; j++) {
        F[j] = 0;
        for (i = j + 1; i < nA; i++) F[j] += !s_has(NB(A[i]), A[j]);
      }
      for (i = 0; i < nA; i++)
        cnt[1] += (uint64_t)s_diff(A, nA, NB(A[i]), A[i], NULL) * (uint64_t)F[i];
      for (i = 0; i < nA; i++) {
        nC = s_diff(A, nA, NB(A[i]), A[i], D1);
        nD = s_isect(A, nA, NB(A[i]), NOUB, D2);
        for (k = 0; k < nD; k++)
          for (j = 0; j < nC; j++)
            if (D1[j] > D2[k] && !s_has(NB(D1[j]), D2[k])) cnt[2]++;
      }
      break;
    }
    default: /* P4, P5, P6: the size-adaptive kernels equal the G2Miner loops */
      cnt[1] += pattern_edge(off, idx, p, v0, v1, L);
      break;
  }
}

uint64_t orc_pattern_solver(int64_t n, const int64_t *off, const int32_t *idx,
                            int p, uint64_t *out, int threads) {
  uint64_t c[6] = {0, 0, 0, 0, 0, 0};
  int64_t maxd = max_degree(n, off), v0;
  int t;
  if (p == 0) {
    /* "Motif4": P1 chain -> sub -> Motif4_edge_warp + P4_edge_warp
     * (src/PatternSolver.cuh:222-240).  Each edge processed once. */
    uint64_t m4[6];
    orc_motif4_g2miner(n, off, idx, m4, threads);
    for (t = 0; t < 6; t++) out[t] = m4[t];
    return m4[1] - m4[2];
  }
  if (p < 1 || p > 8) return 0;
  if (p == 1) {
    /* P1_frequency_count / P1_pair_freq_count / P1_count_correction
     * (new_edge_warp.cuh:18-154): freq(v0,x) = #{v1 in N(v0): v1 > x, x !~ v1}. */
    int64_t e;
    int32_t *freq = (int32_t *)calloc((size_t)(off[n] > 0 ? off[n] : 1), sizeof(int32_t));
    for (v0 = 0; v0 < n; v0++)
      for (e = off[v0]; e < off[v0 + 1]; e++) {
        int32_t v1 = idx[e];
        int64_t f;
        for (f = off[v0]; f < off[v0 + 1]; f++) {
          int32_t key = idx[f];
          if (key < v1 && !s_has(NB(v1), key)) freq[f]++;
        }
      }
    {
      int32_t *A = (int32_t *)malloc(sizeof(int32_t) * (size_t)maxd);
      int32_t *B = (int32_t *)malloc(sizeof(int32_t) * (size_t)maxd);
      for (v0 = 0; v0 < n; v0++)
        for (e = off[v0]; e < off[v0 + 1]; e++) {
          int32_t v2 = idx[e];
          int64_t nA, nB, i, j;
          c[1] += (uint64_t)s_diff(NB(v0), NB(v2), v2, NULL) * (uint64_t)freq[e];
          /* correction for the edge (v0, v1 = v2) */
          nA = s_diff(NB(v0), NB(v2), v2, A);
          nB = s_isect(NB(v0), NB(v2), v2, B);
          for (i = 0; i < nB; i++)
            for (j = 0; j < nA; j++)
              if (A[j] > B[i] && !s_has(NB(A[j]), B[i])) c[2]++;
        }
      free(A);
      free(B);
    }
    free(freq);
  } else {
    set_threads(threads);
    {
      uint64_t c1 = 0, c2 = 0;
#pragma omp parallel reduction(+ : c1, c2)
      {
        int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxd * 5));
        int32_t *L[5];
        uint64_t loc[6] = {0, 0, 0, 0, 0, 0};
        for (t = 0; t < 5; t++) L[t] = buf + t * maxd;
#pragma omp for schedule(dynamic, 64)
        for (v0 = 0; v0 < n; v0++) {
          int64_t e;
          for (e = off[v0]; e < off[v0 + 1]; e++)
            solver_edge(off, idx, p, (int32_t)v0, idx[e], L, loc);
        }
        c1 += loc[1];
        c2 += loc[2];
        free(buf);
      }
      c[1] = c1;
      c[2] = c2;
    }
  }
  for (t = 0; t < 6; t++) out[t] = c[t];
  if (p == 4 || p == 5 || p == 6) return c[1];
  return c[1] - c[2];
}

/* ------------------------------------------------------------------ */
/* brute-force census of connected induced subgraphs (ESU)             */
/* ------------------------------------------------------------------ */
static int adj(const int64_t *off, const int32_t *idx, int32_t a, int32_t b) {
  return s_has(NB(a), b);
}

static void classify(const int64_t *off, const int32_t *idx, const int32_t *s, int k,
                     uint64_t *out) {
  int deg[4] = {0, 0, 0, 0}, e = 0, i, j, maxdeg = 0;
  for (i = 0; i < k; i++)
    for (j = i + 1; j < k; j++)
      if (adj(off, idx, s[i], s[j])) { deg[i]++; deg[j]++; e++; }
  for (i = 0; i < k; i++) if (deg[i] > maxdeg) maxdeg = deg[i];
  if (k == 3) {
    out[e == 3 ? 1 : 0]++;
    return;
  }
  switch (e) {
    case 3: out[2 + (maxdeg == 3 ? 0 : 1)]++; break; /* star / path */
    case 4: out[2 + (maxdeg == 3 ? 2 : 3)]++; break; /* tailed / cycle */
    case 5: out[2 + 4]++; break;
    case 6: out[2 + 5]++; break;
    default: break;
  }
}

static int in_list(const int32_t *a, int n, int32_t x) {
  int i;
  for (i = 0; i < n; i++) if (a[i] == x) return 1;
  return 0;
}

/* ESU: extend sub with vertices > root from the exclusive neighbourhood. */
static void esu_extend(const int64_t *off, const int32_t *idx, int32_t *sub, int ns,
                       int32_t *ext, int ne, int32_t root, int kmax, uint64_t *out) {
  int i;
  if (ns >= 3) classify(off, idx, sub, ns, out);
  if (ns == kmax) return;
  for (i = 0; i < ne; i++) {
    int32_t w = ext[i];
    int32_t next[4096];
    int nn = 0, j;
    int64_t e;
    for (j = i + 1; j < ne && nn < 4096; j++) next[nn++] = ext[j];
    for (e = off[w]; e < off[w + 1]; e++) {
      int32_t u = idx[e];
      int excl = 1;
      if (u <= root || in_list(sub, ns, u) || in_list(next, nn, u) || in_list(ext, ne, u))
        continue;
      for (j = 0; j < ns; j++)
        if (adj(off, idx, sub[j], u)) { excl = 0; break; }
      if (excl && nn < 4096) next[nn++] = u;
    }
    sub[ns] = w;
    esu_extend(off, idx, sub, ns + 1, next, nn, root, kmax, out);
  }
}

void orc_motif_bruteforce(int64_t n, const int64_t *off, const int32_t *idx, uint64_t *out) {
  int64_t v, e;
  int t;
  for (t = 0; t < 8; t++) out[t] = 0;
  for (v = 0; v < n; v++) {
    int32_t sub[4], ext[4096];
    int ne = 0;
    sub[0] = (int32_t)v;
    for (e = off[v]; e < off[v + 1]; e++)
      if (idx[e] > v && ne < 4096) ext[ne++] = idx[e];
    esu_extend(off, idx, sub, 1, ext, ne, (int32_t)v, 4, out);
  }
}

/* ------------------------------------------------------------------ */
/* labelled matching with sub_ceci semantics                           */
/* ------------------------------------------------------------------ */
typedef struct {
  const int64_t *off;
  const int32_t *idx;
  const int32_t *lab;
  int64_t qn;
  const int64_t *qoff;
  const int32_t *qidx;
  const int32_t *qlab;
  int order[64];
  int parent[64];          /* earlier query neighbour used to generate candidates */
  int back[64][64];        /* earlier query neighbours to check */
  int nback[64];
} mctx;

static uint64_t match_rec(const mctx *c, int depth, int32_t *emb) {
  int u = c->order[depth];
  int32_t pv = emb[c->parent[u]];
  int64_t e, qdeg = c->qoff[u + 1] - c->qoff[u];
  uint64_t total = 0;
  for (e = c->off[pv]; e < c->off[pv + 1]; e++) {
    int32_t v = c->idx[e];
    int ok = 1, i;
    if (c->lab[v] != c->qlab[u]) continue;
    if (c->off[v + 1] - c->off[v] < qdeg) continue;
    for (i = 0; i < depth; i++)
      if (emb[c->order[i]] == v) { ok = 0; break; }
    if (!ok) continue;
    for (i = 0; i < c->nback[u]; i++) {
      int32_t w = emb[c->back[u][i]];
      if (!s_has(c->idx + c->off[w], c->off[w + 1] - c->off[w], v)) { ok = 0; break; }
    }
    if (!ok) continue;
    if (depth == c->qn - 1) { total++; continue; }
    emb[u] = v;
    total += match_rec(c, depth + 1, emb);
  }
  return total;
}

uint64_t orc_match(int64_t n, const int64_t *off, const int32_t *idx, const int32_t *labels,
                   int64_t qn, const int64_t *qoff, const int32_t *qidx,
                   const int32_t *qlabels, int threads) {
  mctx c;
  int placed[64];
  int i, j, k;
  int64_t v;
  uint64_t total = 0;
  if (qn <= 0 || qn > 64) return 0;
  memset(&c, 0, sizeof(c));
  c.off = off; c.idx = idx; c.lab = labels;
  c.qn = qn; c.qoff = qoff; c.qidx = qidx; c.qlab = qlabels;
  /* Order: start at the max-degree query vertex, then repeatedly the
   * unplaced vertex with most placed neighbours (ties: higher degree). */
  memset(placed, 0, sizeof(placed));
  {
    int best = 0;
    for (i = 1; i < qn; i++)
      if (qoff[i + 1] - qoff[i] > qoff[best + 1] - qoff[best]) best = i;
    c.order[0] = best;
    placed[best] = 1;
  }
  for (k = 1; k < qn; k++) {
    int best = -1, bs = -1, bd = -1;
    for (i = 0; i < qn; i++) {
      int s = 0;
      int64_t e;
      if (placed[i]) continue;
      for (e = qoff[i]; e < qoff[i + 1]; e++) s += placed[qidx[e]];
      if (s > bs || (s == bs && qoff[i + 1] - qoff[i] > bd)) {
        best = i; bs = s; bd = (int)(qoff[i + 1] - qoff[i]);
      }
    }
    if (bs <= 0) return 0; /* disconnected query: sub_ceci's BFS tree needs connectivity */
    c.order[k] = best;
    placed[best] = 1;
  }
  for (k = 1; k < qn; k++) {
    int u = c.order[k];
    c.parent[u] = -1;
    c.nback[u] = 0;
    for (j = 0; j < k; j++) {
      int w = c.order[j];
      if (s_has(qidx + qoff[u], qoff[u + 1] - qoff[u], w)) {
        if (c.parent[u] < 0) c.parent[u] = w;
        else c.back[u][c.nback[u]++] = w;
      }
    }
  }
  set_threads(threads);
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
  for (v = 0; v < n; v++) {
    int32_t emb[64];
    int u0 = c.order[0];
    if (labels[v] != qlabels[u0]) continue;
    if (off[v + 1] - off[v] < qoff[u0 + 1] - qoff[u0]) continue;
    if (qn == 1) { total++; continue; }
    emb[u0] = (int32_t)v;
    total += match_rec(&c, 1, emb);
  }
  return total;
}

/* Triangle count restricted to the tasks u with keep[u] != 0 (each task
 * still probes the complete lists of its neighbours).  Used to time a
 * bounded sample of a large graph. */
uint64_t orc_tc_tasks(int64_t n, const int64_t *doff, const int32_t *didx, const uint8_t *keep,
                      int threads) {
  uint64_t total = 0;
  set_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int64_t u;
    for (u = 0; u < n; u++) mark[u] = -1;
#pragma omp for schedule(dynamic, 64)
    for (u = 0; u < n; u++) {
      int64_t e, f;
      if (!keep[u] || doff[u + 1] - doff[u] < 2) continue;
      for (e = doff[u]; e < doff[u + 1]; e++) mark[didx[e]] = (int32_t)u;
      for (e = doff[u]; e < doff[u + 1]; e++) {
        int32_t v = didx[e];
        for (f = doff[v]; f < doff[v + 1]; f++) total += (mark[didx[f]] == (int32_t)u);
      }
    }
    free(mark);
  }
  return total;
}

/* Writes a CSR as the Matrix Market coordinate text the reference's loader
 * reads (src/graph/io.h:22-153): a "rows cols entries" line, then one
 * 1-indexed "u v" line per stored entry.  Used to hand the same graph to the
 * reference's own solvers.  Returns the bytes written, -1 on an I/O error. */
static char *put_u64(char *p, uint64_t v) {
  char t[24];
  int k = 0;
  do {
    t[k++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (k) *p++ = t[--k];
  return p;
}

int64_t orc_write_mtx(const char *path, int64_t n, const int64_t *off, const int32_t *idx) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  const size_t cap = (size_t)1 << 22;
  char *buf = (char *)malloc(cap + 64);
  char *p = buf;
  int64_t total = 0, u, e;
  p = put_u64(p, (uint64_t)n);
  *p++ = ' ';
  p = put_u64(p, (uint64_t)n);
  *p++ = ' ';
  p = put_u64(p, (uint64_t)off[n]);
  *p++ = '\n';
  for (u = 0; u < n; u++)
    for (e = off[u]; e < off[u + 1]; e++) {
      p = put_u64(p, (uint64_t)u + 1);
      *p++ = ' ';
      p = put_u64(p, (uint64_t)idx[e] + 1);
      *p++ = '\n';
      if ((size_t)(p - buf) >= cap) {
        if (fwrite(buf, 1, (size_t)(p - buf), f) != (size_t)(p - buf)) total = -1;
        if (total >= 0) total += p - buf;
        p = buf;
      }
    }
  if (p > buf) {
    if (fwrite(buf, 1, (size_t)(p - buf), f) != (size_t)(p - buf)) total = -1;
    if (total >= 0) total += p - buf;
  }
  free(buf);
  if (fclose(f) != 0) total = -1;
  return total;
}

/* Sum over the DAG's triangles u -> v -> w (w in N+(u) & N+(v)) of w[w]:
 * with w = out-degree, the last term of the 4-clique algorithmic byte count
 * (each triangle's pivot list read once).  Marker algorithm, OpenMP. */
uint64_t orc_tc_weighted(int64_t n, const int64_t *doff, const int32_t *didx, const int64_t *wt, int threads) {
  uint64_t total = 0;
  set_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int64_t u;
    for (u = 0; u < n; u++) mark[u] = -1;
#pragma omp for schedule(dynamic, 64)
    for (u = 0; u < n; u++) {
      int64_t e, f;
      if (doff[u + 1] - doff[u] < 2) continue;
      for (e = doff[u]; e < doff[u + 1]; e++) mark[didx[e]] = (int32_t)u;
      for (e = doff[u]; e < doff[u + 1]; e++) {
        int32_t v = didx[e];
        for (f = doff[v]; f < doff[v + 1]; f++)
          if (mark[didx[f]] == (int32_t)u) total += (uint64_t)wt[didx[f]];
      }
    }
    free(mark);
  }
  return total;
}

/* ------------------------------------------------------------------ */
/* seeded synthetic generators                                         */
/* ------------------------------------------------------------------ */
/* The engine draws every synthetic graph from a counter-based generator
 * (splitmix64's finaliser applied to (seed, stream, index)), so edge i of a
 * seed is the same on any thread.  These are the same draws written again in
 * C, so that a harness which must not load the engine -- the CPU reference
 * arm of bench.py, fixture scripts -- builds the very same graphs.  A CPU
 * test checks them against the engine's host generators edge for edge. */
static uint64_t g_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
static uint64_t g_draw(uint64_t seed, uint64_t stream, uint64_t i) {
  return g_mix(g_mix(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ i);
}
static double g_unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t g_below(uint64_t r, uint64_t n) { return (uint32_t)(((r >> 32) * n) >> 32); }

/* R-MAT: edge i descends `scale` levels, level l choosing quadrant a / b / c /
 * d (row bit, column bit) = (0,0) / (0,1) / (1,0) / (1,1) from draw stream 1+l. */
void orc_gen_rmat(int scale, int64_t m, double a, double b, double c, uint64_t seed, int32_t *src,
                  int32_t *dst, int threads) {
  int64_t i;
  const double ab = a + b, abc = a + b + c;
  set_threads(threads);
#pragma omp parallel for schedule(static)
  for (i = 0; i < m; i++) {
    uint32_t x = 0, y = 0;
    int l;
    for (l = 0; l < scale; l++) {
      const double r = g_unit(g_draw(seed, (uint64_t)(1 + l), (uint64_t)i));
      const uint32_t bx = r >= ab, by = (r >= a && r < ab) || r >= abc;
      x = (x << 1) | bx;
      y = (y << 1) | by;
    }
    src[i] = (int32_t)x;
    dst[i] = (int32_t)y;
  }
}

/* Erdos-Renyi G(n, m draws): endpoints uniform from streams 101 and 102. */
void orc_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t *src, int32_t *dst, int threads) {
  int64_t i;
  set_threads(threads);
#pragma omp parallel for schedule(static)
  for (i = 0; i < m; i++) {
    src[i] = (int32_t)g_below(g_draw(seed, 101, (uint64_t)i), (uint64_t)n);
    dst[i] = (int32_t)g_below(g_draw(seed, 102, (uint64_t)i), (uint64_t)n);
  }
}

/* Zipf(s) labels in [0, nlabels): label k with probability (k+1)^-s / H,
 * from draw stream 301 by inverting the cumulative table. */
void orc_gen_zipf_labels(int64_t n, int nlabels, double s, uint64_t seed, int32_t *labels, int threads) {
  double *cdf = (double *)malloc(sizeof(double) * (size_t)(nlabels > 0 ? nlabels : 1));
  double tot = 0, acc = 0;
  int k;
  int64_t i;
  for (k = 0; k < nlabels; k++) tot += 1.0 / pow((double)(k + 1), s);
  for (k = 0; k < nlabels; k++) {
    acc += 1.0 / pow((double)(k + 1), s) / tot;
    cdf[k] = acc;
  }
  cdf[nlabels - 1] = 1.0;
  set_threads(threads);
#pragma omp parallel for schedule(static)
  for (i = 0; i < n; i++) {
    const double r = g_unit(g_draw(seed, 301, (uint64_t)i));
    int j = 0;
    while (j < nlabels - 1 && r >= cdf[j]) j++;
    labels[i] = j;
  }
  free(cdf);
}

/* Writes a symmetric CSR with labels in sub_ceci's "t n m / v id label degree
 * / e u v" format (sub_ceci/graph/graph.cpp:86-166 reads it), each undirected
 * edge once as u < v.  Returns the bytes written, -1 on an I/O error. */
int64_t orc_write_tve(const char *path, int64_t n, const int64_t *off, const int32_t *idx,
                      const int32_t *labels) {
  FILE *f = fopen(path, "wb");
  const size_t cap = (size_t)1 << 22;
  char *buf, *p;
  int64_t total = 0, u, e;
  if (!f) return -1;
  buf = (char *)malloc(cap + 96);
  p = buf;
#define TVE_FLUSH()                                                            \
  if ((size_t)(p - buf) >= cap) {                                              \
    if (fwrite(buf, 1, (size_t)(p - buf), f) != (size_t)(p - buf)) total = -1; \
    if (total >= 0) total += p - buf;                                          \
    p = buf;                                                                   \
  }
  *p++ = 't';
  *p++ = ' ';
  p = put_u64(p, (uint64_t)n);
  *p++ = ' ';
  p = put_u64(p, (uint64_t)(off[n] / 2));
  *p++ = '\n';
  for (u = 0; u < n; u++) {
    *p++ = 'v';
    *p++ = ' ';
    p = put_u64(p, (uint64_t)u);
    *p++ = ' ';
    p = put_u64(p, (uint64_t)labels[u]);
    *p++ = ' ';
    p = put_u64(p, (uint64_t)(off[u + 1] - off[u]));
    *p++ = '\n';
    TVE_FLUSH()
  }
  for (u = 0; u < n; u++)
    for (e = off[u]; e < off[u + 1]; e++) {
      if (idx[e] <= u) continue;
      *p++ = 'e';
      *p++ = ' ';
      p = put_u64(p, (uint64_t)u);
      *p++ = ' ';
      p = put_u64(p, (uint64_t)idx[e]);
      *p++ = '\n';
      TVE_FLUSH()
    }
#undef TVE_FLUSH
  if (p > buf) {
    if (fwrite(buf, 1, (size_t)(p - buf), f) != (size_t)(p - buf)) total = -1;
    if (total >= 0) total += p - buf;
  }
  free(buf);
  if (fclose(f) != 0) total = -1;
  return total;
}

/* Chung-Lu with expected degrees w_i ~ (i + i0)^(-1/(gamma-1)): i0 is the
 * offset at which vertex 0's expected degree equals the structural cut-off
 * sqrt(n * mean_deg) (found by bisection), and each endpoint is drawn by
 * inverting the continuous weight profile's CDF (draw streams 201 / 202);
 * round(n * mean_deg / 2) draws.  Returns that edge count; src may be NULL to
 * ask for it. */
int64_t orc_gen_chung_lu(int64_t n, double gamma, double mean_deg, uint64_t seed, int32_t *src, int32_t *dst,
                         int threads) {
  const int64_t m = llround((double)n * mean_deg / 2.0);
  const double alpha = 1.0 / (gamma - 1.0), a1 = 1.0 - alpha, target = sqrt((double)n * mean_deg);
  double lo = 0.0, hi = (double)n, i0, base, span, inv;
  int it;
  int64_t i;
  if (!src) return m;
  for (it = 0; it < 100; it++) {
    const double mid = 0.5 * (lo + hi);
    const double integral = (pow((double)n + mid, a1) - pow(mid, a1)) / a1;
    const double w0 = mean_deg * (double)n * pow(mid, -alpha) / integral;
    if (w0 > target) lo = mid;
    else hi = mid;
  }
  i0 = 0.5 * (lo + hi);
  if (i0 < 1e-9) i0 = 1e-9;
  base = pow(i0, a1);
  span = pow((double)n + i0, a1) - base;
  inv = 1.0 / a1;
  set_threads(threads);
#pragma omp parallel for schedule(static)
  for (i = 0; i < m; i++) {
    int e;
    for (e = 0; e < 2; e++) {
      const double q = base + g_unit(g_draw(seed, e ? 202 : 201, (uint64_t)i)) * span;
      int64_t k = (int64_t)(pow(q, inv) - i0);
      if (k < 0) k = 0;
      if (k >= n) k = n - 1;
      if (e) dst[i] = (int32_t)k;
      else src[i] = (int32_t)k;
    }
  }
  return m;
}
