/*
 * gpm_oracle.h -- CPU restatement of the AntiRF (GPM-lib/GPM-artifact) count
 * algorithms.  TEST INFRASTRUCTURE ONLY: this library is the checker that the
 * parity tests, the smoke check and the CPU-baseline leg of bench.py compare
 * the CUDA engine against.  No product code path links, loads or calls it.
 *
 * All graphs are CSR with int64 offsets and int32 neighbour ids, every list
 * sorted ascending without duplicates (the reference's binary searches are
 * only defined on such lists, src/graph/search.cuh:20-87).
 *
 * Parity pins: the labelled matcher is pinned by the 200 HPRD known-answer
 * tests shipped with sub_ceci (sub_ceci/test/expected_output.res); the
 * unlabelled counters are pinned by an independent brute-force enumerator
 * (orc_motif_bruteforce) and by the hand-checked fixtures in tests/golden.
 */
#ifndef GPM_ORACLE_H
#define GPM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Symmetric, deduplicated, self-loop-free CSR from a directed edge list.
 * Returns the number of stored (directed) entries, or -1 if cap is too small. */
int64_t orc_build_csr(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                      int symmetrize, int64_t *offsets, int32_t *indices, int64_t cap);

/* Degree orientation, src/graph/graph.h:116-204: keep u->v iff d(v)>d(u) or
 * (d(v)==d(u) and v>u).  Output lists stay sorted.  Returns m+. */
int64_t orc_orient(int64_t n, const int64_t *off, const int32_t *idx,
                   int64_t *doff, int32_t *didx);

/* Triangle count on the oriented DAG, src/TCSolver.cuh:40-54 (sum over DAG
 * edges of |N+(v) & N+(u)|).  orc_tc uses a per-thread marker array and
 * OpenMP; orc_tc_merge is the single-thread merge restatement. */
uint64_t orc_tc(int64_t n, const int64_t *doff, const int32_t *didx, int threads);
uint64_t orc_tc_merge(int64_t n, const int64_t *doff, const int32_t *didx);
/* orc_tc restricted to the tasks u with keep[u] != 0 (bounded CPU samples). */
uint64_t orc_tc_tasks(int64_t n, const int64_t *doff, const int32_t *didx, const uint8_t *keep,
                      int threads);

/* k-clique count on the DAG, src/CFSolver.cuh:15-97 (k=4,5) generalised to
 * any k>=3 by the same nested materialised intersections. */
uint64_t orc_clique(int64_t n, const int64_t *doff, const int32_t *didx, int k, int threads);
/* orc_clique restricted to the first-vertex tasks u with keep[u] != 0. */
uint64_t orc_clique_tasks(int64_t n, const int64_t *doff, const int32_t *didx, int k, const uint8_t *keep,
                          int threads);

/* Motif4_G2Miner restatement, src/gpu_kernels/G2Miner_kernels.cuh:438-552, on
 * the symmetric graph.  out[0..5] = 3-star, 4-path, tailed triangle, 4-cycle,
 * diamond, 4-clique. */
void orc_motif4_g2miner(int64_t n, const int64_t *off, const int32_t *idx,
                        uint64_t *out, int threads);
/* orc_motif4_g2miner restricted to the edge tasks of vertices with keep[v] != 0. */
void orc_motif4_tasks(int64_t n, const int64_t *off, const int32_t *idx, const uint8_t *keep,
                      uint64_t *out, int threads);

/* P1..P8_G2Miner restatements, src/gpu_kernels/G2Miner_kernels.cuh:6-435. */
uint64_t orc_pattern_g2miner(int64_t n, const int64_t *off, const int32_t *idx,
                             int p, int threads);

/* PatternSolver restatements (src/gpu_kernels/new_edge_warp.cuh), each edge
 * processed once.  out[] receives the solver's counter array (6 entries);
 * the function returns the value PatternSolver reports
 * (src/PatternSolver.cuh:250-254). */
uint64_t orc_pattern_solver(int64_t n, const int64_t *off, const int32_t *idx,
                            int p, uint64_t *out, int threads);

/* Brute-force connected induced subgraph census (ESU enumeration), small
 * graphs only.  out[0..1] = 3-vertex path, triangle; out[2..7] = the six
 * 4-vertex motifs in the orc_motif4_g2miner order. */
void orc_motif_bruteforce(int64_t n, const int64_t *off, const int32_t *idx, uint64_t *out);

/* Labelled subgraph matching with sub_ceci semantics
 * (sub_ceci/myceci.cpp:540-668): the number of injective, label-preserving
 * maps of the query vertices into the data graph that map every query edge to
 * a data edge (non-induced; automorphic images counted separately). */
/* Sum over DAG triangles u -> v -> w of wt[w] (with wt = out-degree: the
 * last term of the 4-clique algorithmic byte count). */
uint64_t orc_tc_weighted(int64_t n, const int64_t *doff, const int32_t *didx, const int64_t *wt, int threads);

/* The CSR as 1-indexed Matrix Market coordinate text (the reference
 * loader's input, src/graph/io.h:22-153); bytes written or -1. */
int64_t orc_write_mtx(const char *path, int64_t n, const int64_t *off, const int32_t *idx);

uint64_t orc_match(int64_t n, const int64_t *off, const int32_t *idx, const int32_t *labels,
                   int64_t qn, const int64_t *qoff, const int32_t *qidx,
                   const int32_t *qlabels, int threads);

/* Seeded synthetic generators: the engine's own draws (splitmix64 finaliser
 * over (seed, stream, index)) written again here, so that harnesses which
 * must not load the engine build the same graphs.  R-MAT: m edges of
 * 2^scale vertices, quadrant probabilities a, b, c; ER: m uniform draws;
 * labels: Zipf(s) over [0, nlabels). */
void orc_gen_rmat(int scale, int64_t m, double a, double b, double c, uint64_t seed, int32_t *src,
                  int32_t *dst, int threads);
void orc_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t *src, int32_t *dst, int threads);
int64_t orc_gen_chung_lu(int64_t n, double gamma, double mean_deg, uint64_t seed, int32_t *src, int32_t *dst,
                         int threads);
void orc_gen_zipf_labels(int64_t n, int nlabels, double s, uint64_t seed, int32_t *labels, int threads);

/* A symmetric labelled CSR as sub_ceci's "t/v/e" text (each undirected edge
 * once, u < v); bytes written or -1. */
int64_t orc_write_tve(const char *path, int64_t n, const int64_t *off, const int32_t *idx,
                      const int32_t *labels);

#ifdef __cplusplus
}
#endif
#endif
