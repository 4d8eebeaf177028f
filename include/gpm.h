/*
 * gpm.h -- C ABI of the B200 graph-pattern-mining count engine (libgpm.so).
 *
 * This boundary replaces the header-only template solvers of the AntiRF
 * reference (namespace project_AntiRF).  Each entry point below names the
 * reference interface it stands in for.  Conventions:
 *   - every function returns a gpm_status (0 = GPM_OK); nothing aborts.
 *     gpm_last_error() gives the message of the calling thread's last error;
 *   - host buffers are caller-owned; device memory owned by a handle is
 *     freed by its *_destroy;
 *   - counts are exact uint64 (the reference's AccType, src/utils/utils.h:25);
 *   - neighbour lists are kept sorted ascending and duplicate-free (the
 *     reference's binary searches, src/graph/search.cuh:20-87, are only
 *     defined on such lists);
 *   - "stream" arguments are a cudaStream_t passed as void* (NULL = the
 *     legacy default stream).  Synchronous calls block on that stream;
 *   - a graph handle keeps what its first calls build (the rank-relabelled
 *     copy, task queues and scratch of each count), so repeated counts on it
 *     only launch; calls on one handle from several host threads at once
 *     race on those caches.
 */
#ifndef GPM_H
#define GPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPM_ABI_VERSION 1

typedef enum {
  GPM_OK = 0,
  GPM_EINVAL = 1,       /* bad argument (also: unknown pattern name)          */
  GPM_ECUDA = 2,        /* CUDA runtime error                                 */
  GPM_ENOMEM = 3,       /* device or host allocation failed                   */
  GPM_EUNSUPPORTED = 4, /* request outside what the engine implements         */
  GPM_ETIMEOUT = 5,     /* a device watchdog ended a kernel early             */
  GPM_EIO = 6,          /* file could not be opened or parsed                 */
  GPM_ENODEV = 7        /* no CUDA device                                     */
} gpm_status;

/* src/utils/utils.h:24  enum modes {v_centric, e_centric} */
enum { GPM_V_CENTRIC = 0, GPM_E_CENTRIC = 1 };

/* Triangle-count kernel variants (all return the same count). */
enum {
  GPM_TC_AUTO = 0,     /* engine's default: GPM_TC_BITMAP                              */
  GPM_TC_BSEARCH = 1,  /* warp per stored edge, binary search (TCSolver.cuh:27-59 shape) */
  GPM_TC_HASH = 2,     /* vertex tasks, shared-memory hash of N(u), hub/tail queues
                          with the fixed thresholds of tuning_schedules.cuh:196-197   */
  GPM_TC_MERGE = 3,    /* warp per stored edge, merge-path intersection             */
  GPM_TC_LEARNED = 4,  /* per-task variant and split chosen by the MLP cost model   */
  GPM_TC_BITMAP = 5    /* rank relabel, each edge from its shorter list, shared-memory
                          bitmap membership (the engine's default)                 */
};

/* Pattern families: G2MinerSolver (src/G2MinerSolver.cuh) and PatternSolver
 * (src/PatternSolver.cuh). */
enum { GPM_G2MINER = 0, GPM_PATTERN_SOLVER = 1 };

/* Graph-construction flags for gpm_graph_create. */
enum {
  GPM_SYMMETRIZE = 1  /* add v->u for every u->v (undirected input) */
};

typedef struct gpm_graph gpm_graph;
typedef struct gpm_query gpm_query;
typedef struct gpm_sched gpm_sched;

typedef struct {
  int64_t n;           /* vertices                                  */
  int64_t nnz;         /* stored directed entries                   */
  int32_t max_degree;  /* max stored out-degree                     */
  int32_t oriented;    /* 1 after gpm_graph_orient                   */
  int32_t relabeled;   /* 1 if orient() also relabelled by degree    */
  int32_t has_labels;  /* vertex labels present                      */
} gpm_graph_info;

/* ---- errors / device --------------------------------------------------- */
const char *gpm_last_error(void);
int gpm_abi_version(void);
/* Number of visible CUDA devices (0 when none). */
int gpm_device_count(int *count);

/* ---- file formats (host only, no device needed) ------------------------- */
/* Loader::_load_mtx, src/graph/io.h:84-139: skip lines until one starts with
 * a digit, read the "n n m" header, then integers in pairs (the rest of the
 * second one's line ignored; a last line without a newline is not read),
 * drop self-loops, shift ids by the minimum id.  Parsed on all host threads
 * (line-parallel, with the exact sequential reading for irregular files).
 * Two-call pattern: with src == NULL only *n and *m are returned (the parse
 * is kept for the second call of the same thread).  *vmin receives the id
 * shift (needed by gpm_read_labels). */
int gpm_read_mtx(const char *path, int64_t *n, int64_t *m, int32_t *src, int32_t *dst,
                 int64_t cap, int32_t *vmin);
/* Binary CSR in the layout the reference's converter writes
 * (scripts/gbin_reader/greader.h:229-268; Loader::Load(..., "bin") is
 * declared there but not implemented, io.h:143): <prefix>/graph.vertex.bin
 * (int64 offsets, n+1), <prefix>/graph.edge.bin (int32 ids, nnz),
 * <prefix>/graph.meta.txt ("n", "nnz", "4", "max degree").  Two-call pattern:
 * with offsets == indices == NULL only the sizes (and *max_degree, may be
 * NULL) are returned.  The arrays are checked (sizes, monotone offsets, ids in
 * range) and returned as stored. */
int gpm_read_gbin(const char *prefix, int64_t *n, int64_t *nnz, int64_t *offsets, int32_t *indices,
                  int32_t *max_degree);
/* Writes a CSR in that layout (creates the directory when missing). */
int gpm_write_gbin(const char *prefix, int64_t n, const int64_t *offsets, const int32_t *indices);
/* The reference converter (greader.cpp / greader.h:129-268) with its rules:
 * "n n nnz" header, then each line split at single spaces and kept when it
 * has exactly two tokens; self-loops kept; ids shifted by the minimum id;
 * lists in file order. */
int gpm_convert_mtx_gbin(const char *mtx_path, const char *prefix);
/* Loader::LoadVLabel, src/graph/io.h:35-73: "v label" lines (v shifted by
 * vmin) or the literal "random<N>" (labels rand() % N with the C library's
 * rand(), as the reference does). */
int gpm_read_labels(const char *path, int64_t n, int32_t vmin, int32_t *labels);
/* sub_ceci Graph::loadGraphFromFile (sub_ceci/graph/graph.cpp:86-166) "t/v/e"
 * format, and the querysets "t # 0 / v id label / e u v elabel" format.
 * Two-call pattern as above.  Edges are returned as listed (once each). */
int gpm_read_tve(const char *path, int64_t *n, int64_t *m, int32_t *labels, int32_t *src,
                 int32_t *dst, int64_t cap);

/* ---- seeded synthetic generators (host, OpenMP; identical on device) ------ */
/* R-MAT: scale, edge_factor * 2^scale draws, quadrant probabilities a,b,c. */
int gpm_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                 int32_t *src, int32_t *dst);
/* Erdos-Renyi G(n, m draws): uniform endpoints. */
int gpm_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t *src, int32_t *dst);
/* Chung-Lu: expected degrees w_i ~ (i+i0)^(-1/(gamma-1)) scaled to mean
 * degree mean_deg; m = round(n * mean_deg / 2) draws. Returns *m first when
 * src == NULL. */
int gpm_gen_chung_lu(int64_t n, double gamma, double mean_deg, uint64_t seed, int64_t *m,
                     int32_t *src, int32_t *dst);
/* Zipf(s) labels in [0, nlabels). */
int gpm_gen_zipf_labels(int64_t n, int nlabels, double s, uint64_t seed, int32_t *labels);

/* ---- graphs ---------------------------------------------------------------- */
/* Loader::Build + Graph::Init (src/graph/io.h:75-81, src/graph/graph.h:254-340):
 * builds the device CSR from a host edge list.  Self-loops and duplicate
 * entries are dropped and every list is sorted (Init keeps input order; the
 * reference kernels need sorted lists).  labels may be NULL. */
int gpm_graph_create(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                     const int32_t *labels, int flags, gpm_graph **out);
/* Same, from a host CSR that is already sorted and duplicate-free
 * (offsets[n+1], indices[offsets[n]]). Validated on the device. */
int gpm_graph_create_csr(int64_t n, const int64_t *offsets, const int32_t *indices,
                         const int32_t *labels, gpm_graph **out);
/* Build a graph whose edge list already lives in device memory. */
int gpm_graph_create_device(int64_t n, int64_t m, const int32_t *d_src, const int32_t *d_dst,
                            int flags, gpm_graph **out);
/* Seeded R-MAT / ER / Chung-Lu graph generated and built on the device
 * (symmetrised, simple).  kind: 0 = R-MAT(p0=scale, p1=edge factor, a,b,c),
 * 1 = ER(p0=n, p1=m draws), 2 = Chung-Lu(p0=n, a=gamma, b=mean degree). */
int gpm_graph_generate(int kind, int64_t p0, int64_t p1, double a, double b, double c,
                       uint64_t seed, gpm_graph **out);
int gpm_graph_destroy(gpm_graph *g);
int gpm_graph_get_info(const gpm_graph *g, gpm_graph_info *info);
/* Copy the device CSR to caller buffers (offsets[n+1], indices[nnz]). */
int gpm_graph_copy_csr(const gpm_graph *g, int64_t *offsets, int32_t *indices);
int gpm_graph_set_labels(gpm_graph *g, const int32_t *labels);
/* Graph::orientation (graph.h:116-204): keep u->v iff d(v) > d(u) or
 * (d(v) == d(u) and v > u).  relabel != 0 additionally applies
 * Graph::SortCSRGraph (graph.h:206-252): vertices renumbered by out-degree
 * descending (stable), lists re-sorted.  Runs on the device. */
int gpm_graph_orient(gpm_graph *g, int relabel);
/* Graph::SortCSRGraph (graph.h:206-252) alone, on the current lists. */
int gpm_graph_relabel(gpm_graph *g);
/* Frees what earlier counts cached with g (the rank-relabelled copy, task
 * queues, pipelines, label partition), keeping the graph itself; the next
 * count builds them again.  No reference counterpart: the reference keeps no
 * schedules between calls (and leaks its scratch, src/TCSolver.cuh:72,105). */
int gpm_graph_drop_plans(gpm_graph *g);
/* Algorithmic work figures of the (oriented) graph: *wedge_work =
 * sum over stored u->v of deg(v); *pair_work = sum over u->v of
 * (deg(u) + deg(v)). */
int gpm_graph_work(gpm_graph *g, uint64_t *wedge_work, uint64_t *pair_work);

/* ---- counting ---------------------------------------------------------------- */
/* TCSolver (src/TCSolver.cuh:9-121): sum over stored edges u->v of
 * |N(u) & N(v)|.  On an oriented graph this is the triangle count (the
 * reference's Engine::RunTC orients first, src/Engine.h:47-56).
 * mode: GPM_V_CENTRIC / GPM_E_CENTRIC choose the default variant
 * (GPM_TC_HASH / GPM_TC_BSEARCH) when variant == GPM_TC_AUTO and no trained
 * scheduler is attached. */
int gpm_tc(gpm_graph *g, int mode, uint64_t *out);
/* Explicit variant, asynchronous: writes the count to device memory d_out
 * (8 bytes) on stream; no host synchronisation; capturable. */
int gpm_tc_async(gpm_graph *g, int variant, void *stream, uint64_t *d_out);
/* End to end from host memory: upload a symmetric CSR (sorted,
 * duplicate-free), orient on the device, count, return the count.  This is
 * the RunTC path as one call.  stream may be NULL. */
int gpm_tc_host_csr(int64_t n, const int64_t *offsets, const int32_t *indices, int variant,
                    void *stream, uint64_t *out);
/* Work of GPM_TC_BITMAP's fixed plan on g (built if needed), no reference
 * counterpart: stats[0] partner segments, stats[1] keys streamed from the
 * segments read as keys, stats[2] keys of the owner lists loaded into shared
 * memory, stats[3] owner tasks, stats[4] dense segments (read as 32-bit
 * words of a core bitmap row), stats[5] the words ANDed for them.  stats
 * holds 6 entries. */
int gpm_tc_plan_stats(gpm_graph *g, uint64_t *stats);

/* Triangle count of a device-resident CSR that allocates nothing -- this
 * entry point has no counterpart in the reference.  It serves callers that
 * cannot call cudaMalloc (a framework owning all device memory through its
 * own pool, services that forbid allocation after start-up, code that must
 * avoid the implicit synchronisation of allocation).  d_offsets[n+1] (int64)
 * and d_indices (int32, sorted lists, every id < n) are the caller's device
 * arrays, nothing of them is checked (ids outside [0, n) read out of bounds);
 * the count (sum over stored u->v of |N(u) & N(v)|, the triangle count when
 * the CSR is a degree-oriented DAG, which the caller orients) is written to the caller's device uint64 d_out on
 * `stream` without host synchronisation.  Scratch lives in a fixed 8 MiB
 * array inside the library: at most 1,048,576 vertices (larger n is
 * rejected with GPM_EINVAL); calls that overlap on the GPU race on that
 * array; the first call on a device sets it up, so make it before any
 * stream capture. */
int gpm_tc_csr_noalloc(int64_t n, const int64_t *d_offsets, const int32_t *d_indices, void *stream,
                       uint64_t *d_out);

/* CFSolver (src/CFSolver.cuh:99-158): k-clique count on an oriented graph,
 * k in [3, 8]. */
int gpm_clique(gpm_graph *g, int k, uint64_t *out);
/* Same with an explicit kernel: GPM_CLIQUE_AUTO (local bitset DAG per vertex
 * when the graph is a degree-oriented DAG) or GPM_CLIQUE_EDGE (warp per
 * stored edge with materialised intersections, the shape of
 * clique_4_edge_warp / clique_5_edge_warp). */
enum { GPM_CLIQUE_AUTO = 0, GPM_CLIQUE_EDGE = 1 };
int gpm_clique_ex(gpm_graph *g, int k, int variant, uint64_t *out);

/* Motif counting on a symmetric graph.  k = 3: out[0] = induced 2-paths,
 * out[1] = triangles.  k = 4: out[0..5] = 3-star, 4-path, tailed triangle,
 * 4-cycle, diamond, 4-clique -- the counter order of Motif4_G2Miner
 * (src/gpu_kernels/G2Miner_kernels.cuh:473-548).  The first call of each k
 * builds the pipeline's task queues and scratch and keeps them with g. */
int gpm_motif(gpm_graph *g, int k, uint64_t *out);

/* G2MinerSolver / PatternSolver (src/G2MinerSolver.cuh:17-176,
 * src/PatternSolver.cuh:16-265) on a symmetric graph.  name: "P1".."P8" or
 * "Motif4".  counters (may be NULL) receive the solver's 6-entry counter
 * array; *result the value the solver returns (h_total[0] for G2Miner,
 * h_total[1] or h_total[1]-h_total[2] for PatternSolver). */
int gpm_pattern(gpm_graph *g, const char *name, int family, uint64_t *counters,
                uint64_t *result);

/* ---- learned task scheduler (no reference counterpart; replaces the fixed
 * thresholds USE_CTA / USE_WARP of src/gpu_kernels/tuning_schedules.cuh:196-197,
 * which remain the default schedule and the yardstick of its regret) --------
 * Each owner task of GPM_TC_BITMAP gets one of 6 configurations:
 * queue (cfg / 3: 0 warp, 1 CTA) x long-segment threshold ({16, 64, 256}[cfg % 3]).
 * A 3-layer FP32 MLP (8 -> 32 -> 32 -> 6) predicts log2 active warp-cycles of
 * each configuration from 8 task features; a task takes its cheapest one
 * (owners above the fixed schedule's CTA threshold choose among the CTA
 * configurations only), except that a warp-queue task predicted to cost more than half a warp
 * slot's share of the total takes its cheapest CTA configuration.  Counts
 * never depend on the choice. */
int gpm_sched_create(uint64_t seed, gpm_sched **out);
int gpm_sched_destroy(gpm_sched *s);
int gpm_sched_param_count(void);
int gpm_sched_get_params(const gpm_sched *s, float *params);
int gpm_sched_set_params(gpm_sched *s, const float *params);
/* Runs every owner task of g (oriented) under the 6 configurations with the
 * instrumented kernel and appends (features, log2 cost) rows to s. */
int gpm_sched_collect(gpm_sched *s, gpm_graph *g, int64_t *rows_added);
/* Copies the dataset out (X: rows x 8, Y: rows x 6); NULL buffers: count only. */
int gpm_sched_dataset(const gpm_sched *s, int64_t *rows, float *X, float *Y);
/* Mean squared error over finite targets and its gradient (host arrays). */
int gpm_sched_grad(gpm_sched *s, int64_t N, const float *X, const float *T, float *grad, double *loss);
int gpm_sched_predict(gpm_sched *s, int64_t N, const float *X, float *Y);
/* Full-batch Adam steps on the collected dataset, trained on the device. */
int gpm_sched_train(gpm_sched *s, int steps, float lr, double *final_loss);
/* GPM_TC_LEARNED on g uses s from now on; a destroyed scheduler is detected
 * (GPM_EINVAL) instead of used. */
int gpm_sched_attach(gpm_graph *g, gpm_sched *s);
/* Scheduler used by GPM_TC_LEARNED on graphs without an attached one,
 * including the temporary graph of gpm_tc_host_csr (NULL clears it;
 * destroying the default clears it too). */
int gpm_sched_set_default(gpm_sched *s);
/* The configuration the scheduler gives each vertex's task (255: no task). */
int gpm_sched_assign(gpm_sched *s, gpm_graph *g, uint8_t *cfg);
/* The logged cost (active warp-cycles) of every owner task of g under each
 * of the 6 configurations: cost[6 * v + c] (host, 6 * n floats; 0 for
 * vertices that own no task).  The instrumented runs behind the training data
 * of gpm_sched_collect, per vertex. */
int gpm_tc_task_costs(gpm_graph *g, float *cost);
/* Fixes the per-owner configuration GPM_TC_LEARNED runs on g (host cfg[v] in
 * 0..5, one byte per vertex), e.g. the per-task optimum of gpm_tc_task_costs:
 * it replaces the scheduler's choice until the graph's plans are dropped. */
int gpm_tc_set_schedule(gpm_graph *g, const uint8_t *cfg);

/* ---- batches of graphs (no reference counterpart: the reference runs one
 * solver per graph and synchronises after every kernel,
 * src/PatternSolver.cuh:177-246) ---------------------------------------------- */
typedef struct gpm_batch gpm_batch;
/* Many symmetric graphs held as one device-resident disjoint union.  Member g
 * has n[g] vertices and m[g] undirected edges; src/dst hold all members'
 * edges back to back with member-local ids. */
int gpm_batch_create(int ngraphs, const int64_t *n, const int64_t *m, const int32_t *src, const int32_t *dst,
                     gpm_batch **out);
/* Seeded Chung-Lu members generated on the device (member g uses seed
 * mix(seed + g), n[g] vertices, exponent gamma[g], mean degree mean_deg[g]). */
int gpm_batch_generate_chung_lu(int ngraphs, const int64_t *n, const double *gamma, const double *mean_deg,
                                uint64_t seed, gpm_batch **out);
int gpm_batch_info(const gpm_batch *b, int *ngraphs, int64_t *n_total, int64_t *nnz_total);
/* Member g's symmetric CSR (member-local ids); two-call pattern on NULL buffers. */
int gpm_batch_member_csr(const gpm_batch *b, int g, int64_t *offsets, int32_t *indices, int64_t *n, int64_t *nnz);
/* Chooses the pipeline's three task-split thresholds for this batch by
 * timing candidates; tuned[3] (may be NULL) receives them. */
int gpm_batch_autotune(gpm_batch *b, int *tuned);
/* Device time of the pipeline's three heavy stages run alone: ms[0] triangles
 * per edge, ms[1] 4-cycles, ms[2] 4-cliques (CUDA events). */
int gpm_batch_stage_ms(gpm_batch *b, float *ms);
/* 3- and 4-vertex motifs of every member: out[8*g + i], i as in gpm_motif
 * (0..1: induced 2-paths, triangles; 2..7: 3-star, 4-path, tailed triangle,
 * 4-cycle, diamond, 4-clique).  One launch per pipeline stage covers all
 * members; use_graph != 0 captures the stages into a CUDA graph on the first
 * call and replays it afterwards. */
int gpm_batch_motif(gpm_batch *b, int use_graph, void *stream, uint64_t *out);
/* The same into device memory d_out (8 * ngraphs uint64) without host
 * synchronisation; needs one gpm_batch_motif call before. */
int gpm_batch_motif_async(gpm_batch *b, int use_graph, void *stream, uint64_t *d_out);
int gpm_batch_destroy(gpm_batch *b);

/* ---- labelled subgraph matching (sub_ceci semantics) ----------------------- */
/* Query graph: n vertices (1 <= n <= 64, sub_ceci's MAX_QUERY_VERTEX in
 * sub_ceci/configuration/config.h:12), m undirected edges listed once,
 * labels.  n > 64 fails with GPM_EUNSUPPORTED. */
int gpm_query_create(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                     const int32_t *labels, gpm_query **out);
int gpm_query_destroy(gpm_query *q);
/* Number of injective, label-preserving maps of the query into the data
 * graph that send every query edge to a data edge (sub_ceci/myceci.cpp:540-668
 * counts the same embeddings).  The data graph must be symmetric and carry
 * labels. */
int gpm_match(gpm_graph *data, const gpm_query *q, uint64_t *out);
/* sub_ceci's -num N (myceci.cpp:1021-1027, 615-617): enumeration stops once
 * `limit` embeddings are found; *out = min(total, limit). */
int gpm_match_limit(gpm_graph *data, const gpm_query *q, uint64_t limit, uint64_t *out);
/* Embedding listing (no reference counterpart: sub_ceci counts and never
 * prints its embeddings): up to `limit` embeddings into emb (host, limit * n
 * int32), each the n data-vertex ids of query vertices 0..n-1; *written =
 * min(total, limit).  All embeddings when total <= limit, otherwise an
 * arbitrary `limit` of them. */
int gpm_match_list(gpm_graph *data, const gpm_query *q, uint64_t limit, int32_t *emb, uint64_t *written);

/* ---- batches of labelled queries (no reference counterpart: the reference
 * launches one kernel per pattern and synchronises after each,
 * src/PatternSolver.cuh:177-246) ------------------------------------------- */
typedef struct gpm_match_batch gpm_match_batch;
/* nq queries on one labelled symmetric data graph, counted together in one
 * persistent launch (sub_ceci semantics, as gpm_match).  member (host, n ids
 * in [0, nmembers), may be NULL) names each vertex's member when the data
 * graph is a disjoint union of many graphs: each embedding is counted for its
 * root's member.  The plan (each query's (root, second vertex) tasks,
 * extended breadth first to longer partial embeddings where they are too few
 * to fill the GPU) is built here; `data` must outlive the batch. */
int gpm_match_batch_create(gpm_graph *data, int nq, const gpm_query *const *queries, const int32_t *member,
                           int nmembers, gpm_match_batch **out);
/* Chooses how finely tasks of queries with 4 or more vertices are split (the
 * span of candidates of a task's first unmapped position per task; 0 =
 * unsplit) by timing candidates; *span (may be NULL) receives it. */
int gpm_match_batch_autotune(gpm_match_batch *b, int64_t *span);
/* Counts: out[q * nmembers + m] (host, nq * nmembers uint64, nmembers = 1
 * without member ids).  use_graph != 0 captures the launch into a CUDA graph
 * on the first call and replays it afterwards. */
int gpm_match_batch_run(gpm_match_batch *b, int use_graph, void *stream, uint64_t *out);
/* The same into device memory d_out without host synchronisation. */
int gpm_match_batch_run_async(gpm_match_batch *b, int use_graph, void *stream, uint64_t *d_out);
/* Tasks in the launch and the current split span. */
int gpm_match_batch_info(const gpm_match_batch *b, int64_t *tasks, int64_t *span);
int gpm_match_batch_destroy(gpm_match_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* GPM_H */
