// common.cuh -- shared definitions of libgpm: status/error plumbing, the
// device graph handle, a counter-based RNG usable on host and device, and
// warp helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "gpm.h"

namespace gpm {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);

#define GPM_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      return ::gpm::fail(e_ == cudaErrorMemoryAllocation ? GPM_ENOMEM : GPM_ECUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));   \
    }                                                                           \
  } while (0)

#define GPM_TRY(expr)            \
  do {                           \
    int s_ = (expr);             \
    if (s_ != GPM_OK) return s_; \
  } while (0)

// Checks that a launch was accepted (configuration errors); execution errors
// surface at the next synchronising call.
#define GPM_LAUNCH_CHECK() GPM_CUDA(cudaGetLastError())

int ensure_device();

// ---------------------------------------------------------------- device buffers
// A per-thread pool of device blocks kept across calls.  While an ArenaScope
// is alive on a thread, DevBuf allocations of that thread come from the pool
// and go back to it when freed, so a repeated one-shot call (upload, prepare,
// count, download) performs no cudaMalloc/cudaFree after the first.  Only
// entry points that run all their work on one stream and synchronise it
// before returning open a scope, so a block is never reused while an earlier
// kernel still reads it.
struct Arena;
Arena *current_arena();
void *arena_get(Arena *a, size_t bytes, size_t *cap);
void arena_put(Arena *a, void *p, size_t cap);
struct ArenaScope {
  ArenaScope();
  ~ArenaScope();
  Arena *prev;
};

// Owning device allocation; move-only.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  Arena *arena = nullptr;  // pool the block came from (nullptr: cudaMalloc)
  size_t cap = 0;          // bytes of a pooled block
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), arena(o.arena), cap(o.cap) {
    o.p = nullptr;
    o.n = 0;
    o.arena = nullptr;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      arena = o.arena;
      cap = o.cap;
      o.p = nullptr;
      o.n = 0;
      o.arena = nullptr;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p) {
      if (arena) arena_put(arena, p, cap);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
    arena = nullptr;
  }
  // Grows to at least count elements (contents not preserved).
  int reserve(size_t count) {
    if (count <= n && p) return GPM_OK;
    reset();
    size_t bytes = (count ? count : 1) * sizeof(T);
    if (Arena *a = current_arena()) {
      p = static_cast<T *>(arena_get(a, bytes, &cap));
      if (!p) return fail(GPM_ENOMEM, "device pool allocation of " + std::to_string(bytes) + " B failed");
      arena = a;
      n = count ? count : 1;
      return GPM_OK;
    }
    cudaError_t e = cudaMalloc((void **)&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(GPM_ENOMEM, "cudaMalloc(" + std::to_string(bytes) + " B) failed: " +
                                  cudaGetErrorString(e));
    }
    n = count ? count : 1;
    return GPM_OK;
  }
};

// ---------------------------------------------------------------- RNG
// splitmix64 finaliser: a counter-based generator, so edge i of a seeded
// graph is the same whichever thread (host or device) draws it.
__host__ __device__ inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__host__ __device__ inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ i);
}
__host__ __device__ inline double unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }
// uniform integer in [0, n) for n < 2^32
__host__ __device__ inline uint32_t below(uint64_t r, uint64_t n) {
  return (uint32_t)(((r >> 32) * n) >> 32);
}

// R-MAT edge i: one quadrant draw per bit level, standard recursion.
__host__ __device__ inline void rmat_edge(uint64_t seed, uint64_t i, int scale, double a, double b,
                                          double c, int32_t *u, int32_t *v) {
  uint32_t x = 0, y = 0;
  const double ab = a + b, abc = a + b + c;
  for (int l = 0; l < scale; ++l) {
    double r = unit(draw(seed, 1 + l, i));
    uint32_t bx = 0, by = 0;
    if (r < a) {
    } else if (r < ab) {
      by = 1;
    } else if (r < abc) {
      bx = 1;
    } else {
      bx = 1;
      by = 1;
    }
    x = (x << 1) | bx;
    y = (y << 1) | by;
  }
  *u = (int32_t)x;
  *v = (int32_t)y;
}

__host__ __device__ inline void er_edge(uint64_t seed, uint64_t i, int64_t n, int32_t *u, int32_t *v) {
  *u = (int32_t)below(draw(seed, 101, i), (uint64_t)n);
  *v = (int32_t)below(draw(seed, 102, i), (uint64_t)n);
}

// Chung-Lu endpoint: vertex index drawn with weight (i + i0)^(-alpha) by
// inverting the continuous CDF of the weight profile.
struct ChungLu {
  double alpha, i0, lo, span, inv;  // lo = i0^(1-alpha), span = (n+i0)^(1-alpha) - lo
  int64_t n;
};
__host__ __device__ inline int32_t chung_lu_vertex(const ChungLu &p, uint64_t r) {
  double q = p.lo + unit(r) * p.span;
  double x = pow(q, p.inv) - p.i0;
  int64_t k = (int64_t)x;
  if (k < 0) k = 0;
  if (k >= p.n) k = p.n - 1;
  return (int32_t)k;
}
ChungLu chung_lu_params(int64_t n, double gamma, double mean_deg);

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------- graph handle
struct TcPlan;
struct RankPlan;
struct RankGraph;
struct LabelCsr;
struct MotifPlan;
struct CliquePlan;
struct MotifPlan;

}  // namespace gpm

struct gpm_graph {
  int64_t n = 0;
  int64_t nnz = 0;
  int32_t max_deg = 0;
  int oriented = 0;
  int relabeled = 0;
  int device = 0;
  gpm::DevBuf<int64_t> off;     // n + 1
  gpm::DevBuf<int32_t> adj;     // nnz
  gpm::DevBuf<int32_t> labels;  // n (optional)
  gpm::DevBuf<int32_t> src;     // nnz, COO source of each stored entry (lazy)
  gpm::TcPlan *tc = nullptr;    // cached triangle-count schedule (HASH)
  gpm::RankPlan *rank = nullptr; // cached schedule of the BITMAP path
  gpm::RankGraph *rg = nullptr;  // cached rank-relabelled copy
  gpm::RankPlan *learned = nullptr;  // plan chosen by the attached scheduler
  gpm::LabelCsr *lcsr = nullptr;     // label-partitioned lists (matching)
  gpm::MotifPlan *motif[2] = {nullptr, nullptr};  // cached motif pipelines (3-, 4-vertex)
  gpm::CliquePlan *clique[9] = {};                // cached k-clique schedules, by k
  gpm_sched *sched = nullptr;        // learned scheduler (not owned)
  gpm::DevBuf<uint64_t> result; // small device result scratch
  ~gpm_graph();
};

namespace gpm {
// graph.cu
int build_csr_device(gpm_graph *g, int64_t n, int64_t m, const int32_t *d_src,
                     const int32_t *d_dst, int symmetrize, cudaStream_t st);
int ensure_src(gpm_graph *g, cudaStream_t st);
int compute_max_degree(gpm_graph *g, cudaStream_t st);
void free_tc_plan(TcPlan *p);
void free_rank_plan(RankPlan *p);
void free_rank_graph(RankGraph *r);
void free_label_csr(LabelCsr *p);
void free_motif_plan(MotifPlan *p);  // motif.cu
void free_clique_plan(CliquePlan *p);  // clique.cu
// Drops every cached schedule (after the stored graph changed).
void drop_plans(gpm_graph *g);
int num_sms();

// A launch parameter (a persistent grid size, after the kernel's attributes
// are set) computed by `init` the first time it is needed on each device,
// with that device current: function attributes and SM counts are per
// device.
struct PerDevice {
  static constexpr int kDevices = 64;
  std::atomic<int> v[kDevices] = {};
  template <class F>
  int get(F init) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kDevices) return init();
    int x = v[dev].load(std::memory_order_relaxed);
    if (!x) {
      x = init();
      v[dev].store(x, std::memory_order_relaxed);
    }
    return x;
  }
};
}  // namespace gpm
