// sched.cu -- learned task scheduler for the triangle-count path (no
// counterpart in the reference, whose fixed thresholds USE_CTA = 100 and
// USE_WARP = 2, tuning_schedules.cuh:196-197, and size switches,
// new_edge_warp.cuh:633-639, it replaces; the fixed rule stays as the
// fallback and as the yardstick of the learned schedule's regret).
//
// Decision per owner task of GPM_TC_BITMAP (tc_rank.cu): one of 6
// configurations = queue (warp | CTA) x long-segment threshold (16 | 64 | 256).
// Counts do not depend on the choice; only time does.
//
// Data: the engine logs, for every owner, its cost in active warp-cycles (the
// cycles each of its warps spent on it, barrier waits excluded) under each
// configuration (instrumented kernel k_tc_rank_t<true>) together with 8
// features of the task (list and partner sizes, key span) -- the
// intersection-size trace of the owner.
// Model: 3-layer FP32 MLP 8 -> 32 -> 32 -> 6 (ReLU) predicting log2 cost of
// each configuration; trained on the GPU with full-batch Adam by the kernels
// below (one thread per sample, per-weight gradients reduced with warp
// shuffles into shared memory); inference is fused into the kernel that
// computes the features and writes each owner's configuration.
#include <algorithm>
#include <cmath>
#include <random>
#include <mutex>
#include <set>
#include <vector>

#include "common.cuh"
#include "tc.cuh"
#include "tc_rank.cuh"

namespace gpm {

constexpr int kIn = 8, kH = 32, kOut = 6;
constexpr int kW1 = 0, kB1 = kW1 + kIn * kH, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
              kB3 = kW3 + kH * kOut, kParams = kB3 + kOut;  // 1542

}  // namespace gpm

struct gpm_sched {
  gpm::DevBuf<float> w, g, m, v;  // parameters, gradient, Adam moments
  gpm::DevBuf<float> X, Y;        // dataset: rows x kIn features, rows x kOut log2 costs
  int64_t rows = 0, cap = 0;
  int t = 0;                      // Adam step
  gpm::DevBuf<double> loss;
};

namespace gpm {

// ------------------------------------------------------------ model
__device__ __forceinline__ void mlp_forward(const float *__restrict__ w, const float *x, float *h1, float *h2,
                                            float *y) {
#pragma unroll 4
  for (int j = 0; j < kH; ++j) {
    float a = w[kB1 + j];
    for (int f = 0; f < kIn; ++f) a += x[f] * w[kW1 + f * kH + j];
    h1[j] = fmaxf(a, 0.f);
  }
#pragma unroll 4
  for (int j = 0; j < kH; ++j) {
    float a = w[kB2 + j];
    for (int i = 0; i < kH; ++i) a += h1[i] * w[kW2 + i * kH + j];
    h2[j] = fmaxf(a, 0.f);
  }
  for (int k = 0; k < kOut; ++k) {
    float a = w[kB3 + k];
    for (int j = 0; j < kH; ++j) a += h2[j] * w[kW3 + j * kOut + k];
    y[k] = a;
  }
}

// Adds v (one value per lane) summed over the warp into *dst (shared memory).
__device__ __forceinline__ void wacc(float *dst, float v, unsigned lane) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) atomicAdd(dst, v);
}

// Gradient of L = (1/(N*kOut_valid)) * sum (y - t)^2 over the valid targets
// (finite entries of T), summed into grad; the loss sum into *loss.
__global__ void __launch_bounds__(256) k_mlp_grad(const float *__restrict__ X, const float *__restrict__ T,
                                                  int64_t N, float scale, const float *__restrict__ w,
                                                  float *__restrict__ grad, double *__restrict__ loss) {
  __shared__ float sw[kParams];
  __shared__ float sg[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    sw[i] = w[i];
    sg[i] = 0.f;
  }
  __syncthreads();
  const unsigned lane = threadIdx.x & 31;
  double l = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // whole warps iterate together so the shuffles stay converged
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < N; base += stride) {
    const int64_t s = base + lane;
    const bool ok = s < N;
    float x[kIn], h1[kH], h2[kH], y[kOut], dy[kOut];
    for (int f = 0; f < kIn; ++f) x[f] = ok ? X[s * kIn + f] : 0.f;
    mlp_forward(sw, x, h1, h2, y);
    for (int k = 0; k < kOut; ++k) {
      float t = ok ? T[s * kOut + k] : NAN;
      bool valid = isfinite(t);
      float d = valid ? y[k] - t : 0.f;
      l += (double)d * d;
      dy[k] = 2.f * d * scale;
    }
    for (int k = 0; k < kOut; ++k) wacc(&sg[kB3 + k], dy[k], lane);
    float dh2[kH];
    for (int j = 0; j < kH; ++j) {
      float a = 0.f;
      for (int k = 0; k < kOut; ++k) {
        wacc(&sg[kW3 + j * kOut + k], h2[j] * dy[k], lane);
        a += sw[kW3 + j * kOut + k] * dy[k];
      }
      dh2[j] = h2[j] > 0.f ? a : 0.f;
    }
    float dh1[kH];
    for (int i = 0; i < kH; ++i) dh1[i] = 0.f;
    for (int j = 0; j < kH; ++j) {
      wacc(&sg[kB2 + j], dh2[j], lane);
      for (int i = 0; i < kH; ++i) {
        wacc(&sg[kW2 + i * kH + j], h1[i] * dh2[j], lane);
        dh1[i] += sw[kW2 + i * kH + j] * dh2[j];
      }
    }
    for (int i = 0; i < kH; ++i) {
      float d = h1[i] > 0.f ? dh1[i] : 0.f;
      wacc(&sg[kB1 + i], d, lane);
      for (int f = 0; f < kIn; ++f) wacc(&sg[kW1 + f * kH + i], x[f] * d, lane);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) atomicAdd(&grad[i], sg[i]);
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if (lane == 0) atomicAdd(loss, l);
}

__global__ void k_mlp_forward(const float *__restrict__ X, int64_t N, const float *__restrict__ w,
                              float *__restrict__ Y) {
  __shared__ float sw[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
    float x[kIn], h1[kH], h2[kH], y[kOut];
    for (int f = 0; f < kIn; ++f) x[f] = X[s * kIn + f];
    mlp_forward(sw, x, h1, h2, y);
    for (int k = 0; k < kOut; ++k) Y[s * kOut + k] = y[k];
  }
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float b1, float b2, float c1, float c2, float eps) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
  }
}

// ------------------------------------------------------------ features
// The partner segments of a plan: owner x's long ones at pseg[poff[x] ..
// + plong[x]), its short ones at the back of its room (pshort[x] of them,
// ending at poff[x+1]), its dense ones (plans with a dense core) at
// dseg[doff[x] .. doff[x+1]).
struct SegView {
  const int64_t *poff;
  const Seg *pseg;
  const int32_t *plong, *pshort;
  const int64_t *doff;  // nullptr: no dense segments
  const Seg *dseg;
};
static SegView seg_view(const RankPlan *h) {
  return SegView{h->poff.p, h->pseg.p, h->plong.p, h->pshort.p, h->n_rows ? h->doff.p : nullptr,
                 h->n_rows ? h->dseg.p : nullptr};
}

// Owner x (a task of the heuristic plan): 8 features from its key list and
// all its partner segments (long, dense and short alike).  One warp per
// owner; lane 0 writes.
__device__ __forceinline__ void owner_features(int32_t x, const int64_t *__restrict__ roff,
                                               const int32_t *__restrict__ radj, const SegView &v, unsigned lane,
                                               float *f) {
  const int64_t d = roff[x + 1] - roff[x];
  const int nl = v.plong[x], ns = v.pshort[x];
  const int64_t d0 = v.doff ? v.doff[x] : 0;
  const int nd = v.doff ? (int)(v.doff[x + 1] - d0) : 0;
  const int nseg = nl + nd + ns;
  const int64_t back = v.poff[x + 1] - ns - nl - nd;  // short slot i >= nl + nd lives at back + i
  unsigned long long work = 0;
  long long mx = 0, nlong = 0;
  for (int i = (int)lane; i < nseg; i += 32) {
    const Seg sg = i < nl ? v.pseg[v.poff[x] + i] : i < nl + nd ? v.dseg[d0 + (i - nl)] : v.pseg[back + i];
    const long long len = seg_keys(sg);
    work += (unsigned long long)len;
    mx = max(mx, len);
    nlong += len >= 32;
  }
  work = warp_sum(work);
  nlong = warp_sum(nlong);
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const long long span = d > 0 ? (long long)radj[roff[x + 1] - 1] - radj[roff[x]] + 1 : 0;
  f[0] = log2f(1.f + (float)d);
  f[1] = log2f(1.f + (float)nseg);
  f[2] = log2f(1.f + (float)work);
  f[3] = log2f(1.f + (float)mx);
  f[4] = log2f(1.f + (float)nlong);
  f[5] = log2f(1.f + (float)span);
  f[6] = span <= 32ll * kRankCtaWords ? 1.f : 0.f;      // fits the CTA bitmap
  f[7] = span <= 32ll * kRankCtaWords / 8 ? 1.f : 0.f;  // fits a warp's bitmap
}

__global__ void k_features(const int32_t *__restrict__ tasks, int ntasks, const int64_t *__restrict__ roff,
                           const int32_t *__restrict__ radj, SegView v, float *__restrict__ X) {
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = warp; t < ntasks; t += nw) {
    float f[kIn];
    owner_features(tasks[t], roff, radj, v, lane, f);
    if (lane == 0)
      for (int i = 0; i < kIn; ++i) X[t * kIn + i] = f[i];
  }
}

__global__ void k_gather_costs(const int32_t *__restrict__ tasks, int ntasks, const unsigned long long *__restrict__ rec,
                               int cfg, float *__restrict__ Y) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntasks; t += (int64_t)gridDim.x * blockDim.x)
    Y[t * kOut + cfg] = log2f(1.f + (float)rec[tasks[t]]);
}

// Fused scheduler: features + MLP inference + argmin -> cfg[owner] (over the
// CTA configurations only for owners with more than kRankCtaMin keys).  For a
// task whose cheapest configuration is a warp one, its predicted cost and
// its cheapest CTA configuration go to warp_cost[t] / cta_alt[t] (0 / -
// otherwise); every task's predicted cost is summed into *total.
__global__ void __launch_bounds__(256) k_assign(const int32_t *__restrict__ tasks, int ntasks,
                                                const int64_t *__restrict__ roff, const int32_t *__restrict__ radj,
                                                SegView v, const float *__restrict__ w, uint8_t *__restrict__ cfg,
                                                float *__restrict__ warp_cost, uint8_t *__restrict__ cta_alt,
                                                double *__restrict__ total) {
  __shared__ float sw[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  const unsigned lane = lane_id();
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double sum = 0;
  for (int64_t t = warp; t < ntasks; t += nw) {
    float f[kIn];
    const int32_t x = tasks[t];
    owner_features(x, roff, radj, v, lane, f);
    if (lane == 0) {
      float h1[kH], h2[kH], y[kOut];
      mlp_forward(sw, f, h1, h2, y);
      // owners above the fixed CTA threshold stay CTA tasks (only their
      // segment threshold is learned): demoting a large owner to one warp
      // can only lengthen the run's tail
      int cta = kOut / 2;
      for (int k = kOut / 2 + 1; k < kOut; ++k)
        if (y[k] < y[cta]) cta = k;
      int best = cta;
      if (roff[x + 1] - roff[x] <= kRankCtaMin)
        for (int k = 0; k < kOut / 2; ++k)
          if (y[k] < y[best]) best = k;
      const float cost = exp2f(y[best]) - 1.f;
      cfg[x] = (uint8_t)best;
      warp_cost[t] = best < kOut / 2 ? cost : 0.f;
      cta_alt[t] = (uint8_t)cta;
      sum += cost;
    }
  }
  if (lane == 0 && sum > 0) atomicAdd(total, sum);
}

// Makespan rail.  The CTA queue drains first and the warp queue last, so a
// warp task predicted to cost more than kRail x (total / warp slots) would
// run on after every other warp is done; it takes its cheapest CTA
// configuration instead, spreading it over a CTA's 8 warps.
constexpr float kRail = 0.5f;
__global__ void k_rail(const int32_t *__restrict__ tasks, int ntasks, const float *__restrict__ warp_cost,
                       const uint8_t *__restrict__ cta_alt, const double *__restrict__ total, double slots,
                       uint8_t *__restrict__ cfg) {
  const float bound = (float)(kRail * *total / slots);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntasks; t += (int64_t)gridDim.x * blockDim.x)
    if (warp_cost[t] > bound) cfg[tasks[t]] = cta_alt[t];
}

static int blocks(int64_t work) { return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, num_sms() * 8)); }

// all owners of the heuristic plan, in one device list (the owners whose
// segments are all dense, and so in neither of its queues, included)
static int all_tasks(gpm_graph *g, DevBuf<int32_t> &tasks, int *ntasks, cudaStream_t st) {
  GPM_TRY(rank_build_plan(g, kRankCtaMin, kRankLongMin, st));
  RankPlan *p = g->rank;
  *ntasks = p->n_cta + p->n_warp + p->n_dense_only;
  GPM_TRY(tasks.reserve(std::max(1, *ntasks)));
  if (p->n_cta)
    GPM_CUDA(cudaMemcpyAsync(tasks.p, p->cta_tasks.p, sizeof(int32_t) * p->n_cta, cudaMemcpyDeviceToDevice, st));
  if (p->n_warp)
    GPM_CUDA(cudaMemcpyAsync(tasks.p + p->n_cta, p->warp_tasks.p, sizeof(int32_t) * p->n_warp,
                             cudaMemcpyDeviceToDevice, st));
  if (p->n_dense_only)
    GPM_CUDA(cudaMemcpyAsync(tasks.p + p->n_cta + p->n_warp, p->dense_only.p, sizeof(int32_t) * p->n_dense_only,
                             cudaMemcpyDeviceToDevice, st));
  return GPM_OK;
}

// Configuration of every task of the fixed plan under scheduler s into cfg
// (device, one byte per vertex; entries of non-tasks are left as they are).
static int assign_configs(gpm_graph *g, gpm_sched *s, const int32_t *tasks, int nt, uint8_t *cfg, cudaStream_t st) {
  if (nt <= 0) return GPM_OK;
  DevBuf<float> warp_cost;
  DevBuf<uint8_t> cta_alt;
  DevBuf<double> total;
  GPM_TRY(warp_cost.reserve(nt));
  GPM_TRY(cta_alt.reserve(nt));
  GPM_TRY(total.reserve(1));
  GPM_CUDA(cudaMemsetAsync(total.p, 0, sizeof(double), st));
  RankPlan *h = g->rank;
  k_assign<<<blocks((int64_t)nt * 32), 256, 0, st>>>(tasks, nt, g->rg->roff.p, g->rg->radj.p, seg_view(h), s->w.p,
                                                     cfg, warp_cost.p, cta_alt.p, total.p);
  GPM_LAUNCH_CHECK();
  // warp slots of the count kernel: 8 CTAs of 8 warps per SM
  k_rail<<<blocks(nt), 256, 0, st>>>(tasks, nt, warp_cost.p, cta_alt.p, total.p, 64.0 * num_sms(), cfg);
  GPM_LAUNCH_CHECK();
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

// Live schedulers: a graph keeps a plain pointer to the one attached to it,
// and the process keeps one default, so every use checks that the scheduler
// still exists (destroying it clears the default).
static std::mutex g_sched_mu;
static std::set<gpm_sched *> g_sched_live;
static gpm_sched *g_default_sched = nullptr;

static bool sched_live(gpm_sched *s) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  return s && g_sched_live.count(s);
}

int tc_learned_launch(gpm_graph *g, cudaStream_t st, unsigned long long *d_out) {
  if (!g->learned) {
    gpm_sched *s = g->sched;
    if (!s) {
      std::lock_guard<std::mutex> lk(g_sched_mu);
      s = g_default_sched;
    }
    if (!s)
      return fail(GPM_EUNSUPPORTED, "no trained scheduler attached (gpm_sched_attach / gpm_sched_set_default)");
    if (!sched_live(s)) return fail(GPM_EINVAL, "the graph's scheduler was destroyed");
    DevBuf<int32_t> tasks;
    int nt = 0;
    GPM_TRY(all_tasks(g, tasks, &nt, st));
    DevBuf<uint8_t> cfg;
    GPM_TRY(cfg.reserve(g->n));
    // owners that are not tasks keep the heuristic's class (unused)
    GPM_CUDA(cudaMemsetAsync(cfg.p, 1, g->n, st));
    GPM_TRY(assign_configs(g, s, tasks.p, nt, cfg.p, st));
    RankPlan *p = nullptr;
    GPM_TRY(rank_plan_new(g, kRankCtaMin, kRankLongMin, cfg.p, st, &p));
    g->learned = p;
  }
  return rank_plan_launch(g, g->learned, st, d_out, nullptr);
}

}  // namespace gpm

using namespace gpm;

extern "C" {

int gpm_sched_create(uint64_t seed, gpm_sched **out) {
  if (!out) return fail(GPM_EINVAL, "NULL out");
  GPM_TRY(ensure_device());
  gpm_sched *s = new gpm_sched();
  std::vector<float> h(kParams, 0.f);
  std::mt19937_64 rng(seed);
  auto init = [&](int off, int fan_in, int count) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / fan_in));
    for (int i = 0; i < count; ++i) h[off + i] = nd(rng);
  };
  init(kW1, kIn, kIn * kH);
  init(kW2, kH, kH * kH);
  init(kW3, kH, kH * kOut);
  int st = GPM_OK;
  if ((st = s->w.reserve(kParams)) || (st = s->g.reserve(kParams)) || (st = s->m.reserve(kParams)) ||
      (st = s->v.reserve(kParams)) || (st = s->loss.reserve(1))) {
    delete s;
    return st;
  }
  cudaMemcpy(s->w.p, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice);
  cudaMemset(s->m.p, 0, sizeof(float) * kParams);
  cudaMemset(s->v.p, 0, sizeof(float) * kParams);
  {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched_live.insert(s);
  }
  *out = s;
  return GPM_OK;
}

int gpm_sched_destroy(gpm_sched *s) {
  if (!s) return GPM_OK;
  {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    if (!g_sched_live.erase(s)) return fail(GPM_EINVAL, "gpm_sched_destroy: not a live scheduler");
    if (g_default_sched == s) g_default_sched = nullptr;
  }
  delete s;
  return GPM_OK;
}

int gpm_sched_param_count(void) { return kParams; }

int gpm_sched_get_params(const gpm_sched *s, float *params) {
  if (!s || !params) return fail(GPM_EINVAL, "NULL argument");
  GPM_CUDA(cudaMemcpy(params, s->w.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  return GPM_OK;
}

int gpm_sched_set_params(gpm_sched *s, const float *params) {
  if (!s || !params) return fail(GPM_EINVAL, "NULL argument");
  GPM_CUDA(cudaMemcpy(s->w.p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  return GPM_OK;
}

// Logs every owner task of g under each of the 6 configurations and appends
// (features, log2 active warp-cycles) rows to the dataset.
int gpm_sched_collect(gpm_sched *s, gpm_graph *g, int64_t *rows_added) {
  if (!s || !g) return fail(GPM_EINVAL, "NULL argument");
  cudaStream_t st = 0;
  DevBuf<int32_t> tasks;
  int nt = 0;
  GPM_TRY(all_tasks(g, tasks, &nt, st));
  if (rows_added) *rows_added = nt;
  if (nt == 0) return GPM_OK;
  // grow the dataset
  if (s->rows + nt > s->cap) {
    int64_t cap = std::max<int64_t>(2 * s->cap, s->rows + nt);
    DevBuf<float> X2, Y2;
    GPM_TRY(X2.reserve(cap * kIn));
    GPM_TRY(Y2.reserve(cap * kOut));
    if (s->rows) {
      GPM_CUDA(cudaMemcpy(X2.p, s->X.p, sizeof(float) * s->rows * kIn, cudaMemcpyDeviceToDevice));
      GPM_CUDA(cudaMemcpy(Y2.p, s->Y.p, sizeof(float) * s->rows * kOut, cudaMemcpyDeviceToDevice));
    }
    s->X = std::move(X2);
    s->Y = std::move(Y2);
    s->cap = cap;
  }
  RankPlan *h = g->rank;
  k_features<<<blocks((int64_t)nt * 32), 256, 0, st>>>(tasks.p, nt, g->rg->roff.p, g->rg->radj.p, seg_view(h),
                                                       s->X.p + s->rows * kIn);
  DevBuf<unsigned long long> rec, cnt;
  DevBuf<uint8_t> cfg;
  GPM_TRY(rec.reserve(g->n));
  GPM_TRY(cnt.reserve(1));
  GPM_TRY(cfg.reserve(g->n));
  for (int c = 0; c < kOut; ++c) {
    GPM_CUDA(cudaMemsetAsync(cfg.p, c, g->n, st));
    RankPlan *p = nullptr;
    GPM_TRY(rank_plan_new(g, kRankCtaMin, kRankLongMin, cfg.p, st, &p));
    int s1 = rank_plan_launch(g, p, st, cnt.p, nullptr);  // warm the caches
    if (s1 == GPM_OK && cudaMemsetAsync(rec.p, 0, sizeof(unsigned long long) * g->n, st) != cudaSuccess)
      s1 = fail(GPM_ECUDA, "memset");
    if (s1 == GPM_OK) s1 = rank_plan_launch(g, p, st, cnt.p, rec.p);
    if (s1 == GPM_OK)
      k_gather_costs<<<blocks(nt), 256, 0, st>>>(tasks.p, nt, rec.p, c, s->Y.p + s->rows * kOut);
    cudaError_t e = cudaStreamSynchronize(st);
    free_rank_plan(p);
    if (s1 != GPM_OK) return s1;
    if (e != cudaSuccess) return fail(GPM_ECUDA, cudaGetErrorString(e));
  }
  s->rows += nt;
  return GPM_OK;
}

int gpm_sched_dataset(const gpm_sched *s, int64_t *rows, float *X, float *Y) {
  if (!s || !rows) return fail(GPM_EINVAL, "NULL argument");
  *rows = s->rows;
  if (X && s->rows) GPM_CUDA(cudaMemcpy(X, s->X.p, sizeof(float) * s->rows * kIn, cudaMemcpyDeviceToHost));
  if (Y && s->rows) GPM_CUDA(cudaMemcpy(Y, s->Y.p, sizeof(float) * s->rows * kOut, cudaMemcpyDeviceToHost));
  return GPM_OK;
}

// Loss and gradient of the MSE on host arrays (X: N x 8, T: N x 6, NaN =
// no target) at the current parameters -- the gradient check entry point.
int gpm_sched_grad(gpm_sched *s, int64_t N, const float *X, const float *T, float *grad, double *loss) {
  if (!s || !X || !T || N < 1) return fail(GPM_EINVAL, "bad argument");
  DevBuf<float> dX, dT;
  GPM_TRY(dX.reserve(N * kIn));
  GPM_TRY(dT.reserve(N * kOut));
  GPM_CUDA(cudaMemcpy(dX.p, X, sizeof(float) * N * kIn, cudaMemcpyHostToDevice));
  GPM_CUDA(cudaMemcpy(dT.p, T, sizeof(float) * N * kOut, cudaMemcpyHostToDevice));
  int valid = 0;
  for (int64_t i = 0; i < N * kOut; ++i) valid += std::isfinite(T[i]) ? 1 : 0;
  GPM_CUDA(cudaMemset(s->g.p, 0, sizeof(float) * kParams));
  GPM_CUDA(cudaMemset(s->loss.p, 0, sizeof(double)));
  k_mlp_grad<<<blocks(N), 256>>>(dX.p, dT.p, N, 1.f / std::max(1, valid), s->w.p, s->g.p, s->loss.p);
  GPM_LAUNCH_CHECK();
  if (grad) GPM_CUDA(cudaMemcpy(grad, s->g.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  double l = 0;
  GPM_CUDA(cudaMemcpy(&l, s->loss.p, sizeof(double), cudaMemcpyDeviceToHost));
  if (loss) *loss = l / std::max(1, valid);
  return GPM_OK;
}

int gpm_sched_predict(gpm_sched *s, int64_t N, const float *X, float *Y) {
  if (!s || !X || !Y || N < 1) return fail(GPM_EINVAL, "bad argument");
  DevBuf<float> dX, dY;
  GPM_TRY(dX.reserve(N * kIn));
  GPM_TRY(dY.reserve(N * kOut));
  GPM_CUDA(cudaMemcpy(dX.p, X, sizeof(float) * N * kIn, cudaMemcpyHostToDevice));
  k_mlp_forward<<<blocks(N), 256>>>(dX.p, N, s->w.p, dY.p);
  GPM_LAUNCH_CHECK();
  GPM_CUDA(cudaMemcpy(Y, dY.p, sizeof(float) * N * kOut, cudaMemcpyDeviceToHost));
  return GPM_OK;
}

// Full-batch Adam on the collected dataset.
int gpm_sched_train(gpm_sched *s, int steps, float lr, double *final_loss) {
  if (!s || steps < 0) return fail(GPM_EINVAL, "bad argument");
  if (s->rows == 0) return fail(GPM_EINVAL, "empty dataset: run gpm_sched_collect first");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float scale = 1.f / (float)(s->rows * kOut);
  double l = 0;
  for (int it = 0; it < steps; ++it) {
    GPM_CUDA(cudaMemsetAsync(s->g.p, 0, sizeof(float) * kParams));
    GPM_CUDA(cudaMemsetAsync(s->loss.p, 0, sizeof(double)));
    k_mlp_grad<<<blocks(s->rows), 256>>>(s->X.p, s->Y.p, s->rows, scale, s->w.p, s->g.p, s->loss.p);
    ++s->t;
    float c1 = 1.f - std::pow(b1, (float)s->t), c2 = 1.f - std::pow(b2, (float)s->t);
    k_adam<<<(kParams + 255) / 256, 256>>>(s->w.p, s->g.p, s->m.p, s->v.p, kParams, lr, b1, b2, c1, c2, eps);
    GPM_LAUNCH_CHECK();
  }
  GPM_CUDA(cudaMemcpy(&l, s->loss.p, sizeof(double), cudaMemcpyDeviceToHost));
  if (final_loss) *final_loss = l * scale;
  return GPM_OK;
}

// g's GPM_TC_LEARNED variant uses s (s must outlive g or be detached).
int gpm_sched_attach(gpm_graph *g, gpm_sched *s) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  if (s && !sched_live(s)) return fail(GPM_EINVAL, "gpm_sched_attach: not a live scheduler");
  free_rank_plan(g->learned);
  g->learned = nullptr;
  g->sched = s;
  return GPM_OK;
}

// Process-wide scheduler for graphs without an attached one (NULL clears it).
int gpm_sched_set_default(gpm_sched *s) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  if (s && !g_sched_live.count(s)) return fail(GPM_EINVAL, "gpm_sched_set_default: not a live scheduler");
  g_default_sched = s;
  return GPM_OK;
}

// Logged cost (active warp-cycles) of every owner under each configuration:
// cost[6 * v + c], 0 for vertices that own no task.
int gpm_tc_task_costs(gpm_graph *g, float *cost) {
  if (!g || !cost) return fail(GPM_EINVAL, "NULL argument");
  cudaStream_t st = 0;
  DevBuf<int32_t> tasks;
  int nt = 0;
  GPM_TRY(all_tasks(g, tasks, &nt, st));
  DevBuf<unsigned long long> rec, cnt;
  DevBuf<uint8_t> cfg;
  GPM_TRY(rec.reserve(g->n));
  GPM_TRY(cnt.reserve(1));
  GPM_TRY(cfg.reserve(g->n));
  std::vector<unsigned long long> h(g->n);
  for (int c = 0; c < kOut; ++c) {
    GPM_CUDA(cudaMemsetAsync(cfg.p, c, g->n, st));
    RankPlan *p = nullptr;
    GPM_TRY(rank_plan_new(g, kRankCtaMin, kRankLongMin, cfg.p, st, &p));
    int s1 = rank_plan_launch(g, p, st, cnt.p, nullptr);  // warm the caches
    if (s1 == GPM_OK && cudaMemsetAsync(rec.p, 0, sizeof(unsigned long long) * g->n, st) != cudaSuccess)
      s1 = fail(GPM_ECUDA, "memset");
    if (s1 == GPM_OK) s1 = rank_plan_launch(g, p, st, cnt.p, rec.p);
    if (s1 == GPM_OK && cudaMemcpy(h.data(), rec.p, sizeof(unsigned long long) * g->n, cudaMemcpyDeviceToHost) !=
                            cudaSuccess)
      s1 = fail(GPM_ECUDA, "cost copy");
    free_rank_plan(p);
    if (s1 != GPM_OK) return s1;
    for (int64_t v = 0; v < g->n; ++v) cost[6 * v + c] = (float)h[v];
  }
  return GPM_OK;
}

// An explicit per-owner configuration for GPM_TC_LEARNED on g (host cfg[v] in
// 0..5): replaces whatever schedule the scheduler chose, until the graph's
// plans are dropped or a scheduler is attached.
int gpm_tc_set_schedule(gpm_graph *g, const uint8_t *cfg) {
  if (!g || !cfg) return fail(GPM_EINVAL, "NULL argument");
  for (int64_t v = 0; v < g->n; ++v)
    if (cfg[v] >= kOut) return fail(GPM_EINVAL, "configuration out of range (0..5)");
  DevBuf<uint8_t> d;
  GPM_TRY(d.reserve(std::max<int64_t>(g->n, 1)));
  if (g->n) GPM_CUDA(cudaMemcpy(d.p, cfg, g->n, cudaMemcpyHostToDevice));
  RankPlan *p = nullptr;
  GPM_TRY(rank_plan_new(g, kRankCtaMin, kRankLongMin, d.p, 0, &p));
  free_rank_plan(g->learned);
  g->learned = p;
  return GPM_OK;
}

// Configuration each owner task would get: cfg[v] in 0..5 (255: no task).
int gpm_sched_assign(gpm_sched *s, gpm_graph *g, uint8_t *cfg) {
  if (!s || !g || !cfg) return fail(GPM_EINVAL, "NULL argument");
  DevBuf<int32_t> tasks;
  int nt = 0;
  GPM_TRY(all_tasks(g, tasks, &nt, 0));
  DevBuf<uint8_t> d;
  GPM_TRY(d.reserve(g->n));
  GPM_CUDA(cudaMemset(d.p, 255, g->n));
  GPM_TRY(assign_configs(g, s, tasks.p, nt, d.p, 0));
  GPM_CUDA(cudaMemcpy(cfg, d.p, g->n, cudaMemcpyDeviceToHost));
  return GPM_OK;
}

}  // extern "C"
