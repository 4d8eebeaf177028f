// graph.cu -- device-side graph preparation: edge list -> sorted simple CSR,
// degree orientation (Graph::orientation, src/graph/graph.h:116-204) and the
// degree-descending relabel (Graph::SortCSRGraph, graph.h:206-252).
//
// HBM layout of a graph: off[n+1] (int64), adj[nnz] (int32), lists sorted
// ascending, optional labels[n] (int32) and a lazily built COO source array
// src[nnz] (int32) for edge-parallel kernels.
#include <atomic>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "tc.cuh"

namespace gpm {

int num_sms() {
  // per device: a process may drive GPUs with different SM counts
  constexpr int kDevs = 64;
  static std::atomic<int> sms[kDevs];
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < kDevs && (v = sms[dev].load(std::memory_order_relaxed)) > 0) return v;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (v <= 0) v = 148;
  if (dev >= 0 && dev < kDevs) sms[dev].store(v, std::memory_order_relaxed);
  return v;
}

static constexpr uint64_t kSentinel = ~0ull;

__global__ void k_make_keys(int64_t m, int64_t n, const int32_t *__restrict__ src,
                            const int32_t *__restrict__ dst, int symmetrize,
                            uint64_t *__restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    int32_t u = src[i], v = dst[i];
    bool ok = u != v && u >= 0 && v >= 0 && u < n && v < n;
    uint64_t k0 = ok ? (((uint64_t)(uint32_t)u << 32) | (uint32_t)v) : kSentinel;
    if (symmetrize) {
      keys[2 * i] = k0;
      keys[2 * i + 1] = ok ? (((uint64_t)(uint32_t)v << 32) | (uint32_t)u) : kSentinel;
    } else {
      keys[i] = k0;
    }
  }
}

template <typename L>
__global__ void k_gen_edges(int64_t m, L gen, int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    gen(i, &src[i], &dst[i]);
}

__global__ void k_split_keys(int64_t nnz, const uint64_t *__restrict__ keys,
                             int32_t *__restrict__ adj, unsigned long long *__restrict__ deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys[i];
    adj[i] = (int32_t)(k & 0xffffffffu);
    atomicAdd(&deg[k >> 32], 1ull);
  }
}

__global__ void k_deg_to_i64(int64_t n, const unsigned long long *__restrict__ deg, int64_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)deg[i];
}

static int grid_for(int64_t work, int block = 256) {
  int64_t g = (work + block - 1) / block;
  int64_t cap = (int64_t)num_sms() * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Exclusive scan of n int64 counts into off[0..n] (off[n] = total).
static int scan_offsets(int64_t n, const int64_t *counts, int64_t *off, cudaStream_t st) {
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, counts, off + 1, (int)n, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cudaMemsetAsync(off, 0, sizeof(int64_t), st));
  if (n > 0) GPM_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, counts, off + 1, (int)n, st));
  return GPM_OK;
}

int build_csr_device(gpm_graph *g, int64_t n, int64_t m, const int32_t *d_src,
                     const int32_t *d_dst, int symmetrize, cudaStream_t st) {
  if (n < 0 || n >= (1ll << 31) || m < 0) return fail(GPM_EINVAL, "graph size out of range");
  int64_t nk = symmetrize ? 2 * m : m;
  if (nk >= (1ll << 31)) return fail(GPM_EUNSUPPORTED, "more than 2^31 directed entries");
  DevBuf<uint64_t> k0, k1;
  GPM_TRY(k0.reserve(nk));
  GPM_TRY(k1.reserve(nk));
  if (m > 0) {
    k_make_keys<<<grid_for(m), 256, 0, st>>>(m, n, d_src, d_dst, symmetrize, k0.p);
    GPM_LAUNCH_CHECK();
  }
  int end_bit = 64;
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, k0.p, k1.p, (int)nk, 0, end_bit, st));
  DevBuf<int64_t> nsel;
  GPM_TRY(nsel.reserve(1));
  size_t tmp2 = 0;
  GPM_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, k1.p, k0.p, nsel.p, (int)nk, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(std::max(tmp, tmp2)));
  int64_t nuniq = 0;
  if (nk > 0) {
    GPM_CUDA(cub::DeviceRadixSort::SortKeys(t.p, tmp, k0.p, k1.p, (int)nk, 0, end_bit, st));
    GPM_CUDA(cub::DeviceSelect::Unique(t.p, tmp2, k1.p, k0.p, nsel.p, (int)nk, st));
    GPM_CUDA(cudaMemcpyAsync(&nuniq, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    GPM_CUDA(cudaStreamSynchronize(st));
    if (nuniq > 0) {
      uint64_t last = 0;
      GPM_CUDA(cudaMemcpy(&last, k0.p + nuniq - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost));
      if (last == kSentinel) --nuniq;
    }
  }
  k1.reset();
  g->n = n;
  g->nnz = nuniq;
  GPM_TRY(g->off.reserve(n + 1));
  GPM_TRY(g->adj.reserve(nuniq));
  DevBuf<unsigned long long> deg;
  DevBuf<int64_t> deg64;
  GPM_TRY(deg.reserve(n));
  GPM_TRY(deg64.reserve(n));
  GPM_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(unsigned long long) * (size_t)std::max<int64_t>(n, 1), st));
  if (nuniq > 0) {
    k_split_keys<<<grid_for(nuniq), 256, 0, st>>>(nuniq, k0.p, g->adj.p, deg.p);
    GPM_LAUNCH_CHECK();
  }
  if (n > 0) {
    k_deg_to_i64<<<grid_for(n), 256, 0, st>>>(n, deg.p, deg64.p);
    GPM_LAUNCH_CHECK();
  }
  GPM_TRY(scan_offsets(n, deg64.p, g->off.p, st));
  g->src.reset();
  GPM_TRY(compute_max_degree(g, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  return GPM_OK;
}

__global__ void k_degrees(int64_t n, const int64_t *__restrict__ off, int32_t *__restrict__ deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    deg[i] = (int32_t)(off[i + 1] - off[i]);
}

int compute_max_degree(gpm_graph *g, cudaStream_t st) {
  if (g->n == 0) {
    g->max_deg = 0;
    return GPM_OK;
  }
  DevBuf<int32_t> deg, mx;
  GPM_TRY(deg.reserve(g->n));
  GPM_TRY(mx.reserve(1));
  k_degrees<<<grid_for(g->n), 256, 0, st>>>(g->n, g->off.p, deg.p);
  GPM_LAUNCH_CHECK();
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceReduce::Max(nullptr, tmp, deg.p, mx.p, (int)g->n, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cub::DeviceReduce::Max(t.p, tmp, deg.p, mx.p, (int)g->n, st));
  int32_t h = 0;
  GPM_CUDA(cudaMemcpyAsync(&h, mx.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  g->max_deg = h;
  return GPM_OK;
}

// COO source of every stored entry: warp per vertex.
__global__ void k_fill_src(int64_t n, const int64_t *__restrict__ off, int32_t *__restrict__ src) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t u = warp; u < n; u += nw)
    for (int64_t e = off[u] + lane_id(); e < off[u + 1]; e += 32) src[e] = (int32_t)u;
}

int ensure_src(gpm_graph *g, cudaStream_t st) {
  if (g->src.p && g->src.n >= (size_t)g->nnz) return GPM_OK;
  GPM_TRY(g->src.reserve(g->nnz));
  if (g->n > 0) {
    k_fill_src<<<grid_for(g->n * 32), 256, 0, st>>>(g->n, g->off.p, g->src.p);
    GPM_LAUNCH_CHECK();
  }
  return GPM_OK;
}

// Orientation rule of graph.h:128-129 on the current (pre-orientation) degrees.
__device__ __forceinline__ bool keep_edge(int32_t u, int32_t v, int64_t du, int64_t dv) {
  return dv > du || (dv == du && v > u);
}

__global__ void k_orient_count(int64_t n, const int64_t *__restrict__ off,
                               const int32_t *__restrict__ adj, int64_t *__restrict__ cnt) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t u = warp; u < n; u += nw) {
    int64_t s = off[u], e = off[u + 1], du = e - s, c = 0;
    for (int64_t i = s + lane_id(); i < e; i += 32) {
      int32_t v = adj[i];
      int64_t dv = off[v + 1] - off[v];
      c += keep_edge((int32_t)u, v, du, dv);
    }
    c = warp_sum(c);
    if (lane_id() == 0) cnt[u] = c;
  }
}

__global__ void k_orient_write(int64_t n, const int64_t *__restrict__ off,
                               const int32_t *__restrict__ adj, const int64_t *__restrict__ doff,
                               int32_t *__restrict__ dadj) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned lane = lane_id();
  for (int64_t u = warp; u < n; u += nw) {
    int64_t s = off[u], e = off[u + 1], du = e - s, w = doff[u];
    for (int64_t base = s; base < e; base += 32) {
      int64_t i = base + lane;
      bool k = false;
      int32_t v = 0;
      if (i < e) {
        v = adj[i];
        k = keep_edge((int32_t)u, v, du, off[v + 1] - off[v]);
      }
      unsigned mask = __ballot_sync(0xffffffffu, k);
      if (k) dadj[w + __popc(mask & ((1u << lane) - 1u))] = v;
      w += __popc(mask);
    }
  }
}

int orient_on_stream(gpm_graph *g, cudaStream_t st) {
  int64_t n = g->n;
  DevBuf<int64_t> cnt, doff;
  GPM_TRY(cnt.reserve(n));
  GPM_TRY(doff.reserve(n + 1));
  if (n > 0) {
    k_orient_count<<<grid_for(n * 32), 256, 0, st>>>(n, g->off.p, g->adj.p, cnt.p);
    GPM_LAUNCH_CHECK();
  }
  GPM_TRY(scan_offsets(n, cnt.p, doff.p, st));
  int64_t m2 = 0;
  GPM_CUDA(cudaMemcpyAsync(&m2, doff.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  GPM_CUDA(cudaStreamSynchronize(st));
  DevBuf<int32_t> dadj;
  GPM_TRY(dadj.reserve(m2));
  if (n > 0) {
    k_orient_write<<<grid_for(n * 32), 256, 0, st>>>(n, g->off.p, g->adj.p, doff.p, dadj.p);
    GPM_LAUNCH_CHECK();
  }
  g->off = std::move(doff);
  g->adj = std::move(dadj);
  g->nnz = m2;
  g->oriented = 1;
  g->src.reset();
  return GPM_OK;
}

// SortCSRGraph: stable order of vertices by out-degree descending.
__global__ void k_relabel_keys(int64_t n, const int64_t *__restrict__ off, int32_t maxd,
                               int32_t *__restrict__ key, int32_t *__restrict__ val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    key[i] = maxd - (int32_t)(off[i + 1] - off[i]);
    val[i] = (int32_t)i;
  }
}
__global__ void k_inverse(int64_t n, const int32_t *__restrict__ index, int32_t *__restrict__ rindex,
                          const int64_t *__restrict__ off, int64_t *__restrict__ newdeg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = index[i];
    rindex[v] = (int32_t)i;
    newdeg[i] = off[v + 1] - off[v];
  }
}
__global__ void k_relabel_copy(int64_t n, const int32_t *__restrict__ index,
                               const int32_t *__restrict__ rindex, const int64_t *__restrict__ off,
                               const int32_t *__restrict__ adj, const int64_t *__restrict__ noff,
                               int32_t *__restrict__ nadj) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < n; i += nw) {
    int32_t v = index[i];
    int64_t s = off[v], e = off[v + 1], o = noff[i];
    for (int64_t k = s + lane_id(); k < e; k += 32) nadj[o + (k - s)] = rindex[adj[k]];
  }
}

static int relabel_device(gpm_graph *g, cudaStream_t st) {
  int64_t n = g->n, nnz = g->nnz;
  if (n == 0) return GPM_OK;
  DevBuf<int32_t> key, key2, val, index, rindex;
  GPM_TRY(key.reserve(n));
  GPM_TRY(key2.reserve(n));
  GPM_TRY(val.reserve(n));
  GPM_TRY(index.reserve(n));
  GPM_TRY(rindex.reserve(n));
  GPM_TRY(compute_max_degree(g, st));
  k_relabel_keys<<<grid_for(n), 256, 0, st>>>(n, g->off.p, g->max_deg, key.p, val.p);
  GPM_LAUNCH_CHECK();
  size_t tmp = 0;
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key2.p, val.p, index.p, (int)n, 0, 32, st));
  DevBuf<char> t;
  GPM_TRY(t.reserve(tmp));
  GPM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, key2.p, val.p, index.p, (int)n, 0, 32, st));
  DevBuf<int64_t> newdeg, noff;
  GPM_TRY(newdeg.reserve(n));
  GPM_TRY(noff.reserve(n + 1));
  k_inverse<<<grid_for(n), 256, 0, st>>>(n, index.p, rindex.p, g->off.p, newdeg.p);
  GPM_LAUNCH_CHECK();
  GPM_TRY(scan_offsets(n, newdeg.p, noff.p, st));
  DevBuf<int32_t> nadj, sorted;
  GPM_TRY(nadj.reserve(nnz));
  GPM_TRY(sorted.reserve(nnz));
  k_relabel_copy<<<grid_for(n * 32), 256, 0, st>>>(n, index.p, rindex.p, g->off.p, g->adj.p, noff.p, nadj.p);
  GPM_LAUNCH_CHECK();
  if (nnz > 0) {
    size_t tmp2 = 0;
    GPM_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp2, nadj.p, sorted.p, (int)nnz, (int)n,
                                                noff.p, noff.p + 1, st));
    DevBuf<char> t2;
    GPM_TRY(t2.reserve(tmp2));
    GPM_CUDA(cub::DeviceSegmentedSort::SortKeys(t2.p, tmp2, nadj.p, sorted.p, (int)nnz, (int)n,
                                                noff.p, noff.p + 1, st));
  }
  if (g->labels.p) {
    // labels follow their vertices
    DevBuf<int32_t> nl;
    GPM_TRY(nl.reserve(n));
    // reuse k_relabel_copy pattern: nl[i] = labels[index[i]]
    std::vector<int32_t> hidx(n), hl(n), out(n);
    GPM_CUDA(cudaMemcpyAsync(hidx.data(), index.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    GPM_CUDA(cudaMemcpyAsync(hl.data(), g->labels.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    GPM_CUDA(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < n; ++i) out[i] = hl[hidx[i]];
    GPM_CUDA(cudaMemcpy(nl.p, out.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    g->labels = std::move(nl);
  }
  g->off = std::move(noff);
  g->adj = std::move(sorted);
  g->relabeled = 1;
  g->src.reset();
  return GPM_OK;
}

// Σ over stored u->v of deg(v), and of deg(u)+deg(v).
__global__ void k_work(int64_t n, const int64_t *__restrict__ off, const int32_t *__restrict__ adj,
                       unsigned long long *__restrict__ out) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long w = 0, p = 0;
  for (int64_t u = warp; u < n; u += nw) {
    int64_t du = off[u + 1] - off[u];
    for (int64_t k = off[u] + lane_id(); k < off[u + 1]; k += 32) {
      int32_t v = adj[k];
      int64_t dv = off[v + 1] - off[v];
      w += (unsigned long long)dv;
      p += (unsigned long long)(du + dv);
    }
  }
  w = warp_sum(w);
  p = warp_sum(p);
  if (lane_id() == 0) {
    atomicAdd(&out[0], w);
    atomicAdd(&out[1], p);
  }
}

}  // namespace gpm

using namespace gpm;

namespace gpm {
void drop_plans(gpm_graph *g) {
  free_tc_plan(g->tc);
  g->tc = nullptr;
  free_rank_plan(g->rank);
  g->rank = nullptr;
  free_rank_graph(g->rg);
  g->rg = nullptr;
  free_rank_plan(g->learned);
  g->learned = nullptr;
  free_label_csr(g->lcsr);
  g->lcsr = nullptr;
  for (MotifPlan *&m : g->motif) {
    free_motif_plan(m);
    m = nullptr;
  }
  for (CliquePlan *&c : g->clique) {
    free_clique_plan(c);
    c = nullptr;
  }
}
}  // namespace gpm

gpm_graph::~gpm_graph() { drop_plans(this); }

extern "C" {

int gpm_graph_create_device(int64_t n, int64_t m, const int32_t *d_src, const int32_t *d_dst,
                            int flags, gpm_graph **out) {
  if (!out || (m > 0 && (!d_src || !d_dst))) return fail(GPM_EINVAL, "gpm_graph_create_device: NULL argument");
  GPM_TRY(ensure_device());
  gpm_graph *g = new gpm_graph();
  cudaGetDevice(&g->device);
  int s = build_csr_device(g, n, m, d_src, d_dst, (flags & GPM_SYMMETRIZE) ? 1 : 0, 0);
  if (s != GPM_OK) {
    delete g;
    return s;
  }
  *out = g;
  return GPM_OK;
}

int gpm_graph_create(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                     const int32_t *labels, int flags, gpm_graph **out) {
  if (!out || (m > 0 && (!src || !dst)) || n < 0 || m < 0)
    return fail(GPM_EINVAL, "gpm_graph_create: bad argument");
  GPM_TRY(ensure_device());
  DevBuf<int32_t> ds, dd;
  GPM_TRY(ds.reserve(m));
  GPM_TRY(dd.reserve(m));
  if (m > 0) {
    GPM_CUDA(cudaMemcpy(ds.p, src, sizeof(int32_t) * m, cudaMemcpyHostToDevice));
    GPM_CUDA(cudaMemcpy(dd.p, dst, sizeof(int32_t) * m, cudaMemcpyHostToDevice));
  }
  gpm_graph *g = nullptr;
  GPM_TRY(gpm_graph_create_device(n, m, ds.p, dd.p, flags, &g));
  if (labels) {
    int s = gpm_graph_set_labels(g, labels);
    if (s != GPM_OK) {
      delete g;
      return s;
    }
  }
  *out = g;
  return GPM_OK;
}

__global__ void k_validate(int64_t n, const int64_t *__restrict__ off, const int32_t *__restrict__ adj,
                           int *__restrict__ bad) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = off[u], e = off[u + 1];
    if (e < s) { atomicOr(bad, 1); continue; }
    for (int64_t k = s; k < e; ++k) {
      int32_t v = adj[k];
      if (v < 0 || v >= n || v == u || (k > s && adj[k - 1] >= v)) { atomicOr(bad, 2); break; }
    }
  }
}

int gpm_graph_create_csr(int64_t n, const int64_t *offsets, const int32_t *indices,
                         const int32_t *labels, gpm_graph **out) {
  if (!out || !offsets || n < 0 || n >= (1ll << 31)) return fail(GPM_EINVAL, "gpm_graph_create_csr: bad argument");
  int64_t nnz = offsets[n];
  if (nnz < 0 || offsets[0] != 0 || (nnz > 0 && !indices)) return fail(GPM_EINVAL, "gpm_graph_create_csr: bad offsets");
  GPM_TRY(ensure_device());
  gpm_graph *g = new gpm_graph();
  cudaGetDevice(&g->device);
  g->n = n;
  g->nnz = nnz;
  int s = g->off.reserve(n + 1);
  if (s == GPM_OK) s = g->adj.reserve(nnz);
  if (s != GPM_OK) { delete g; return s; }
  cudaMemcpy(g->off.p, offsets, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice);
  if (nnz > 0) cudaMemcpy(g->adj.p, indices, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice);
  DevBuf<int> bad;
  int hbad = 0;
  s = bad.reserve(1);
  if (s == GPM_OK && n > 0) {
    cudaMemset(bad.p, 0, sizeof(int));
    k_validate<<<grid_for(n), 256>>>(n, g->off.p, g->adj.p, bad.p);
    cudaMemcpy(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { delete g; return fail(GPM_ECUDA, cudaGetErrorString(e)); }
  if (hbad) { delete g; return fail(GPM_EINVAL, "CSR lists must be sorted, duplicate-free, in range and loop-free"); }
  s = compute_max_degree(g, 0);
  if (s == GPM_OK && labels) s = gpm_graph_set_labels(g, labels);
  if (s != GPM_OK) { delete g; return s; }
  *out = g;
  return GPM_OK;
}

int gpm_graph_generate(int kind, int64_t p0, int64_t p1, double a, double b, double c,
                       uint64_t seed, gpm_graph **out) {
  if (!out) return fail(GPM_EINVAL, "out is NULL");
  GPM_TRY(ensure_device());
  int64_t n = 0, m = 0;
  DevBuf<int32_t> s, d;
  if (kind == 0) {
    int scale = (int)p0;
    if (scale < 1 || scale > 30 || p1 < 1) return fail(GPM_EINVAL, "bad R-MAT parameters");
    n = (int64_t)1 << scale;
    m = n * p1;
    GPM_TRY(s.reserve(m));
    GPM_TRY(d.reserve(m));
    auto gen = [=] __device__(int64_t i, int32_t *u, int32_t *v) { rmat_edge(seed, (uint64_t)i, scale, a, b, c, u, v); };
    k_gen_edges<<<grid_for(m), 256>>>(m, gen, s.p, d.p);
  } else if (kind == 1) {
    n = p0;
    m = p1;
    if (n < 1 || n >= (1ll << 31) || m < 0) return fail(GPM_EINVAL, "bad ER parameters");
    GPM_TRY(s.reserve(m));
    GPM_TRY(d.reserve(m));
    auto gen = [=] __device__(int64_t i, int32_t *u, int32_t *v) { er_edge(seed, (uint64_t)i, n, u, v); };
    if (m > 0) k_gen_edges<<<grid_for(m), 256>>>(m, gen, s.p, d.p);
  } else if (kind == 2) {
    n = p0;
    if (n < 2 || a <= 2.0 || b <= 0) return fail(GPM_EINVAL, "bad Chung-Lu parameters");
    m = (int64_t)llround((double)n * b / 2.0);
    ChungLu p = chung_lu_params(n, a, b);
    GPM_TRY(s.reserve(m));
    GPM_TRY(d.reserve(m));
    auto gen = [=] __device__(int64_t i, int32_t *u, int32_t *v) {
      *u = chung_lu_vertex(p, draw(seed, 201, (uint64_t)i));
      *v = chung_lu_vertex(p, draw(seed, 202, (uint64_t)i));
    };
    if (m > 0) k_gen_edges<<<grid_for(m), 256>>>(m, gen, s.p, d.p);
  } else {
    return fail(GPM_EINVAL, "unknown generator kind");
  }
  GPM_LAUNCH_CHECK();
  return gpm_graph_create_device(n, m, s.p, d.p, GPM_SYMMETRIZE, out);
}

int gpm_graph_destroy(gpm_graph *g) {
  delete g;
  return GPM_OK;
}

int gpm_graph_get_info(const gpm_graph *g, gpm_graph_info *info) {
  if (!g || !info) return fail(GPM_EINVAL, "NULL argument");
  info->n = g->n;
  info->nnz = g->nnz;
  info->max_degree = g->max_deg;
  info->oriented = g->oriented;
  info->relabeled = g->relabeled;
  info->has_labels = g->labels.p != nullptr;
  return GPM_OK;
}

int gpm_graph_copy_csr(const gpm_graph *g, int64_t *offsets, int32_t *indices) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  if (offsets) GPM_CUDA(cudaMemcpy(offsets, g->off.p, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost));
  if (indices && g->nnz > 0) GPM_CUDA(cudaMemcpy(indices, g->adj.p, sizeof(int32_t) * g->nnz, cudaMemcpyDeviceToHost));
  return GPM_OK;
}

int gpm_graph_set_labels(gpm_graph *g, const int32_t *labels) {
  if (!g || !labels) return fail(GPM_EINVAL, "NULL argument");
  GPM_TRY(g->labels.reserve(g->n));
  if (g->n > 0) GPM_CUDA(cudaMemcpy(g->labels.p, labels, sizeof(int32_t) * g->n, cudaMemcpyHostToDevice));
  free_label_csr(g->lcsr);  // the label partition follows the labels
  g->lcsr = nullptr;
  return GPM_OK;
}

int gpm_graph_orient(gpm_graph *g, int relabel) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  drop_plans(g);
  GPM_TRY(orient_on_stream(g, 0));
  if (relabel) GPM_TRY(relabel_device(g, 0));
  GPM_TRY(compute_max_degree(g, 0));
  GPM_CUDA(cudaDeviceSynchronize());
  return GPM_OK;
}

int gpm_graph_relabel(gpm_graph *g) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  drop_plans(g);
  GPM_TRY(relabel_device(g, 0));
  GPM_TRY(compute_max_degree(g, 0));
  GPM_CUDA(cudaDeviceSynchronize());
  return GPM_OK;
}

int gpm_graph_drop_plans(gpm_graph *g) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  GPM_CUDA(cudaDeviceSynchronize());  // no kernel may still read what is freed
  drop_plans(g);
  return GPM_OK;
}

int gpm_graph_work(gpm_graph *g, uint64_t *wedge_work, uint64_t *pair_work) {
  if (!g) return fail(GPM_EINVAL, "NULL graph");
  DevBuf<unsigned long long> o;
  GPM_TRY(o.reserve(2));
  GPM_CUDA(cudaMemset(o.p, 0, 16));
  if (g->n > 0) {
    k_work<<<grid_for(g->n * 32), 256>>>(g->n, g->off.p, g->adj.p, o.p);
    GPM_LAUNCH_CHECK();
  }
  unsigned long long h[2];
  GPM_CUDA(cudaMemcpy(h, o.p, 16, cudaMemcpyDeviceToHost));
  if (wedge_work) *wedge_work = h[0];
  if (pair_work) *pair_work = h[1];
  return GPM_OK;
}

}  // extern "C"
