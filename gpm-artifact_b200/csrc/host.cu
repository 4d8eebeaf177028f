// host.cu -- host-side parts of libgpm: error state, file readers that follow
// the reference loaders, and the seeded generators (host copies of the same
// counter-based draws the device generator makes).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

namespace gpm {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int status, const std::string &msg) {
  g_last_error = msg;
  return status;
}

// ------------------------------------------------------------------ device pool
struct Arena {
  std::multimap<size_t, void *> free_blocks;  // size -> block
  int device = -1;
  ~Arena() {
    for (auto &b : free_blocks) cudaFree(b.second);
  }
};

static thread_local Arena *tl_active = nullptr;
static thread_local Arena tl_arena;

Arena *current_arena() { return tl_active; }

void *arena_get(Arena *a, size_t bytes, size_t *cap) {
  const size_t gran = (size_t)1 << 18;  // 256 KiB granules keep reuse likely
  size_t want = (bytes + gran - 1) / gran * gran;
  auto it = a->free_blocks.lower_bound(want);
  if (it != a->free_blocks.end() && it->first <= 2 * want + ((size_t)8 << 20)) {
    void *p = it->second;
    *cap = it->first;
    a->free_blocks.erase(it);
    return p;
  }
  void *p = nullptr;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    // give the cached blocks back and retry once
    for (auto &b : a->free_blocks) cudaFree(b.second);
    a->free_blocks.clear();
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  *cap = want;
  return p;
}

void arena_put(Arena *a, void *p, size_t cap) { a->free_blocks.emplace(cap, p); }

ArenaScope::ArenaScope() : prev(tl_active) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (tl_arena.device != dev) {  // blocks belong to one device
    for (auto &b : tl_arena.free_blocks) cudaFree(b.second);
    tl_arena.free_blocks.clear();
    tl_arena.device = dev;
  }
  tl_active = &tl_arena;
}
ArenaScope::~ArenaScope() { tl_active = prev; }

int ensure_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(GPM_ENODEV, "no CUDA device available");
  }
  return GPM_OK;
}

ChungLu chung_lu_params(int64_t n, double gamma, double mean_deg) {
  // Weight profile w_i ~ (i + i0)^(-alpha), alpha = 1/(gamma-1).  i0 is set
  // so the largest expected degree is the structural cut-off sqrt(n * mean).
  ChungLu p;
  p.n = n;
  p.alpha = 1.0 / (gamma - 1.0);
  double target = std::sqrt((double)n * mean_deg);
  double lo = 0.0, hi = (double)n;
  for (int it = 0; it < 100; ++it) {
    double i0 = 0.5 * (lo + hi);
    // mean-normalised weight of vertex 0: n * (i0^-a) / integral_0^n (x+i0)^-a dx
    double a1 = 1.0 - p.alpha;
    double integral = (std::pow((double)n + i0, a1) - std::pow(i0, a1)) / a1;
    double w0 = mean_deg * (double)n * std::pow(i0, -p.alpha) / integral;
    if (w0 > target) lo = i0; else hi = i0;
  }
  p.i0 = std::max(0.5 * (lo + hi), 1e-9);
  double a1 = 1.0 - p.alpha;
  p.lo = std::pow(p.i0, a1);
  p.span = std::pow((double)n + p.i0, a1) - p.lo;
  p.inv = 1.0 / a1;
  return p;
}

}  // namespace gpm

using namespace gpm;

extern "C" {

const char *gpm_last_error(void) { return g_last_error.c_str(); }
int gpm_abi_version(void) { return GPM_ABI_VERSION; }

int gpm_device_count(int *count) {
  if (!count) return fail(GPM_EINVAL, "count is NULL");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return GPM_OK;
}

// ------------------------------------------------------------------ readers
int gpm_read_mtx(const char *path, int64_t *n, int64_t *m, int32_t *src, int32_t *dst,
                 int64_t cap, int32_t *vmin_out) {
  if (!path || !n || !m) return fail(GPM_EINVAL, "gpm_read_mtx: NULL argument");
  FILE *f = fopen(path, "r");
  if (!f) return fail(GPM_EIO, std::string("cannot open file ") + path);
  // skip comment lines until a line that starts with a digit (io.h:89-95)
  int c;
  while ((c = fgetc(f)) != EOF) {
    if (c >= '0' && c <= '9') {
      ungetc(c, f);
      break;
    }
    while (c != '\n' && c != EOF) c = fgetc(f);
  }
  long long h0 = 0, h1 = 0, h2 = 0;
  if (fscanf(f, "%lld %lld %lld", &h0, &h1, &h2) != 3) {
    fclose(f);
    return fail(GPM_EIO, std::string("bad mtx header in ") + path);
  }
  std::vector<std::pair<int64_t, int64_t>> edges;
  edges.reserve((size_t)std::max<long long>(h2, 0));
  int64_t vmin = std::numeric_limits<int64_t>::max(), vmax = std::numeric_limits<int64_t>::min();
  char line[512];
  // finish the header line
  if (!fgets(line, sizeof line, f)) line[0] = 0;
  while (fgets(line, sizeof line, f)) {
    long long a, b;
    if (sscanf(line, "%lld %lld", &a, &b) != 2) continue;
    // The reference stops when the stream hits EOF right after a pair, so an
    // unterminated last line is not read (io.h:111-114); keep that.
    size_t len = strlen(line);
    if (len == 0 || line[len - 1] != '\n') break;
    if (a == b) continue;  // self-loops dropped (io.h:115-116)
    vmin = std::min<int64_t>(vmin, std::min<int64_t>(a, b));
    vmax = std::max<int64_t>(vmax, std::max<int64_t>(a, b));
    edges.emplace_back(a, b);
  }
  fclose(f);
  if (edges.empty()) {
    vmin = 0;
    vmax = -1;
  }
  *n = vmax - vmin + 1;
  *m = (int64_t)edges.size();
  if (vmin_out) *vmin_out = (int32_t)vmin;
  if (src) {
    if (!dst || cap < (int64_t)edges.size()) return fail(GPM_EINVAL, "gpm_read_mtx: buffer too small");
    for (size_t i = 0; i < edges.size(); ++i) {
      src[i] = (int32_t)(edges[i].first - vmin);
      dst[i] = (int32_t)(edges[i].second - vmin);
    }
  }
  return GPM_OK;
}

int gpm_read_labels(const char *path, int64_t n, int32_t vmin, int32_t *labels) {
  if (!path || !labels) return fail(GPM_EINVAL, "gpm_read_labels: NULL argument");
  if (strncmp(path, "random", 6) == 0) {  // io.h:41-47
    long range = strtol(path + 6, nullptr, 10);
    if (range <= 0) return fail(GPM_EINVAL, "random<N> needs N > 0");
    for (int64_t i = 0; i < n; ++i) labels[i] = (int32_t)(rand() % range);
    return GPM_OK;
  }
  FILE *f = fopen(path, "r");
  if (!f) return fail(GPM_EIO, std::string("cannot open ") + path);
  std::vector<std::pair<int64_t, int32_t>> tmp;
  char line[256];
  while (fgets(line, sizeof line, f)) {
    long long v;
    int lab;
    if (sscanf(line, "%lld %d", &v, &lab) != 2) continue;
    tmp.emplace_back(v, lab);
  }
  fclose(f);
  if ((int64_t)tmp.size() != n) return fail(GPM_EINVAL, "vertex size not match");  // io.h:64-66
  for (auto &p : tmp) {
    int64_t v = p.first - vmin;
    if (v < 0 || v >= n) return fail(GPM_EINVAL, "label vertex id out of range");
    labels[v] = p.second;
  }
  return GPM_OK;
}

int gpm_read_tve(const char *path, int64_t *n, int64_t *m, int32_t *labels, int32_t *src,
                 int32_t *dst, int64_t cap) {
  if (!path || !n || !m) return fail(GPM_EINVAL, "gpm_read_tve: NULL argument");
  std::ifstream in(path);
  if (!in.is_open()) return fail(GPM_EIO, std::string("cannot open ") + path);
  std::string line;
  std::vector<std::pair<int64_t, int32_t>> vs;
  std::vector<std::pair<int32_t, int32_t>> es;
  int64_t maxv = -1;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string t;
    if (!(ss >> t)) continue;
    if (t == "v") {
      long long id;
      long long lab = 0;
      if (!(ss >> id)) continue;
      ss >> lab;
      vs.emplace_back(id, (int32_t)lab);
      maxv = std::max<int64_t>(maxv, id);
    } else if (t == "e") {
      long long a, b;
      if (!(ss >> a >> b)) continue;
      es.emplace_back((int32_t)a, (int32_t)b);
    }
  }
  *n = maxv + 1;
  *m = (int64_t)es.size();
  if (labels) {
    for (int64_t i = 0; i <= maxv; ++i) labels[i] = 0;
    for (auto &p : vs) labels[p.first] = p.second;
  }
  if (src) {
    if (!dst || cap < (int64_t)es.size()) return fail(GPM_EINVAL, "gpm_read_tve: buffer too small");
    for (size_t i = 0; i < es.size(); ++i) {
      src[i] = es[i].first;
      dst[i] = es[i].second;
    }
  }
  return GPM_OK;
}

// ------------------------------------------------------------------ generators
int gpm_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                 int32_t *src, int32_t *dst) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || !src || !dst)
    return fail(GPM_EINVAL, "gpm_gen_rmat: bad arguments");
  int64_t m = ((int64_t)1 << scale) * edge_factor;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) rmat_edge(seed, (uint64_t)i, scale, a, b, c, &src[i], &dst[i]);
  return GPM_OK;
}

int gpm_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t *src, int32_t *dst) {
  if (n < 1 || n >= (1ll << 31) || m < 0 || !src || !dst) return fail(GPM_EINVAL, "gpm_gen_er: bad arguments");
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) er_edge(seed, (uint64_t)i, n, &src[i], &dst[i]);
  return GPM_OK;
}

int gpm_gen_chung_lu(int64_t n, double gamma, double mean_deg, uint64_t seed, int64_t *m,
                     int32_t *src, int32_t *dst) {
  if (n < 2 || gamma <= 2.0 || mean_deg <= 0 || !m) return fail(GPM_EINVAL, "gpm_gen_chung_lu: bad arguments");
  int64_t mm = (int64_t)llround((double)n * mean_deg / 2.0);
  *m = mm;
  if (!src) return GPM_OK;
  if (!dst) return fail(GPM_EINVAL, "gpm_gen_chung_lu: dst is NULL");
  ChungLu p = chung_lu_params(n, gamma, mean_deg);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < mm; ++i) {
    src[i] = chung_lu_vertex(p, draw(seed, 201, (uint64_t)i));
    dst[i] = chung_lu_vertex(p, draw(seed, 202, (uint64_t)i));
  }
  return GPM_OK;
}

int gpm_gen_zipf_labels(int64_t n, int nlabels, double s, uint64_t seed, int32_t *labels) {
  if (n < 0 || nlabels < 1 || !labels) return fail(GPM_EINVAL, "gpm_gen_zipf_labels: bad arguments");
  std::vector<double> cdf(nlabels);
  double tot = 0;
  for (int k = 0; k < nlabels; ++k) tot += 1.0 / std::pow((double)(k + 1), s);
  double acc = 0;
  for (int k = 0; k < nlabels; ++k) {
    acc += 1.0 / std::pow((double)(k + 1), s) / tot;
    cdf[k] = acc;
  }
  cdf[nlabels - 1] = 1.0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double r = unit(draw(seed, 301, (uint64_t)i));
    int k = 0;
    while (k < nlabels - 1 && r >= cdf[k]) ++k;
    labels[i] = k;
  }
  return GPM_OK;
}

}  // extern "C"
