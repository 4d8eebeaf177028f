// host.cu -- host-side parts of libgpm: error state, file readers that follow
// the reference loaders, and the seeded generators (host copies of the same
// counter-based draws the device generator makes).
#include <omp.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

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
// .mtx as the reference loader reads it (Loader::_load_mtx, io.h:84-139):
// skip lines until one starts with a digit; three header integers; then a
// stream of integers read in pairs (whitespace, newlines included, separates
// them), the rest of the second one's line ignored; a pair whose line has no
// terminating newline ends the stream unread; self-loops dropped; ids shifted
// by the smallest id, n = largest - smallest + 1.  Where the reference's
// stream fails (a non-integer or out-of-range token) it stops reading; so
// does this parser (the reference may then append one stale pair; this one
// does not).
namespace {

struct MtxParse {
  std::vector<int32_t> src, dst;
  int64_t n = 0;
  int32_t vmin = 0;
};

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// one integer token at p (istream >> int): optional sign, digits; false if
// none or out of int range
inline bool parse_int(const char *&p, const char *end, int64_t &v) {
  const char *q = p;
  bool neg = false;
  if (q < end && (*q == '+' || *q == '-')) neg = *q++ == '-';
  if (q >= end || *q < '0' || *q > '9') return false;
  int64_t x = 0;
  while (q < end && *q >= '0' && *q <= '9') {
    x = x * 10 + (*q++ - '0');
    if (x > (int64_t)std::numeric_limits<int32_t>::max() + 1) return false;
  }
  x = neg ? -x : x;
  if (x > std::numeric_limits<int32_t>::max() || x < std::numeric_limits<int32_t>::min()) return false;
  v = x;
  p = q;
  return true;
}

// the exact token stream from p (after the header) to end
void mtx_stream(const char *p, const char *end, std::vector<std::pair<int32_t, int32_t>> &out) {
  while (true) {
    int64_t a, b;
    while (p < end && is_ws(*p)) ++p;
    if (!parse_int(p, end, a)) return;
    while (p < end && is_ws(*p)) ++p;
    if (!parse_int(p, end, b)) return;
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    if (!nl) return;  // the reference hits end of file while skipping: pair dropped
    p = nl + 1;
    if (a != b) out.emplace_back((int32_t)a, (int32_t)b);
  }
}

// lines [p, end) (whole lines) that each start with "int int": the fast path.
// false as soon as one does not, for the exact stream to take over.
bool mtx_lines(const char *p, const char *end, std::vector<std::pair<int32_t, int32_t>> &out) {
  while (p < end) {
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    if (!nl) return false;
    int64_t a, b;
    while (p < nl && (*p == ' ' || *p == '\t')) ++p;
    if (!parse_int(p, nl, a)) return false;
    if (p >= nl || (*p != ' ' && *p != '\t')) return false;
    while (p < nl && (*p == ' ' || *p == '\t')) ++p;
    if (!parse_int(p, nl, b)) return false;
    if (p < nl && !is_ws(*p)) return false;
    if (a != b) out.emplace_back((int32_t)a, (int32_t)b);
    p = nl + 1;
  }
  return true;
}

// read-only mapping of a whole file (the threads fault its pages in parallel)
struct MappedFile {
  const char *p = nullptr;
  size_t len = 0;
  ~MappedFile() {
    if (p && len) munmap((void *)p, len);
  }
};

int mtx_parse(const char *path, MtxParse &res) {
  MappedFile mf;
  {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return fail(GPM_EIO, std::string("cannot open file ") + path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
      close(fd);
      return fail(GPM_EIO, std::string("cannot stat ") + path);
    }
    mf.len = (size_t)st.st_size;
    if (mf.len > 0) {
      void *m = mmap(nullptr, mf.len, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m == MAP_FAILED) {
        close(fd);
        mf.len = 0;
        return fail(GPM_EIO, std::string("cannot map ") + path);
      }
      mf.p = (const char *)m;
      madvise(m, mf.len, MADV_WILLNEED);
    }
    close(fd);
  }
  const char *p = mf.p, *end = mf.p + mf.len;
  // comment lines: until one starts with a digit (a file with none would make
  // the reference loop forever; here it is an error)
  while (p < end && !(*p >= '0' && *p <= '9')) {
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    p = nl ? nl + 1 : end;
  }
  int64_t h[3];
  for (int i = 0; i < 3; ++i) {
    while (p < end && is_ws(*p)) ++p;
    if (!parse_int(p, end, h[i])) return fail(GPM_EIO, std::string("bad mtx header in ") + path);
  }
  // the first pair may share the header's line; everything from the next
  // line start is split over threads at line boundaries
  std::vector<std::pair<int32_t, int32_t>> head;
  const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
  const char *body = nl ? nl + 1 : end;
  bool exact = false;
  {
    const char *q = p;
    while (q < body && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
    if (q < body && *q != '\n') exact = true;  // tokens after the header on its line
  }
  const int T = std::max(1, omp_get_max_threads());
  std::vector<std::vector<std::pair<int32_t, int32_t>>> part(T);
  std::vector<const char *> cut(T + 1);
  if (!exact) {
    const size_t len = (size_t)(end - body);
    cut[0] = body;
    cut[T] = end;
    for (int t = 1; t < T; ++t) {
      const char *c = body + len * t / T;
      const char *q = c > body ? (const char *)memchr(c - 1, '\n', (size_t)(end - (c - 1))) : body;
      cut[t] = q ? std::max(q + 1, cut[t - 1]) : end;
      if (cut[t] > end) cut[t] = end;
    }
    // the last chunk may end without a newline: the exact rule handles it
    int bad = 0;
#pragma omp parallel for num_threads(T) reduction(| : bad) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
      const char *c0 = cut[t], *c1 = cut[t + 1];
      part[t].reserve((size_t)(c1 - c0) / 8 + 16);  // lines are at least 4 bytes
      if (t == T - 1) {
        // whole lines only; an unterminated tail goes through the stream
        const char *last = c1;
        while (last > c0 && last[-1] != '\n') --last;
        if (!mtx_lines(c0, last, part[t])) bad = 1;
        else {
          std::vector<std::pair<int32_t, int32_t>> tail;
          mtx_stream(last, c1, tail);
          part[t].insert(part[t].end(), tail.begin(), tail.end());
        }
      } else if (!mtx_lines(c0, c1, part[t])) {
        bad = 1;
      }
    }
    exact = bad != 0;
  }
  if (exact) {
    for (auto &v : part) std::vector<std::pair<int32_t, int32_t>>().swap(v);
    mtx_stream(p, end, part[0]);
  }
  // every thread shifts its own part into place
  std::vector<int64_t> at(T + 1, 0);
  for (int t = 0; t < T; ++t) at[t + 1] = at[t] + (int64_t)part[t].size();
  const int64_t m = at[T];
  int64_t vmin = std::numeric_limits<int64_t>::max(), vmax = std::numeric_limits<int64_t>::min();
#pragma omp parallel for num_threads(T) reduction(min : vmin) reduction(max : vmax) schedule(static, 1)
  for (int t = 0; t < T; ++t)
    for (auto &e : part[t]) {
      vmin = std::min<int64_t>(vmin, std::min(e.first, e.second));
      vmax = std::max<int64_t>(vmax, std::max(e.first, e.second));
    }
  if (m == 0) {
    vmin = 0;
    vmax = -1;
  }
  res.n = vmax - vmin + 1;
  res.vmin = (int32_t)vmin;
  res.src.resize(m);
  res.dst.resize(m);
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t) {
    int64_t k = at[t];
    for (auto &e : part[t]) {
      res.src[k] = (int32_t)(e.first - vmin);
      res.dst[k++] = (int32_t)(e.second - vmin);
    }
    std::vector<std::pair<int32_t, int32_t>>().swap(part[t]);
  }
  return GPM_OK;
}

// the last parse of this thread, so the two-call pattern reads a file once
thread_local std::string tl_mtx_path;
thread_local long long tl_mtx_stamp = -1;
thread_local MtxParse tl_mtx;

long long file_stamp(const char *path) {
  struct stat st;
  if (stat(path, &st) != 0) return -1;
  return (long long)st.st_size * 1000003ll + (long long)st.st_mtime;
}

}  // namespace

int gpm_read_mtx(const char *path, int64_t *n, int64_t *m, int32_t *src, int32_t *dst,
                 int64_t cap, int32_t *vmin_out) {
  if (!path || !n || !m) return fail(GPM_EINVAL, "gpm_read_mtx: NULL argument");
  const long long stamp = file_stamp(path);
  if (!(tl_mtx_stamp >= 0 && stamp == tl_mtx_stamp && tl_mtx_path == path)) {
    tl_mtx = MtxParse();
    tl_mtx_stamp = -1;
    GPM_TRY(mtx_parse(path, tl_mtx));
    tl_mtx_path = path;
    tl_mtx_stamp = stamp;
  }
  const int64_t me = (int64_t)tl_mtx.src.size();
  *n = tl_mtx.n;
  *m = me;
  if (vmin_out) *vmin_out = tl_mtx.vmin;
  if (src) {
    if (!dst || cap < me) return fail(GPM_EINVAL, "gpm_read_mtx: buffer too small");
    memcpy(src, tl_mtx.src.data(), sizeof(int32_t) * me);
    memcpy(dst, tl_mtx.dst.data(), sizeof(int32_t) * me);
    tl_mtx = MtxParse();  // handed over: the cache is dropped
    tl_mtx_stamp = -1;
  }
  return GPM_OK;
}

// ---- binary CSR (the layout scripts/gbin_reader/greader.h:229-268 writes):
// <prefix>/graph.vertex.bin  int64 offsets, n + 1 of them
// <prefix>/graph.edge.bin    int32 targets, ne of them
// <prefix>/graph.meta.txt    "n\nne\n4\nmax_degree\n" (4 = bytes of an id)
namespace {
bool read_meta(const std::string &prefix, int64_t &n, int64_t &ne, int64_t &bytes, int64_t &maxd) {
  std::ifstream in(prefix + "/graph.meta.txt");
  return (bool)(in >> n >> ne >> bytes >> maxd);
}
long long file_size(const std::string &path) {
  struct stat st;
  return stat(path.c_str(), &st) == 0 ? (long long)st.st_size : -1;
}
}  // namespace

int gpm_read_gbin(const char *prefix, int64_t *n, int64_t *nnz, int64_t *offsets, int32_t *indices,
                  int32_t *max_degree) {
  if (!prefix || !n || !nnz) return fail(GPM_EINVAL, "gpm_read_gbin: NULL argument");
  const std::string pre(prefix);
  int64_t vn, ne, bytes, maxd;
  if (!read_meta(pre, vn, ne, bytes, maxd)) return fail(GPM_EIO, "cannot read " + pre + "/graph.meta.txt");
  if (bytes != 4 || vn < 0 || ne < 0) return fail(GPM_EIO, "unsupported graph.meta.txt in " + pre);
  const std::string vp = pre + "/graph.vertex.bin", ep = pre + "/graph.edge.bin";
  if (file_size(vp) != 8 * (vn + 1) || file_size(ep) != 4 * ne)
    return fail(GPM_EIO, "graph.vertex.bin / graph.edge.bin sizes do not match graph.meta.txt in " + pre);
  *n = vn;
  *nnz = ne;
  if (max_degree) *max_degree = (int32_t)maxd;
  if (!offsets && !indices) return GPM_OK;
  if (!offsets || !indices) return fail(GPM_EINVAL, "gpm_read_gbin: offsets and indices go together");
  FILE *fv = fopen(vp.c_str(), "rb");
  FILE *fe = fopen(ep.c_str(), "rb");
  bool ok = fv && fe && fread(offsets, 8, (size_t)(vn + 1), fv) == (size_t)(vn + 1) &&
            fread(indices, 4, (size_t)ne, fe) == (size_t)ne;
  if (fv) fclose(fv);
  if (fe) fclose(fe);
  if (!ok) return fail(GPM_EIO, "short read of the binary graph in " + pre);
  if (offsets[0] != 0 || offsets[vn] != ne) return fail(GPM_EIO, "graph.vertex.bin is not a CSR offset array");
  for (int64_t i = 0; i < vn; ++i)
    if (offsets[i + 1] < offsets[i]) return fail(GPM_EIO, "graph.vertex.bin offsets decrease");
  for (int64_t k = 0; k < ne; ++k)
    if (indices[k] < 0 || indices[k] >= vn) return fail(GPM_EIO, "graph.edge.bin holds an id out of range");
  return GPM_OK;
}

int gpm_write_gbin(const char *prefix, int64_t n, const int64_t *offsets, const int32_t *indices) {
  if (!prefix || !offsets || n < 0 || (offsets[n] > 0 && !indices)) return fail(GPM_EINVAL, "gpm_write_gbin: bad argument");
  const std::string pre(prefix);
  mkdir(prefix, 0777);  // as the converter does when the directory is missing
  const int64_t ne = offsets[n];
  int64_t maxd = 0;
  for (int64_t i = 0; i < n; ++i) maxd = std::max(maxd, offsets[i + 1] - offsets[i]);
  FILE *fv = fopen((pre + "/graph.vertex.bin").c_str(), "wb");
  FILE *fe = fopen((pre + "/graph.edge.bin").c_str(), "wb");
  FILE *fm = fopen((pre + "/graph.meta.txt").c_str(), "w");
  bool ok = fv && fe && fm && fwrite(offsets, 8, (size_t)(n + 1), fv) == (size_t)(n + 1) &&
            (ne == 0 || fwrite(indices, 4, (size_t)ne, fe) == (size_t)ne) &&
            fprintf(fm, "%lld\n%lld\n4\n%lld\n", (long long)n, (long long)ne, (long long)maxd) > 0;
  if (fv) ok = (fclose(fv) == 0) && ok;
  if (fe) ok = (fclose(fe) == 0) && ok;
  if (fm) ok = (fclose(fm) == 0) && ok;
  return ok ? GPM_OK : fail(GPM_EIO, "cannot write the binary graph to " + pre);
}

// The converter of scripts/gbin_reader (greader.h:129-268), with its own
// rules, which differ from the loader's: "n n ne" read first, then every line
// split at single spaces and kept only when it has exactly two tokens;
// self-loops kept; ids shifted by the smallest id, n = largest - smallest + 1;
// each vertex's list in file order.  (A comment line makes the original read
// its header as zeros and loop forever; here it is an error.)
int gpm_convert_mtx_gbin(const char *mtx_path, const char *prefix) {
  if (!mtx_path || !prefix) return fail(GPM_EINVAL, "gpm_convert_mtx_gbin: NULL argument");
  std::ifstream in(mtx_path);
  if (!in.good()) return fail(GPM_EIO, std::string("cannot open file ") + mtx_path);
  long long h0, h1, h2;
  if (!(in >> h0 >> h1 >> h2)) return fail(GPM_EIO, std::string("no \"n n ne\" header in ") + mtx_path);
  std::vector<std::pair<int64_t, int64_t>> edges;
  std::string line;
  int64_t vmin = std::numeric_limits<int32_t>::max(), vmax = std::numeric_limits<int32_t>::min();
  while (std::getline(in, line)) {
    std::vector<std::string> tok;
    size_t a = 0;
    while (a <= line.size()) {
      size_t b = line.find(' ', a);
      if (b == std::string::npos) b = line.size();
      if (b > a) tok.push_back(line.substr(a, b - a));
      a = b + 1;
    }
    if (tok.size() != 2) continue;
    char *e0, *e1;
    const long long v0 = strtoll(tok[0].c_str(), &e0, 10), v1 = strtoll(tok[1].c_str(), &e1, 10);
    if (e0 == tok[0].c_str() || e1 == tok[1].c_str()) return fail(GPM_EIO, "non-numeric edge line: " + line);
    vmin = std::min<int64_t>(vmin, std::min(v0, v1));
    vmax = std::max<int64_t>(vmax, std::max(v0, v1));
    edges.emplace_back(v0, v1);
  }
  const int64_t n = edges.empty() ? 0 : vmax - vmin + 1, ne = (int64_t)edges.size();
  std::vector<int64_t> off(n + 1, 0);
  for (auto &e : edges) ++off[e.first - vmin + 1];
  for (int64_t i = 0; i < n; ++i) off[i + 1] += off[i];
  std::vector<int64_t> fill(off.begin(), off.end() - (n >= 0 ? 1 : 0));
  std::vector<int32_t> idx(ne);
  for (auto &e : edges) idx[fill[e.first - vmin]++] = (int32_t)(e.second - vmin);
  return gpm_write_gbin(prefix, n, off.data(), idx.data());
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
