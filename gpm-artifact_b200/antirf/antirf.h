// antirf.h -- C++ drop-in for the AntiRF solver API (namespace project_AntiRF),
// implemented over the libgpm C ABI (include/gpm.h).
//
// The names, signatures and behaviour follow the reference headers:
//   enums / AccType          src/utils/utils.h:23-25
//   Pattern                  src/utils/sm_pattern.h:22-38
//   Graph                    src/graph/graph.h:88-438
//   Loader                   src/graph/io.h:20-153
//   TCSolver                 src/TCSolver.cuh:9-121
//   G2MinerSolver            src/G2MinerSolver.cuh:17-176
//   PatternSolver            src/PatternSolver.cuh:16-265
//   CFSolver                 src/CFSolver.cuh:99-158
//   Engine                   src/Engine.h:17-69
// Errors abort with a message, as the reference's LOG(FATAL) does; the C ABI
// underneath returns status codes instead.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "gpm.h"

namespace project_AntiRF {

enum algorithms { TC, SM, CF, MC, FSM };
enum modes { v_centric, e_centric };
typedef unsigned long long AccType;

inline void gpm_check(int status, const char *what) {
  if (status != GPM_OK) {
    std::fprintf(stderr, "F %s: %s\n", what, gpm_last_error());
    std::abort();
  }
}

class Pattern {
 public:
  Pattern() : Pattern("") {}
  Pattern(std::string name) : name_(std::move(name)) {}
  bool is_rectangle() const { return name_ == "rectangle"; }
  bool is_pentagon() const { return name_ == "pentagon"; }
  bool is_house() const { return name_ == "house"; }
  std::string get_name() const { return name_; }

 private:
  std::string name_;
};

template <typename VID, typename VLABEL>
class Graph {
 public:
  Graph() = default;
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;
  ~Graph() {
    if (g_) gpm_graph_destroy(g_);
  }

  // Graph::Init (graph.h:254-340): a directed CSR from the loader's edge
  // list.  Lists are sorted and duplicates dropped (see gpm_graph_create).
  void Init(std::vector<VID> const &vids, std::vector<VLABEL> const &vlabels,
            std::vector<std::pair<VID, VID>> const &edges, bool use_label = false) {
    std::vector<int32_t> s(edges.size()), d(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) {
      s[i] = (int32_t)edges[i].first;
      d[i] = (int32_t)edges[i].second;
    }
    std::vector<int32_t> lab;
    if (use_label || !vlabels.empty()) lab.assign(vlabels.begin(), vlabels.end());
    if (g_) gpm_graph_destroy(g_);
    g_ = nullptr;
    gpm_check(gpm_graph_create((int64_t)vids.size(), (int64_t)edges.size(), s.data(), d.data(),
                               lab.size() == vids.size() ? lab.data() : nullptr, 0, &g_),
              "Graph::Init");
    dirty_ = true;
  }

  // Graph::orientation (graph.h:116-204)
  void orientation(bool NeedToLoadToDevice = true) {
    (void)NeedToLoadToDevice;
    gpm_check(gpm_graph_orient(g_, 0), "Graph::orientation");
    dirty_ = true;
  }
  // Graph::SortCSRGraph (graph.h:206-252): renumber by out-degree, descending
  void SortCSRGraph(bool NeedToLoadToDevice = true) {
    (void)NeedToLoadToDevice;
    gpm_check(gpm_graph_relabel(g_), "Graph::SortCSRGraph");
    dirty_ = true;
  }

  VID get_vnum() const { return (VID)info().n; }
  VID get_enum() const { return (VID)info().nnz; }
  VID getMaxDegree() const { return (VID)info().max_degree; }
  VID getOutDegree(VID v) { sync(); return (VID)(off_[v + 1] - off_[v]); }
  VID edge_begin(VID v) { sync(); return (VID)off_[v]; }
  VID edge_end(VID v) { sync(); return (VID)off_[v + 1]; }
  VID *getNeighbor(VID v) { sync(); return adj_.data() + off_[v]; }
  gpm_graph *DeviceObject() const { return g_; }

 private:
  gpm_graph_info info() const {
    gpm_graph_info inf{};
    gpm_check(gpm_graph_get_info(g_, &inf), "Graph::info");
    return inf;
  }
  void sync() {
    if (!dirty_) return;
    gpm_graph_info inf = info();
    off_.resize(inf.n + 1);
    std::vector<int32_t> adj(inf.nnz);
    gpm_check(gpm_graph_copy_csr(g_, off_.data(), adj.data()), "Graph::copy");
    adj_.assign(adj.begin(), adj.end());
    dirty_ = false;
  }
  gpm_graph *g_ = nullptr;
  bool dirty_ = true;
  std::vector<int64_t> off_;
  std::vector<VID> adj_;
};

template <typename VID, typename VLABEL>
class Loader {
 public:
  // Loader::Load (io.h:22-33): "mtx", and "bin" -- a directory in the layout
  // of scripts/gbin_reader (graph.vertex.bin / graph.edge.bin /
  // graph.meta.txt), which the reference declares but leaves unimplemented
  // (io.h:143); its stored pairs are taken as the mtx pairs are (self-loops
  // dropped, ids already start at 0).  "txt" is unimplemented in both.
  void Load(std::string const &path, std::string const &format) {
    if (format == "bin") {
      int64_t n = 0, nnz = 0;
      gpm_check(gpm_read_gbin(path.c_str(), &n, &nnz, nullptr, nullptr, nullptr), "Loader::Load");
      std::vector<int64_t> off(n + 1);
      std::vector<int32_t> idx(nnz > 0 ? nnz : 1);
      gpm_check(gpm_read_gbin(path.c_str(), &n, &nnz, off.data(), idx.data(), nullptr), "Loader::Load");
      vsize_ = (size_t)n;
      vmin_ = 0;
      edges_.clear();
      edges_.reserve(nnz);
      for (int64_t v = 0; v < n; ++v)
        for (int64_t k = off[v]; k < off[v + 1]; ++k)
          if (idx[k] != v) edges_.push_back({(VID)v, (VID)idx[k]});
      vlabels_.clear();
      return;
    }
    if (format != "mtx") {
      std::fprintf(stderr, "F unknown or unimplemented format %s\n", format.c_str());
      std::abort();
    }
    int64_t n = 0, m = 0;
    int32_t vmin = 0;
    gpm_check(gpm_read_mtx(path.c_str(), &n, &m, nullptr, nullptr, 0, &vmin), "Loader::Load");
    std::vector<int32_t> s(m), d(m);
    gpm_check(gpm_read_mtx(path.c_str(), &n, &m, s.data(), d.data(), m, &vmin), "Loader::Load");
    vsize_ = (size_t)n;
    vmin_ = vmin;
    edges_.resize(m);
    for (int64_t i = 0; i < m; ++i) edges_[i] = {(VID)s[i], (VID)d[i]};
    vlabels_.clear();
  }
  // Loader::LoadVLabel (io.h:35-73): a "v label" file or "random<N>"
  void LoadVLabel(std::string const &path) {
    std::vector<int32_t> lab(vsize_);
    gpm_check(gpm_read_labels(path.c_str(), (int64_t)vsize_, vmin_, lab.data()), "Loader::LoadVLabel");
    vlabels_.assign(lab.begin(), lab.end());
  }
  // Loader::Build (io.h:75-81)
  void Build(Graph<VID, VLABEL> &hg) {
    std::vector<VID> vids(vsize_);
    for (size_t i = 0; i < vsize_; ++i) vids[i] = (VID)i;
    hg.Init(vids, vlabels_, edges_);
  }

 private:
  size_t vsize_ = 0;
  int32_t vmin_ = 0;
  std::vector<std::pair<VID, VID>> edges_;
  std::vector<VLABEL> vlabels_;
};

// TCSolver (TCSolver.cuh:9-121): sum over stored edges of |N(u) & N(v)|
template <typename VID, typename VLABEL>
void TCSolver(Graph<VID, VLABEL> &hg, uint64_t &result, int n_dev, modes cal_m) {
  (void)n_dev;
  if (cal_m != v_centric && cal_m != e_centric) {
    std::fprintf(stderr, "F Wrong Calculation Mode.\n");
    std::abort();
  }
  uint64_t r = 0;
  gpm_check(gpm_tc(hg.DeviceObject(), cal_m == v_centric ? GPM_V_CENTRIC : GPM_E_CENTRIC, &r), "TCSolver");
  result = r;
}

// G2MinerSolver (G2MinerSolver.cuh:17-176); counters receives all six
// counters (the reference only logs them)
template <typename VID, typename VLABEL>
void G2MinerSolver(Graph<VID, VLABEL> &hg, uint64_t &result, int n_dev, modes cal_m, Pattern p,
                   std::vector<uint64_t> *counters = nullptr) {
  (void)n_dev;
  (void)cal_m;
  uint64_t c[6], r = 0;
  gpm_check(gpm_pattern(hg.DeviceObject(), p.get_name().c_str(), GPM_G2MINER, c, &r), "G2MinerSolver");
  result = r;
  if (counters) counters->assign(c, c + 6);
}

// PatternSolver (PatternSolver.cuh:16-265)
template <typename VID, typename VLABEL>
void PatternSolver(Graph<VID, VLABEL> &hg, uint64_t &result, int n_dev, modes cal_m, Pattern p,
                   std::vector<uint64_t> *counters = nullptr) {
  (void)n_dev;
  (void)cal_m;
  uint64_t c[6], r = 0;
  gpm_check(gpm_pattern(hg.DeviceObject(), p.get_name().c_str(), GPM_PATTERN_SOLVER, c, &r), "PatternSolver");
  result = r;
  if (counters) counters->assign(c, c + 6);
}

// CFSolver (CFSolver.cuh:99-158): the caller orients first; the reference's
// v_centric branch is empty and leaves the result at 0
template <typename VID, typename VLABEL>
void CFSolver(Graph<VID, VLABEL> &hg, int k, uint64_t &result, int n_dev, modes cal_m) {
  (void)n_dev;
  if (k <= 3) {
    std::fprintf(stderr, "F Assertion failed: k > 3\n");
    std::abort();
  }
  if (cal_m == v_centric) {
    result = 0;
    return;
  }
  uint64_t r = 0;
  gpm_check(gpm_clique(hg.DeviceObject(), k, &r), "CFSolver");
  result = r;
}

template <typename VID, typename VLABEL>
class Engine {
 public:
  Engine(Graph<VID, VLABEL> &hg, int n_dev, algorithms al, modes cal_m)
      : hg_(hg), n_devices(n_dev), algo(al), cal_mode(cal_m) {}
  Engine(Graph<VID, VLABEL> &hg, int n_dev, algorithms al, modes cal_m, int k)
      : hg_(hg), n_devices(n_dev), algo(al), cal_mode(cal_m), motif_k(k) {}
  Engine(Graph<VID, VLABEL> &hg, int n_dev, algorithms al, modes cal_m, Pattern p)
      : hg_(hg), n_devices(n_dev), algo(al), cal_mode(cal_m), s_pattern(p) {}

  // Engine::RunTC (Engine.h:47-56): orient (and relabel for v_centric) first
  uint64_t RunTC() {
    if (cal_mode == v_centric) {
      hg_.orientation(false);
      hg_.SortCSRGraph(true);
    } else {
      hg_.orientation();
    }
    TCSolver(hg_, result, n_devices, cal_mode);
    return result;
  }
  uint64_t RunPatternEnum() {
    PatternSolver(hg_, result, n_devices, cal_mode, s_pattern, &motif_result);
    return result;
  }
  uint64_t RunG2Miner() {
    G2MinerSolver(hg_, result, n_devices, cal_mode, s_pattern, &motif_result);
    return result;
  }
  // The six Motif4 counters of the last pattern run (logged only by the reference).
  const std::vector<uint64_t> &MotifResult() const { return motif_result; }

 private:
  Graph<VID, VLABEL> &hg_;
  uint64_t result = 0;
  int n_devices = 1;
  algorithms algo;
  modes cal_mode;
  int motif_k = 0;
  std::vector<uint64_t> motif_result;
  Pattern s_pattern;
};

}  // namespace project_AntiRF
