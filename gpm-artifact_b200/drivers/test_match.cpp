// Labelled matching with the command line of sub_ceci (myceci.cpp:862-1119):
//   test_match -d <data.graph> -q <query.graph>   prints "#Embeddings: N"
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "gpm.h"

static void check(int s, const char *what) {
  if (s != GPM_OK) {
    std::cerr << what << ": " << gpm_last_error() << std::endl;
    std::exit(1);
  }
}

int main(int argc, char *argv[]) {
  std::string dpath, qpath;
  for (int i = 1; i + 1 < argc; ++i) {
    if (!std::strcmp(argv[i], "-d")) dpath = argv[++i];
    else if (!std::strcmp(argv[i], "-q")) qpath = argv[++i];
  }
  if (dpath.empty() || qpath.empty()) {
    std::cerr << "Usage: " << argv[0] << " -d <data.graph> -q <query.graph>" << std::endl;
    return 1;
  }
  int64_t n = 0, m = 0, qn = 0, qm = 0;
  check(gpm_read_tve(dpath.c_str(), &n, &m, nullptr, nullptr, nullptr, 0), "data graph");
  std::vector<int32_t> lab(n), s(m), d(m);
  check(gpm_read_tve(dpath.c_str(), &n, &m, lab.data(), s.data(), d.data(), m), "data graph");
  check(gpm_read_tve(qpath.c_str(), &qn, &qm, nullptr, nullptr, nullptr, 0), "query graph");
  std::vector<int32_t> qlab(qn), qs(qm), qd(qm);
  check(gpm_read_tve(qpath.c_str(), &qn, &qm, qlab.data(), qs.data(), qd.data(), qm), "query graph");
  gpm_graph *g = nullptr;
  gpm_query *q = nullptr;
  check(gpm_graph_create(n, m, s.data(), d.data(), lab.data(), GPM_SYMMETRIZE, &g), "build");
  check(gpm_query_create(qn, qm, qs.data(), qd.data(), qlab.data(), &q), "query");
  uint64_t cnt = 0;
  check(gpm_match(g, q, &cnt), "match");
  std::cout << "#Embeddings: " << cnt << std::endl;
  gpm_query_destroy(q);
  gpm_graph_destroy(g);
  return 0;
}
