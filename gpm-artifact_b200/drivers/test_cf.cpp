// k-clique driver (the reference ships CFSolver without a driver): orient, then CFSolver.
#include <cstdlib>
#include <iostream>

#include "antirf/antirf.h"
using namespace project_AntiRF;

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::cerr << "Usage: " << argv[0] << " <graph_path> <k>" << std::endl;
    return 1;
  }
  Loader<int, int> loader;
  Graph<int, int> hg;
  loader.Load(argv[1], "mtx");
  loader.Build(hg);
  hg.orientation();
  uint64_t r = 0;
  CFSolver(hg, std::atoi(argv[2]), r, 1, e_centric);
  std::cout << "Result: " << r << "\n";
  return 0;
}
