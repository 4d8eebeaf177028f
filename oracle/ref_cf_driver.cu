// Driver for the reference's CFSolver (src/CFSolver.cuh:99-158), which ships
// without one: load an .mtx graph, orient it (Graph::orientation), count
// k-cliques edge-centrically.  Test infrastructure, built into oracle/_ref.
#include <cstdlib>
#include <iostream>

#include "src/Engine.h"
#include "src/graph/io.h"
#include "src/CFSolver.cuh"

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::cerr << "Usage: " << argv[0] << " <graph.mtx> <k>" << std::endl;
    return 1;
  }
  project_AntiRF::Loader<int, int> loader;
  project_AntiRF::Graph<int, int> hg;
  loader.Load(argv[1], "mtx");
  loader.Build(hg);
  hg.orientation();
  uint64_t result = 0;
  CFSolver(hg, std::atoi(argv[2]), result, 1, project_AntiRF::e_centric);
  std::cout << "Result: " << result << std::endl;
  return 0;
}
