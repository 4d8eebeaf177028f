// Driver for the reference's CFSolver (src/CFSolver.cuh:99-158), which ships
// without one: load an .mtx graph, orient it (Graph::orientation), count
// k-cliques edge-centrically.  Test infrastructure, built into oracle/_ref.
#include <chrono>
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
  // the reference times nothing here: the whole call is timed, including its
  // own device copy of the graph and frontier allocation
  const auto t0 = std::chrono::steady_clock::now();
  CFSolver(hg, std::atoi(argv[2]), result, 1, project_AntiRF::e_centric);
  const auto t1 = std::chrono::steady_clock::now();
  std::cout << "Result: " << result << std::endl;
  std::cout << "CFSolver call time: " << std::chrono::duration<double>(t1 - t0).count() << " seconds" << std::endl;
  return 0;
}
