// Mirrors test/test_trianglecounting.cu: v-centric triangle count of an .mtx graph.
#include <iostream>

#include "antirf/antirf.h"
using namespace project_AntiRF;

int main(int argc, char *argv[]) {
  if (argc < 2) {
    std::cerr << "Usage: " << argv[0] << " <graph_path>" << std::endl;
    return 1;
  }
  Loader<int, int> loader;
  Graph<int, int> hg;
  loader.Load(argv[1], "mtx");
  loader.Build(hg);
  Engine<int, int> engine(hg, 1, TC, v_centric);
  uint64_t r = engine.RunTC();
  std::cout << "Num of Patterns: 1\nPattern 0: " << r << "\n";
  return 0;
}
