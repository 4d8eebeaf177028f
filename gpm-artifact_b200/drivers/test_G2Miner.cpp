// Mirrors test/test_G2Miner.cu: named pattern (P1..P8 or Motif4) on the symmetric graph.
#include <iostream>

#include "antirf/antirf.h"
using namespace project_AntiRF;

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::cerr << "Usage: " << argv[0] << " <graph_path> <pattern_name>" << std::endl;
    return 1;
  }
  Pattern pattern(argv[2]);
  Loader<int, int> loader;
  Graph<int, int> hg;
  loader.Load(argv[1], "mtx");
  loader.Build(hg);
  Engine<int, int> engine(hg, 1, CF, e_centric, pattern);
  uint64_t r = engine.RunG2Miner();
  std::cout << "Result: " << r << "\n";
  if (pattern.get_name() == "Motif4")
    for (int i = 0; i < 6; ++i) std::cout << "Result" << i << ": " << engine.MotifResult()[i] << "\n";
  return 0;
}
