// Mirrors test/test_engine.cu: e-centric triangle count, labels loaded (and
// unused).  A directory as <graph_path> is read as a binary CSR ("bin").
#include <sys/stat.h>

#include <iostream>

#include "antirf/antirf.h"
using namespace project_AntiRF;

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::cerr << "Usage: " << argv[0] << " <graph_path> <graph_label>" << std::endl;
    return 1;
  }
  Loader<int, int> loader;
  Graph<int, int> hg;
  struct stat st;
  const bool dir = stat(argv[1], &st) == 0 && S_ISDIR(st.st_mode);
  loader.Load(argv[1], dir ? "bin" : "mtx");
  loader.LoadVLabel(argv[2]);
  loader.Build(hg);
  Engine<int, int> engine(hg, 1, TC, e_centric);
  std::cout << "Result: " << engine.RunTC() << "\n";
  return 0;
}
