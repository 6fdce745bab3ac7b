// facade_check.cc -- drives the C++ facade (rdmce_b200/csrc/rdmce_graph.h) the
// way host code written against the reference's Graph / MceGpuSolver classes
// (include/graph.h:12-52, include/mce_gpu.cuh:15-24) would, and checks the
// results.  Built and run by tests/test_gpu_boundary.py.
//
//   facade_check <coo.txt> <scratch dir> <expected count>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "rdmce_graph.h"

#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 4) return 2;
  const std::string coo = argv[1], dir = argv[2];
  const unsigned long long want = std::strtoull(argv[3], nullptr, 10);
  rdmce::Graph g;
  g.LoadFromFile(coo);
  g.SortByOrder(rdmce::OrderType::DEG);
  rdmce::MceGpuSolver s(g, 0);
  s.Solve();
  CHECK(s.mce_count_ == want);
  CHECK(s.result_.count == want);
  unsigned long long hist_total = 0;
  for (int k = 0; k < MCE_HIST_LEN; k++) hist_total += s.result_.hist[k];
  CHECK(hist_total == want);

  // host CSR, as Graph::ConvertToCsr fills it
  g.ConvertToCsr();
  CHECK(g.GetRowOffset() != nullptr);
  CHECK(g.GetRowOffset()[g.GetNumVertices()] == 2 * g.GetNumEdges());

  // .bin round trip: StoreIntoBin writes <name>.bin next to the given path
  g.StoreIntoBin(dir + "/facade.txt");
  rdmce::Graph h;
  h.LoadFromBin(dir + "/facade.bin");
  CHECK(h.GetNumVertices() == g.GetNumVertices());
  CHECK(h.GetNumEdges() == g.GetNumEdges());
  CHECK(h.GetDegeneracy() == g.GetDegeneracy());
  rdmce::MceGpuSolver s2(h, 0);
  s2.Solve();
  CHECK(s2.mce_count_ == want);
  CHECK(s2.result_.checksum == s.result_.checksum);

  // errors are exceptions, not exit()
  bool threw = false;
  try {
    rdmce::Graph bad;
    bad.LoadFromBin(dir + "/does_not_exist.bin");
    bad.Handle();
  } catch (const rdmce::Error &e) {
    threw = e.status == MCE_ERR_IO || e.status == MCE_ERR_FORMAT;
  }
  CHECK(threw);
  std::printf("FACADE OK count %llu checksum %016llx\n", (unsigned long long)s.mce_count_,
              (unsigned long long)s.result_.checksum);
  return 0;
}
