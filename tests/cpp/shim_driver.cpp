// A driver written the way the reference's Algorithms/BFS/bfs.cu:436-477 and
// Algorithms/PageRank/PageRank.cu drive the engine (CsrProblem +
// EnactorVertexCentric + ExtractResults), compiled against the C++ shim
// mapgraph_b200_gas.hpp. Usage: shim_driver <bfs|sssp|cc|pagerank> <graph.mtx> <src>
// Prints one result per line.
#include <cstdio>
#include <cstring>
#include <vector>

#include "mapgraph_b200_gas.hpp"
#include "mapgraph_b200_io.h"

template <typename Program, typename Value>
static int run(const mg_host_csr &g, int src, Value *vals) {
  typedef GASengine::CsrProblem<Program, int, int, Value, false, true> CsrProblem;
  GASengine::Config cfg;
  CsrProblem csr_problem(cfg);
  if (csr_problem.FromHostProblem(false, (int)g.n, (int)g.m, g.col_idx, g.row_offsets, vals, nullptr, nullptr, 1,
                                  1))
    return 1;
  GASengine::EnactorVertexCentric<CsrProblem, Program, true> vertex_centric(cfg, false);
  int srcs[1] = {src};
  if (vertex_centric.EnactIterativeSearch(csr_problem, g.row_offsets, 1, 1, srcs,
                                          cfg.getParameter<int>("iter_num"), cfg.getParameter<int>("threshold"))) {
    std::fprintf(stderr, "%s\n", mg_last_error());
    return 1;
  }
  std::vector<typename Program::DataType> h_values(g.n);
  if (csr_problem.ExtractResults(h_values.data())) return 1;
  for (int64_t i = 0; i < g.n; i++) {
    if (sizeof(h_values[0]) == 4 && std::is_floating_point<typename Program::DataType>::value)
      std::printf("%.6f\n", (double)h_values[i]);
    else
      std::printf("%lld\n", (long long)h_values[i]);
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  mg_host_csr g;
  std::memset(&g, 0, sizeof(g));
  if (mg_read_market(argv[2], 0, &g) != MG_OK) return 1;
  const int src = std::atoi(argv[3]);
  int rc = 2;
  if (!std::strcmp(argv[1], "bfs")) rc = run<GASengine::bfs, int>(g, src, g.weights_i32);
  else if (!std::strcmp(argv[1], "sssp")) rc = run<GASengine::sssp, int>(g, src, g.weights_i32);
  else if (!std::strcmp(argv[1], "cc")) rc = run<GASengine::cc, int>(g, src, g.weights_i32);
  else if (!std::strcmp(argv[1], "pagerank")) rc = run<GASengine::pagerank, float>(g, src, (float *)nullptr);
  mg_host_csr_free(&g);
  return rc;
}
