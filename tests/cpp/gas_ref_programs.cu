// Drives MapGraph's own bundled vertex programs (Algorithms/BFS/bfs.h,
// Algorithms/SSSP/sssp.h, Algorithms/CC/cc.h, Algorithms/PageRank/PageRank.h,
// included unchanged from the reference tree at build time) through the compat
// CsrProblem / EnactorVertexCentric, in the call order of the reference's drivers
// (Algorithms/BFS/bfs.cu:436-477). Built by oracle/build_ref.sh into oracle/_ref
// twice: with the tuned dispatch, and with -DMG_GAS_GENERIC_ONLY (every program
// on the generic kernels). Usage: <bfs|sssp|cc|pagerank> <graph.mtx> <src> <directed> <out>
// writes one value per line to <out> (the programs print to stdout themselves).
#include <cstdio>
#include <cstring>
#include <vector>

#include "GASengine/csr_problem.cuh"
#include "GASengine/enactor_vertex_centric.cuh"
#include "mapgraph_b200_io.h"

#include <Algorithms/BFS/bfs.h>
#include <Algorithms/CC/cc.h>
#include <Algorithms/PageRank/PageRank.h>
#include <Algorithms/SSSP/sssp.h>

struct NoConfig {};

template <typename Program, typename Value>
static int run(const mg_host_csr &g, Value *vals, int num_srcs, int *srcs, int directed, const char *out) {
  typedef GASengine::CsrProblem<Program, int, int, Value, false, true> CsrProblem;
  CsrProblem csr_problem{NoConfig()};
  if (csr_problem.FromHostProblem(false, (int)g.n, (int)g.m, g.col_idx, g.row_offsets, vals, nullptr, nullptr, 1,
                                  directed))
    return 1;
  GASengine::EnactorVertexCentric<CsrProblem, Program, false> vertex_centric{NoConfig()};
  if (vertex_centric.EnactIterativeSearch(csr_problem, g.row_offsets, directed, num_srcs, srcs, INT_MAX, 1000))
    return 1;
  std::vector<typename Program::DataType> h_values(g.n);
  csr_problem.ExtractResults(h_values.data());
  FILE *f = std::fopen(out, "w");
  if (!f) return 1;
  for (int64_t i = 0; i < g.n; i++) {
    if (std::is_floating_point<typename Program::DataType>::value) std::fprintf(f, "%.7f\n", (double)h_values[i]);
    else std::fprintf(f, "%lld\n", (long long)h_values[i]);
  }
  std::fclose(f);
  std::fprintf(stderr, "iterations %lld\n", vertex_centric.iteration[0]);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 6) return 2;
  mg_host_csr g;
  std::memset(&g, 0, sizeof(g));
  if (mg_read_market(argv[2], 0, &g) != MG_OK) return 1;
  int src = std::atoi(argv[3]);
  const int directed = std::atoi(argv[4]);
  int rc = 2;
  if (!std::strcmp(argv[1], "bfs")) rc = run<bfs, int>(g, g.weights_i32, 1, &src, directed, argv[5]);
  else if (!std::strcmp(argv[1], "sssp")) rc = run<sssp, int>(g, g.weights_i32, 1, &src, directed, argv[5]);
  else if (!std::strcmp(argv[1], "cc")) rc = run<cc, int>(g, g.weights_i32, (int)g.n, nullptr, 0, argv[5]);
  else if (!std::strcmp(argv[1], "pagerank")) rc = run<pagerank, float>(g, g.weights_f32, (int)g.n, nullptr, directed, argv[5]);
  mg_host_csr_free(&g);
  return rc;
}
