// Test infrastructure (the checker): a C ABI around the reference's own serial
// CPU correctness functions. Compiled only by oracle/build_ref.sh, which cuts the
// function bodies out of the reference drivers into oracle/_ref/*.inc; the
// reference's Matrix Market reader and CsrGraph come from the reference tree
// through -I. Output goes to oracle/_ref/libmgref.so only.
//
// Every entry point silences the reference's console prints (they go to stdout)
// and returns the wall time of the wrapped call in seconds, measured with
// std::chrono::steady_clock (the reference's own time(NULL) prints have a
// resolution of one second).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>
#include <cmath>
#include <chrono>
#include <deque>
#include <vector>
#include <set>
#include <numeric>
#include <iostream>
#include <string>
#include <algorithm>
#include <unistd.h>
#include <fcntl.h>

#include <cuda_runtime.h>
#include <b40c/graph/builder/market.cuh>

using namespace b40c;
using namespace graph;
using namespace std;

// The two constants the extracted functions read from the vertex-program structs
// (Algorithms/SSSP/sssp.h:43, Algorithms/CC/cc.h:41).
struct sssp { typedef int DataType; static const DataType INIT_VALUE = INT_MAX; };
struct cc { typedef int DataType; static const int INIT_VALUE = INT_MAX; };

#include "cpubfs.inc"
#include "cpusssp.inc"
#include "cpucc.inc"
#include "cpupr.inc"

namespace {

// Redirects stdout (fd 1) to a temporary file for the lifetime of the object;
// text() returns what was printed meanwhile.
struct Quiet {
  int saved;
  FILE *tmp;
  Quiet() {
    fflush(stdout);
    saved = dup(1);
    tmp = tmpfile();
    dup2(fileno(tmp), 1);
  }
  std::string text() {
    fflush(stdout);
    long len = ftell(tmp);
    std::string s(len > 0 ? (size_t)len : 0, '\0');
    rewind(tmp);
    if (len > 0) fread(&s[0], 1, (size_t)len, tmp);
    return s;
  }
  ~Quiet() {
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    fclose(tmp);
  }
};

template <typename Value>
CsrGraph<int, Value, int> view(int n, int m, const int* ro, const int* ci, const int* co,
                               const int* ri, const Value* vals) {
  CsrGraph<int, Value, int> g(false);
  g.nodes = n;
  g.edges = m;
  g.row_offsets = const_cast<int*>(ro);
  g.column_indices = const_cast<int*>(ci);
  g.column_offsets = const_cast<int*>(co);
  g.row_indices = const_cast<int*>(ri);
  g.edge_values = const_cast<Value*>(vals);
  g.node_values = NULL;
  return g;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

// CPUBFS (Algorithms/BFS/bfs.cu:56-143). co/ri (CSC) are read only when directed==0.
double mgref_bfs(int n, int m, const int* ro, const int* ci, const int* co, const int* ri,
                 int directed, int src, int* depth) {
  CsrGraph<int, int, int> g = view<int>(n, m, ro, ci, co, ri, NULL);
  Quiet q;
  auto t0 = std::chrono::steady_clock::now();
  CPUBFS<int, int, int>(directed, 1, g, depth, src);
  return seconds_since(t0);
}

// CPUSSSP (Algorithms/SSSP/sssp.cu:127-199). Unreached vertices come back as
// 100000000, the reference CPU sentinel (sssp.cu:139).
double mgref_sssp(int n, int m, const int* ro, const int* ci, const int* co, const int* ri,
                  const int* w, int directed, int src, int* dist) {
  CsrGraph<int, int, int> g = view<int>(n, m, ro, ci, co, ri, w);
  Quiet q;
  auto t0 = std::chrono::steady_clock::now();
  CPUSSSP<int, int, int>(directed != 0, g, dist, src);
  return seconds_since(t0);
}

// CPUCC (Algorithms/CC/cc.cu:132-199): min-label propagation over CSR and CSC.
double mgref_cc(int n, int m, const int* ro, const int* ci, const int* co, const int* ri,
                int* label) {
  CsrGraph<int, int, int> g = view<int>(n, m, ro, ci, co, ri, NULL);
  Quiet q;
  auto t0 = std::chrono::steady_clock::now();
  CPUCC<int, int, int>(g, label);
  return seconds_since(t0);
}

// CPUPR (Algorithms/PageRank/PageRank.cu:108-163): Gauss-Seidel sweeps of
// x = 0.15 + 0.85 * sum x_u/outdeg_u over the CSC, stopping when no |dx| >= 0.01.
// *sweeps gets the sweep count the function prints ("CPU iterations: N").
double mgref_pr(int n, int m, const int* ro, const int* ci, const int* co, const int* ri,
                float* rank, int* sweeps) {
  CsrGraph<int, float, int> g = view<float>(n, m, ro, ci, co, ri, NULL);
  Quiet q;
  auto t0 = std::chrono::steady_clock::now();
  CPUPR<int, float, int>(g, rank);
  double t = seconds_since(t0);
  std::string out = q.text();
  size_t at = out.find("CPU iterations:");
  *sweeps = at == std::string::npos ? -1 : atoi(out.c_str() + at + 15);
  return t;
}

// The reference's Matrix Market ingest: BuildMarketGraph<true> with undirected=false
// (b40c/graph/builder/market.cuh:173-205 -> csr_graph.cuh:74-164), as every driver
// calls it. Returns a handle; mgref_graph_get copies the arrays out.
void* mgref_load_market(const char* path, int* n, int* m) {
  CsrGraph<int, int, int>* g = new CsrGraph<int, int, int>(false);
  int rc;
  {
    Quiet q;
    rc = builder::BuildMarketGraph<true>(const_cast<char*>(path), *g, false);
  }
  if (rc != 0) {
    delete g;
    return NULL;
  }
  *n = g->nodes;
  *m = g->edges;
  return g;
}

void mgref_graph_get(void* h, int* ro, int* ci, int* vals, int* co, int* ri) {
  CsrGraph<int, int, int>* g = static_cast<CsrGraph<int, int, int>*>(h);
  memcpy(ro, g->row_offsets, sizeof(int) * (g->nodes + 1));
  memcpy(ci, g->column_indices, sizeof(int) * g->edges);
  memcpy(vals, g->edge_values, sizeof(int) * g->edges);
  memcpy(co, g->column_offsets, sizeof(int) * (g->nodes + 1));
  memcpy(ri, g->row_indices, sizeof(int) * g->edges);
}

void mgref_graph_free(void* h) {
  // CsrGraph::Free() would also free from_nodes/to_nodes, which the reference's
  // constructor leaves uninitialised, so the arrays FromCoo allocated are freed here.
  CsrGraph<int, int, int>* g = static_cast<CsrGraph<int, int, int>*>(h);
  free(g->row_offsets);
  free(g->column_indices);
  free(g->column_offsets);
  free(g->row_indices);
  free(g->edge_values);
  free(g->node_values);
  delete g;
}

}  // extern "C"
