// Vertex programs written against MapGraph's Program contract (the structure of
// Algorithms/*/*.h: VertexType, EdgeType, Initialize, five selectors, device
// functors, extractResult) and run through the compat EnactorVertexCentric's
// generic kernels. Usage: gas_user_programs <minlabel|insum> <graph.mtx> [directed]
// prints one value per vertex.
#include <cstdio>
#include <cstring>
#include <vector>

#include "GASengine/csr_problem.cuh"
#include "GASengine/enactor_vertex_centric.cuh"
#include "mapgraph_b200_io.h"

// Smallest vertex id reachable through the expansion edges, by label propagation:
// every vertex starts in the frontier; an edge offers the sender's label to the
// receiver, which keeps the smaller one and re-enters the frontier when it shrank.
struct minlabel {
  typedef int DataType;
  typedef int MiscType;
  typedef int GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = INT_MAX;
  static const bool allow_duplicates = true;
  struct VertexType {
    int *d_label = nullptr;
    int nodes = 0;
  };
  struct EdgeType {
    int nodes = 0, edges = 0;
  };
  static void Initialize(const int, const int nodes, const int edges, int, int *, int *, int *, int *, int *, int *,
                         VertexType &vl, EdgeType &el, int *d_frontier_keys[3], MiscType *[3]) {
    vl.nodes = nodes;
    el.nodes = nodes;
    el.edges = edges;
    cudaMalloc((void **)&vl.d_label, sizeof(int) * (nodes + 1));
    util::SequenceKernel<int><<<(nodes + 255) / 256 + 1, 256>>>(vl.d_label, nodes);
    util::SequenceKernel<int><<<(nodes + 255) / 256 + 1, 256>>>(d_frontier_keys[0], nodes);
    util::SequenceKernel<int><<<(nodes + 255) / 256 + 1, 256>>>(d_frontier_keys[1], nodes);
    cudaDeviceSynchronize();
  }
  static SrcVertex srcVertex() { return ALL; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return NO_APPLY_VERTICES; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }
  static PostApplyVertices postApplyOverEdges() { return POST_APPLY_FRONTIER; }
  struct gather_sum {
    __device__ int operator()(int a, int b) { return a < b ? a : b; }
  };
  struct gather_vertex {
    __device__ void operator()(const int, const int, VertexType &, EdgeType &) {}
  };
  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, int &) {}
  };
  struct apply {
    __device__ void operator()(const int, const int, int, VertexType &, EdgeType &, char &changed) { changed = 1; }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, int *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int vertex_id, const int neighbor_id_in, const int,
                               VertexType &vl, EdgeType &, int &frontier, int &misc_value) {
      frontier = neighbor_id_in;
      misc_value = vl.d_label[vertex_id];
    }
  };
  struct contract {
    __device__ void operator()(const int, int &vertex_id, VertexType &vl, EdgeType &, int *, int &misc_value) {
      const int old = atomicMin(vl.d_label + vertex_id, misc_value);
      if (misc_value >= old) vertex_id = -1;
    }
  };
  static void extractResult(VertexType &vl, DataType *h_output) {
    cudaMemcpy(h_output, vl.d_label, sizeof(int) * vl.nodes, cudaMemcpyDeviceToHost);
  }
};

// One gather sweep: value[v] = INIT (0) + sum over in-edges (u, v) of (u + 1),
// through gather_edge / gather_sum / apply; nothing is expanded, so the run ends
// after one iteration.
struct insum {
  typedef long long DataType;
  typedef int MiscType;
  typedef long long GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const long long INIT_VALUE = 0;
  static const bool allow_duplicates = false;
  struct VertexType {
    long long *d_value = nullptr;
    int nodes = 0;
  };
  struct EdgeType {
    int nodes = 0;
  };
  static void Initialize(const int, const int nodes, const int, int, int *, int *, int *, int *, int *,
                         long long *, VertexType &vl, EdgeType &el, int *d_frontier_keys[3], MiscType *[3]) {
    vl.nodes = nodes;
    el.nodes = nodes;
    cudaMalloc((void **)&vl.d_value, sizeof(long long) * (nodes + 1));
    cudaMemset(vl.d_value, 0xff, sizeof(long long) * (nodes + 1));
    util::SequenceKernel<int><<<(nodes + 255) / 256 + 1, 256>>>(d_frontier_keys[1], nodes);
    cudaDeviceSynchronize();
  }
  static SrcVertex srcVertex() { return ALL; }
  static GatherEdges gatherOverEdges() { return GATHER_IN_EDGES; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static ExpandEdges expandOverEdges() { return NO_EXPAND_EDGES; }
  static PostApplyVertices postApplyOverEdges() { return NO_POST_APPLY_VERTICES; }
  struct gather_sum {
    __device__ long long operator()(long long a, long long b) { return a + b; }
  };
  struct gather_edge {
    __device__ void operator()(const int, const int, const int neighbor_id_in, VertexType &, EdgeType &,
                               long long &new_value) {
      new_value = neighbor_id_in + 1;
    }
  };
  struct apply {
    __device__ void operator()(const int vertex_id, const int, long long gathervalue, VertexType &vl, EdgeType &,
                               char &changed) {
      vl.d_value[vertex_id] = gathervalue;
      changed = 0;
    }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, long long *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return false; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int, const int, const int, VertexType &, EdgeType &,
                               int &frontier, int &) {
      frontier = -1;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &, VertexType &, EdgeType &, long long *, int &) {}
  };
  static void extractResult(VertexType &vl, DataType *h_output) {
    cudaMemcpy(h_output, vl.d_value, sizeof(long long) * vl.nodes, cudaMemcpyDeviceToHost);
  }
};

struct NoConfig {};

template <typename Program>
static int run(const mg_host_csr &g, int directed) {
  typedef GASengine::CsrProblem<Program, int, int, typename Program::DataType, false, false> Problem;
  Problem problem{NoConfig()};
  if (problem.FromHostProblem(false, (int)g.n, (int)g.m, g.col_idx, g.row_offsets, nullptr, nullptr, nullptr, 1,
                              directed))
    return 1;
  GASengine::EnactorVertexCentric<Problem, Program> enactor{NoConfig()};
  if (enactor.EnactIterativeSearch(problem, g.row_offsets, directed, (int)g.n, nullptr, INT_MAX, 1000)) return 1;
  std::vector<typename Program::DataType> out(g.n);
  problem.ExtractResults(out.data());
  for (int64_t i = 0; i < g.n; i++) std::printf("%lld\n", (long long)out[i]);
  std::fprintf(stderr, "iterations %lld\n", enactor.iteration[0]);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  mg_host_csr g;
  std::memset(&g, 0, sizeof(g));
  if (mg_read_market(argv[2], 0, &g) != MG_OK) return 1;
  const int directed = argc > 3 ? std::atoi(argv[3]) : 1;
  int rc = 2;
  if (!std::strcmp(argv[1], "minlabel")) rc = run<minlabel>(g, directed);
  else if (!std::strcmp(argv[1], "insum")) rc = run<insum>(g, directed);
  mg_host_csr_free(&g);
  return rc;
}
