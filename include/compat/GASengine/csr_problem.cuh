// GASengine/csr_problem.cuh -- source-compatible replacement of MapGraph's
// GASengine/csr_problem.cuh (CsrProblem, GraphSlice, the vertex-program selector
// enums and the b40c utilities that the bundled vertex programs call), backed by
// the mapgraph_b200 engine.
//
// Put include/compat ahead of the MapGraph tree on the include path and a vertex
// program written for MapGraph (a struct with VertexType / EdgeType, Initialize,
// the five selectors, the gather/apply/post_apply/expand/contract functors and
// extractResult) compiles against this header and
// GASengine/enactor_vertex_centric.cuh unchanged. The graph lives in an mg_graph
// (mg_graph_create, one upload and a device CSC build); GraphSlice exposes its
// device arrays under the reference's names (csr_problem.cuh:149-163 there).
// Errors are returned as cudaError_t, as in the reference; the engine's detail is
// in mg_last_error().
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <type_traits>

#include "mapgraph_b200.h"

namespace b40c {
namespace util {

// Prints a failed CUDA call with its location and returns the error
// (b40c/util/error_utils.cuh semantics: cudaSuccess passes through silently).
inline cudaError_t B40CPerror(cudaError_t error, const char *message, const char *filename, int line,
                              bool print = true) {
  if (error && print) {
    std::fprintf(stderr, "[%s, %d] %s (CUDA error %d: %s)\n", filename, line, message, (int)error,
                 cudaGetErrorString(error));
    std::fflush(stderr);
  }
  return error;
}

inline cudaError_t B40CPerror(cudaError_t error, bool print = true) {
  if (error && print) {
    std::fprintf(stderr, "(CUDA error %d: %s)\n", (int)error, cudaGetErrorString(error));
    std::fflush(stderr);
  }
  return error;
}

// d_out[i] = value for i < length (grid-strided).
template <typename T>
__global__ void MemsetKernel(T *d_out, T value, int length) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < length; i += gridDim.x * blockDim.x) d_out[i] = value;
}

// d_out[i] = i for i < length (grid-strided).
template <typename T>
__global__ void SequenceKernel(T *d_out, int length) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < length; i += gridDim.x * blockDim.x) d_out[i] = (T)i;
}

}  // namespace util
}  // namespace b40c

#ifndef B40C_MIN
#define B40C_MIN(a, b) (((a) < (b)) ? (a) : (b))
#endif
#ifndef B40C_MAX
#define B40C_MAX(a, b) (((a) > (b)) ? (a) : (b))
#endif

using namespace b40c;

// Vertex-program selectors (the reference's enumerators, at global scope as there).
enum SrcVertex { SINGLE, ALL };
enum GatherEdges { NO_GATHER_EDGES, GATHER_IN_EDGES, GATHER_OUT_EDGES, GATHER_ALL_EDGES };
enum ExpandEdges { NO_EXPAND_EDGES, EXPAND_IN_EDGES, EXPAND_OUT_EDGES, EXPAND_ALL_EDGES };
enum ApplyVertices { NO_APPLY_VERTICES, APPLY_ALL, APPLY_FRONTIER };
enum PostApplyVertices { NO_POST_APPLY_VERTICES, POST_APPLY_ALL, POST_APPLY_FRONTIER };

namespace GASengine {

enum FrontierType { VERTEX_FRONTIERS, EDGE_FRONTIERS, MIXED_FRONTIERS, MULTI_GPU_FRONTIERS };

template <typename _Program, typename _VertexId, typename _SizeT, typename _Value, bool MARK_PREDECESSORS,
          bool WITH_VALUE>
struct CsrProblem {
  typedef _Program Program;
  typedef _VertexId VertexId;
  typedef _SizeT SizeT;
  typedef typename Program::VertexType VertexType;
  typedef typename Program::EdgeType EdgeType;
  typedef typename Program::MiscType MiscType;
  typedef typename Program::DataType EValue;
  typedef unsigned char VisitedMask;

  // The device view of the graph and the run's queues (GraphSlice in the
  // reference). Graph arrays belong to the engine's graph handle.
  struct GraphSlice {
    VertexId *d_column_indices = nullptr;
    SizeT *d_row_offsets = nullptr;
    VertexId *d_row_indices = nullptr;
    SizeT *d_column_offsets = nullptr;
    VertexId *d_edgeCSC_indices = nullptr;  // CSC slot -> CSR edge id
    EValue *d_edge_values = nullptr;
    char *d_changed = nullptr;              // set by apply, read by expand_vertex
    VisitedMask *d_visited_mask = nullptr;  // one bit per vertex (n / 8 bytes, 4-byte aligned)
    VertexType vertex_list;
    EdgeType edge_list;
    struct {
      VertexId *d_keys[3] = {nullptr, nullptr, nullptr};
      MiscType *d_values[3] = {nullptr, nullptr, nullptr};
    } frontier_queues;
    SizeT frontier_elements[3] = {0, 0, 0};
    VertexId nodes = 0;
    SizeT edges = 0;
    cudaStream_t stream = nullptr;
  };

  GraphSlice *graph_slices[1] = {nullptr};
  mg_graph *graph = nullptr;
  int num_gpus = 1;
  VertexId nodes = 0;
  SizeT edges = 0;

  CsrProblem() { graph_slices[0] = new GraphSlice(); }
  template <typename Cfg>
  explicit CsrProblem(const Cfg &) : CsrProblem() {}
  ~CsrProblem() {
    FreeQueues();
    if (graph) mg_graph_destroy(graph);
    delete graph_slices[0];
  }
  CsrProblem(const CsrProblem &) = delete;
  CsrProblem &operator=(const CsrProblem &) = delete;

  // Uploads the host CSR (csr_problem.cuh:401-411 there). The caller's CSC
  // arrays are not needed: the engine builds the transpose on the device.
  cudaError_t FromHostProblem(bool /*stream_from_host*/, SizeT n, SizeT m, VertexId *h_column_indices,
                              SizeT *h_row_offsets, EValue *h_edge_values, VertexId * /*h_row_indices*/,
                              SizeT * /*h_column_offsets*/, int gpus, int /*directed*/) {
    static_assert(sizeof(VertexId) == 4 && sizeof(SizeT) == 4, "the engine stores int32 ids and offsets");
    FreeQueues();
    if (graph) {
      mg_graph_destroy(graph);
      graph = nullptr;
    }
    num_gpus = gpus;
    nodes = n;
    edges = m;
    const void *vals = nullptr;
    mg_dtype vt = MG_DTYPE_NONE;
    if (WITH_VALUE && h_edge_values && sizeof(EValue) == 4) {
      vals = h_edge_values;
      vt = std::is_floating_point<EValue>::value ? MG_DTYPE_F32 : MG_DTYPE_I32;
    }
    if (mg_graph_create(reinterpret_cast<const int32_t *>(h_row_offsets),
                        reinterpret_cast<const int32_t *>(h_column_indices), vals, vt, n, m, 0,
                        &graph) != MG_OK) {
      std::fprintf(stderr, "CsrProblem::FromHostProblem: %s\n", mg_last_error());
      return cudaErrorUnknown;
    }
    GraphSlice &s = *graph_slices[0];
    const int32_t *ro, *ci, *co, *ri, *perm;
    const void *ev;
    mg_graph_device_arrays(graph, &ro, &ci, &ev, &co, &ri, &perm);
    void *st = nullptr;
    mg_graph_stream(graph, &st);
    s.d_row_offsets = (SizeT *)ro;
    s.d_column_indices = (VertexId *)ci;
    s.d_column_offsets = (SizeT *)co;
    s.d_row_indices = (VertexId *)ri;
    s.d_edgeCSC_indices = (VertexId *)perm;
    s.d_edge_values = (EValue *)ev;
    s.nodes = n;
    s.edges = m;
    s.stream = (cudaStream_t)st;
    return cudaSuccess;
  }

  // Allocates the frontier queues (two vertex frontiers of n, one edge frontier
  // of max(queue_sizing, 1) * m + n), the changed flags and the visited mask
  // (csr_problem.cuh:627-827 there).
  cudaError_t Reset(FrontierType, double queue_sizing, int directed = 1) {
    GraphSlice &s = *graph_slices[0];
    FreeQueues();
    const double qs = std::max(queue_sizing, directed == 0 ? 2.0 : 1.0);
    const SizeT ecap = (SizeT)std::min<double>(qs * (double)s.edges + (double)s.nodes + 1.0, 2147483000.0);
    const SizeT vcap = s.nodes + 1;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 3 && e == cudaSuccess; i++) {
      const SizeT cap = i < 2 ? vcap : ecap;
      e = cudaMalloc((void **)&s.frontier_queues.d_keys[i], sizeof(VertexId) * (size_t)cap);
      if (e == cudaSuccess) e = cudaMalloc((void **)&s.frontier_queues.d_values[i], sizeof(MiscType) * (size_t)cap);
      s.frontier_elements[i] = cap;
    }
    if (e == cudaSuccess) e = cudaMalloc((void **)&s.d_changed, (size_t)s.nodes + 1);
    const size_t mask_bytes = (((size_t)s.nodes + 31) / 32) * 4;
    if (e == cudaSuccess) e = cudaMalloc((void **)&s.d_visited_mask, mask_bytes);
    if (e == cudaSuccess) e = cudaMemset(s.d_changed, 0, (size_t)s.nodes + 1);
    if (e == cudaSuccess) e = cudaMemset(s.d_visited_mask, 0, mask_bytes);
    return util::B40CPerror(e, "CsrProblem::Reset failed", __FILE__, __LINE__);
  }

  // The last run's per-vertex results (csr_problem.cuh:371 there).
  cudaError_t ExtractResults(EValue *h_values) {
    Program::extractResult(graph_slices[0]->vertex_list, h_values);
    return cudaGetLastError();
  }

 private:
  void FreeQueues() {
    GraphSlice *s = graph_slices[0];
    if (!s) return;
    for (int i = 0; i < 3; i++) {
      if (s->frontier_queues.d_keys[i]) cudaFree(s->frontier_queues.d_keys[i]);
      if (s->frontier_queues.d_values[i]) cudaFree(s->frontier_queues.d_values[i]);
      s->frontier_queues.d_keys[i] = nullptr;
      s->frontier_queues.d_values[i] = nullptr;
    }
    if (s->d_changed) cudaFree(s->d_changed);
    if (s->d_visited_mask) cudaFree(s->d_visited_mask);
    s->d_changed = nullptr;
    s->d_visited_mask = nullptr;
  }
};

}  // namespace GASengine
