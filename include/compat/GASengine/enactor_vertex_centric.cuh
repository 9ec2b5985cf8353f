// GASengine/enactor_vertex_centric.cuh -- source-compatible replacement of
// MapGraph's EnactorVertexCentric (GASengine/enactor_vertex_centric.cuh:280,
// EnactIterativeSearch at :2398-2966 there), running any vertex program written
// against the reference's Program contract.
//
// MapGraph's four bundled programs (structs named bfs, sssp, cc and pagerank at
// global scope, Algorithms/*/*.h) are dispatched to the engine's tuned entry
// points (mg_bfs, mg_sssp, mg_cc, mg_pagerank in its reference-compatible mode),
// which write into the program's own result arrays. Every other program runs
// through the generic kernels below, which inline the program's device functors;
// define MG_GAS_GENERIC_ONLY to send the bundled programs there as well.
//
// One iteration of the generic loop, with the reference's hook order
// (vertex frontier F, edge frontier E):
//   gather      if gatherOverEdges() != NO_GATHER_EDGES: for v in F,
//               gather_tmp[v] = INIT_VALUE (+) gather_edge(...) over the gather edges
//               (in-edges, out-edges or both; both when directed == 0), (+) being
//               gather_sum; a warp per vertex above 8 edges, a lane per vertex below
//   apply       if applyOverEdges() == APPLY_FRONTIER: apply(v, iteration,
//               gather_tmp[v], ..., changed[v]) for v in F
//   post_apply  POST_APPLY_FRONTIER: for v in F (POST_APPLY_ALL: every vertex),
//               clear v's visited bit, then post_apply(v, ..., gather_tmp)
//   expand      for v in F, c = expand_vertex(v, changed[v], ...), then for every
//               expansion edge expand_edge(c, iteration, v, neighbour, edge_id, ...,
//               key, misc); keys other than -1 go to E (edge ids are CSR ids, also
//               for in-edges)
//   contract    for (key, misc) in E: contract(iteration, key, ..., gather_tmp, misc);
//               a key still not -1 whose visited bit this thread sets joins the next F
// until F is empty or iter_num iterations ran. The visited mask dedups exactly
// (atomic bit claims), which the reference approximates with a byte mask plus
// warp and history hashes; with the mask the frontier is free of duplicates in
// both the allow_duplicates cases of the reference.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <type_traits>

#include "GASengine/csr_problem.cuh"
#include "mapgraph_b200.h"

// MapGraph's bundled vertex programs (defined by their own headers, if at all).
struct bfs;
struct sssp;
struct cc;
struct pagerank;

namespace GASengine {

template <typename P>
struct TunedProgram {
  static const int kind = 0;
};
#ifndef MG_GAS_GENERIC_ONLY
template <>
struct TunedProgram<::bfs> {
  static const int kind = 1;
};
template <>
struct TunedProgram<::sssp> {
  static const int kind = 2;
};
template <>
struct TunedProgram<::cc> {
  static const int kind = 3;
};
template <>
struct TunedProgram<::pagerank> {
  static const int kind = 4;
};
#endif

namespace gas {

constexpr int NT = 256;
constexpr int LANE_SERIAL = 8;  // edges a lane handles alone; larger vertices get the warp
constexpr unsigned FULLMASK = 0xffffffffu;

struct Control {
  int next_len;  // entries appended to the output frontier
  int overflow;  // an append ran past the capacity
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Warp-aggregated append; every lane of the warp calls it.
template <typename M>
__device__ __forceinline__ void append(bool pred, int key, M misc, int *keys, M *vals, int cap, Control *ctl) {
  const unsigned pm = __ballot_sync(FULLMASK, pred);
  if (!pm) return;
  int base = 0;
  const int leader = __ffs(pm) - 1;
  if (lane_id() == leader) base = atomicAdd(&ctl->next_len, __popc(pm));
  base = __shfl_sync(FULLMASK, base, leader);
  if (pred) {
    const int pos = base + __popc(pm & ((1u << lane_id()) - 1u));
    if (pos < cap) {
      keys[pos] = key;
      if (vals) vals[pos] = misc;
    } else {
      ctl->overflow = 1;
    }
  }
}

// Edge lists of one vertex for a direction: the CSR (out) or the CSC (in; its
// edge ids are mapped back to CSR ids).
struct Adj {
  const int *off, *idx, *perm;
};

template <typename Program>
__global__ void __launch_bounds__(NT) gather_kernel(int fsize, const int *frontier, Adj in, Adj out, int use_in,
                                                   int use_out, typename Program::VertexType vl,
                                                   typename Program::EdgeType el,
                                                   typename Program::GatherType *gtmp) {
  typedef typename Program::GatherType G;
  static_assert(std::is_arithmetic<G>::value, "the generic gather reduces arithmetic GatherType values");
  typename Program::gather_edge gather_edge;
  typename Program::gather_sum gather_sum;
  const int lane = lane_id();
  // A vertex with at most LANE_SERIAL gather edges is folded by its own lane; a
  // larger one by the whole warp (per-lane partials, then a warp reduction into
  // the owning lane's value).
  for (int base = blockIdx.x * NT; base < fsize; base += gridDim.x * NT) {
    const int i = base + threadIdx.x;
    const bool valid = i < fsize;
    const int v = valid ? frontier[i] : 0;
    G own = (G)Program::INIT_VALUE;
    G warp_acc = (G)0;
    bool warp_have = false;
    auto flush = [&](int owner_lane) {
      G x = warp_acc;
      bool h = warp_have;
      for (int o = 16; o > 0; o >>= 1) {
        const G y = __shfl_xor_sync(FULLMASK, x, o);
        const bool hy = __shfl_xor_sync(FULLMASK, (int)h, o) != 0;
        if (h && hy) x = (lane & o) ? gather_sum(y, x) : gather_sum(x, y);
        else if (hy) {
          x = y;
          h = true;
        }
      }
      if (lane == owner_lane && h) own = gather_sum(own, x);
      warp_acc = (G)0;
      warp_have = false;
    };
    for (int dir = 0; dir < 2; dir++) {
      if (dir == 0 && !use_in) continue;
      if (dir == 1 && !use_out) continue;
      const Adj &a = dir == 0 ? in : out;
      const int b = valid ? a.off[v] : 0, e = valid ? a.off[v + 1] : 0;
      const bool small = e - b <= LANE_SERIAL;
      for (int t = 0; t < LANE_SERIAL; t++) {
        const int k = b + t;
        if (valid && small && k < e) {
          G nv;
          gather_edge(v, a.perm ? a.perm[k] : k, a.idx[k], vl, el, nv);
          own = gather_sum(own, nv);
        }
      }
      unsigned pend = __ballot_sync(FULLMASK, valid && !small);
      while (pend) {
        const int l = __ffs(pend) - 1;
        pend &= pend - 1;
        const int vb = __shfl_sync(FULLMASK, b, l), ve = __shfl_sync(FULLMASK, e, l);
        const int vv = __shfl_sync(FULLMASK, v, l);
        for (int k = vb + lane; k < ve; k += 32) {
          G nv;
          gather_edge(vv, a.perm ? a.perm[k] : k, a.idx[k], vl, el, nv);
          warp_acc = warp_have ? gather_sum(warp_acc, nv) : nv;
          warp_have = true;
        }
        flush(l);
      }
    }
    if (valid) gtmp[v] = own;
  }
}

template <typename Program>
__global__ void apply_kernel(int fsize, const int *frontier, long long iteration, typename Program::VertexType vl,
                             typename Program::EdgeType el, typename Program::GatherType *gtmp, char *changed) {
  typename Program::apply apply;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < fsize; i += gridDim.x * blockDim.x) {
    const int v = frontier[i];
    apply(v, (int)iteration, gtmp[v], vl, el, changed[v]);
  }
}

template <typename Program>
__global__ void post_apply_kernel(int count, const int *frontier, typename Program::VertexType vl,
                                  typename Program::EdgeType el, typename Program::GatherType *gtmp,
                                  unsigned *visited) {
  typename Program::post_apply post_apply;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int v = frontier ? frontier[i] : i;
    atomicAnd(visited + (v >> 5), ~(1u << (v & 31)));
    post_apply(v, vl, el, gtmp);
  }
}

template <typename Program>
__global__ void __launch_bounds__(NT) expand_kernel(int fsize, const int *frontier, Adj in, Adj out, int use_in,
                                                   int use_out, int iteration, typename Program::VertexType vl,
                                                   typename Program::EdgeType el, const char *changed, int *ekeys,
                                                   typename Program::MiscType *evals, int ecap, Control *ctl) {
  typedef typename Program::MiscType M;
  typename Program::expand_vertex expand_vertex;
  typename Program::expand_edge expand_edge;
  for (int base = blockIdx.x * NT; base < fsize; base += gridDim.x * NT) {
    const int i = base + threadIdx.x;
    const bool valid = i < fsize;
    const int v = valid ? frontier[i] : 0;
    bool c = false;
    if (valid) c = expand_vertex(v, changed[v], vl, el);
    for (int dir = 0; dir < 2; dir++) {
      if (dir == 0 && !use_out) continue;
      if (dir == 1 && !use_in) continue;
      const Adj &a = dir == 0 ? out : in;
      const int lane = lane_id();
      const int b = valid ? a.off[v] : 0, e = valid ? a.off[v + 1] : 0;
      const bool small = e - b <= LANE_SERIAL;
      for (int t = 0; t < LANE_SERIAL; t++) {
        const int k = b + t;
        int key = -1;
        M misc = M();
        if (valid && small && k < e) expand_edge(c, iteration, v, a.idx[k], a.perm ? a.perm[k] : k, vl, el, key, misc);
        append<M>(key != -1, key, misc, ekeys, evals, ecap, ctl);
      }
      unsigned pend = __ballot_sync(FULLMASK, valid && !small);
      while (pend) {
        const int l = __ffs(pend) - 1;
        pend &= pend - 1;
        const int vb = __shfl_sync(FULLMASK, b, l), ve = __shfl_sync(FULLMASK, e, l);
        const int vv = __shfl_sync(FULLMASK, v, l);
        const bool vc = __shfl_sync(FULLMASK, (int)c, l) != 0;
        for (int k0 = vb; k0 < ve; k0 += 32) {
          const int k = k0 + lane;
          int key = -1;
          M misc = M();
          if (k < ve) expand_edge(vc, iteration, vv, a.idx[k], a.perm ? a.perm[k] : k, vl, el, key, misc);
          append<M>(key != -1, key, misc, ekeys, evals, ecap, ctl);
        }
      }
    }
  }
}

template <typename Program>
__global__ void __launch_bounds__(NT) contract_kernel(int esize, int *ekeys, typename Program::MiscType *evals,
                                                     int iteration, typename Program::VertexType vl,
                                                     typename Program::EdgeType el,
                                                     typename Program::GatherType *gtmp, unsigned *visited,
                                                     int *vkeys, int vcap, Control *ctl) {
  typedef typename Program::MiscType M;
  typename Program::contract contract;
  for (int base = blockIdx.x * NT; base < esize; base += gridDim.x * NT) {
    const int i = base + threadIdx.x;
    int key = i < esize ? ekeys[i] : -1;
    M misc = i < esize ? evals[i] : M();
    if (key != -1) contract(iteration, key, vl, el, gtmp, misc);
    bool keep = false;
    if (key != -1) {
      const unsigned bit = 1u << (key & 31);
      keep = !(atomicOr(visited + (key >> 5), bit) & bit);
    }
    append<M>(keep, key, misc, vkeys, (M *)nullptr, vcap, ctl);
  }
}

}  // namespace gas

template <typename CsrProblem, typename Program, bool INSTRUMENT = false>
class EnactorVertexCentric {
 public:
  typedef typename CsrProblem::VertexId VertexId;
  typedef typename CsrProblem::SizeT SizeT;
  typedef typename Program::GatherType GatherType;
  typedef typename Program::MiscType MiscType;

  long long iteration[1] = {0};
  double elapsed_ms = 0.0;

  template <typename Cfg>
  explicit EnactorVertexCentric(const Cfg &cfg, bool DEBUG = false) : debug_(DEBUG) {
    queue_sizing_ = cfg_queue_sizing(cfg, 0);
  }
  EnactorVertexCentric() = default;

  cudaError_t EnactIterativeSearch(CsrProblem &csr_problem, SizeT * /*h_row_offsets*/, int directed, int num_srcs,
                                   int *srcs, int iter_num, int threshold) {
    typename CsrProblem::GraphSlice *s = csr_problem.graph_slices[0];
    if (!csr_problem.graph) return cudaErrorInvalidValue;
    cudaError_t e = csr_problem.Reset(EDGE_FRONTIERS, queue_sizing_, directed);
    if (e) return e;
    GatherType *gtmp = nullptr;
    if ((e = cudaMalloc((void **)&gtmp, sizeof(GatherType) * ((size_t)s->nodes + 1)))) return e;
    util::MemsetKernel<GatherType><<<B40C_MIN(32 * 1024, (s->nodes + 255) / 256 + 1), 256>>>(
        gtmp, (GatherType)Program::INIT_VALUE, s->nodes);
    Program::Initialize(directed, s->nodes, s->edges, num_srcs, srcs, s->d_row_offsets, s->d_column_indices,
                        s->d_column_offsets, s->d_row_indices, s->d_edge_values, s->vertex_list, s->edge_list,
                        s->frontier_queues.d_keys, s->frontier_queues.d_values);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaDeviceSynchronize();
    cudaEventRecord(t0);
    if (TunedProgram<Program>::kind != 0) e = tuned(csr_problem, directed, num_srcs, srcs, iter_num);
    else e = generic(csr_problem, directed, num_srcs, iter_num, threshold, gtmp);
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    elapsed_ms = ms;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(gtmp);
    if (debug_ || INSTRUMENT) {
      std::printf("Kernel time took: %f ms\n", elapsed_ms);
      std::printf("Total iteration: %lld\n", iteration[0]);
    }
    return e;
  }

 private:
  template <typename Cfg>
  static auto cfg_queue_sizing(const Cfg &cfg, int) -> decltype(cfg.template getParameter<double>("max_queue_sizing")) {
    return cfg.template getParameter<double>("max_queue_sizing");
  }
  template <typename Cfg>
  static double cfg_queue_sizing(const Cfg &, long) {
    return 1.5;
  }

  // MapGraph's bundled programs on the engine's tuned entry points, writing into
  // the arrays that the program's Initialize allocated.
  cudaError_t tuned(CsrProblem &p, int directed, int num_srcs, int *srcs, int iter_num) {
    typename CsrProblem::GraphSlice *s = p.graph_slices[0];
    mg_opts o{};
    o.directed = directed;
    o.iter_num = iter_num == INT_MAX ? 0 : iter_num;
    o.device_output = 1;
    mg_stats st{};
    mg_status r = MG_OK;
    if constexpr (TunedProgram<Program>::kind == 1) {
      r = mg_bfs(p.graph, srcs, num_srcs, s->vertex_list.d_labels, &o, &st);
    } else if constexpr (TunedProgram<Program>::kind == 2) {
      r = mg_sssp(p.graph, srcs, num_srcs, s->vertex_list.d_dists, &o, &st);
    } else if constexpr (TunedProgram<Program>::kind == 3) {
      r = mg_cc(p.graph, s->vertex_list.d_dists, &o, &st);
    } else if constexpr (TunedProgram<Program>::kind == 4) {
      mg_pr_opts po{};
      po.mode = MG_PR_REFCOMPAT;
      po.directed = directed;
      po.max_iter = o.iter_num;
      po.device_output = 1;
      r = mg_pagerank(p.graph, nullptr, 1, s->vertex_list.d_dists, &po, &st);
    }
    iteration[0] = st.iterations;
    if (r != MG_OK) {
      std::fprintf(stderr, "EnactIterativeSearch: %s\n", mg_last_error());
      return cudaErrorUnknown;
    }
    return cudaSuccess;
  }

  cudaError_t generic(CsrProblem &p, int directed, int num_srcs, int iter_num, int /*threshold*/,
                      GatherType *gtmp) {
    typename CsrProblem::GraphSlice *s = p.graph_slices[0];
    gas::Control *ctl = nullptr, host{};
    cudaError_t e = cudaMalloc((void **)&ctl, sizeof(gas::Control));
    if (e) return e;
    const gas::Adj out{s->d_row_offsets, s->d_column_indices, nullptr};
    const gas::Adj in{s->d_column_offsets, s->d_row_indices, s->d_edgeCSC_indices};
    const int g = Program::gatherOverEdges();
    const int x = Program::expandOverEdges();
    const bool gather = g != NO_GATHER_EDGES;
    const int g_in = gather && (g == GATHER_IN_EDGES || g == GATHER_ALL_EDGES || directed == 0);
    const int g_out = gather && (g == GATHER_OUT_EDGES || g == GATHER_ALL_EDGES || directed == 0);
    const bool expand = x != NO_EXPAND_EDGES;
    const int x_out = expand && (x == EXPAND_OUT_EDGES || x == EXPAND_ALL_EDGES || directed == 0);
    const int x_in = expand && (x == EXPAND_IN_EDGES || x == EXPAND_ALL_EDGES || directed == 0);
    // The program's Initialize seeds the vertex frontier into d_keys[0] and [1].
    int *vcur = s->frontier_queues.d_keys[1], *vnext = s->frontier_queues.d_keys[0];
    int *ekeys = s->frontier_queues.d_keys[2];
    MiscType *evals = s->frontier_queues.d_values[2];
    const int vcap = s->frontier_elements[0], ecap = s->frontier_elements[2];
    unsigned *visited = reinterpret_cast<unsigned *>(s->d_visited_mask);
    int fsize = num_srcs;
    const int grid = 148 * 8;
    iteration[0] = 0;
    for (int i = 0; i < iter_num && fsize > 0; i++) {
      const int it = (int)iteration[0];
      if (gather)
        gas::gather_kernel<Program><<<grid, gas::NT>>>(fsize, vcur, in, out, g_in, g_out, s->vertex_list,
                                                       s->edge_list, gtmp);
      if (Program::applyOverEdges() == APPLY_FRONTIER)
        gas::apply_kernel<Program><<<grid, gas::NT>>>(fsize, vcur, iteration[0], s->vertex_list, s->edge_list,
                                                      gtmp, s->d_changed);
      if (Program::postApplyOverEdges() == POST_APPLY_FRONTIER)
        gas::post_apply_kernel<Program><<<grid, gas::NT>>>(fsize, vcur, s->vertex_list, s->edge_list, gtmp,
                                                           visited);
      else if (Program::postApplyOverEdges() == POST_APPLY_ALL)
        gas::post_apply_kernel<Program><<<grid, gas::NT>>>(s->nodes, nullptr, s->vertex_list, s->edge_list, gtmp,
                                                           visited);
      if ((e = cudaMemsetAsync(ctl, 0, sizeof(gas::Control)))) break;
      gas::expand_kernel<Program><<<grid, gas::NT>>>(fsize, vcur, in, out, x_in, x_out, it, s->vertex_list,
                                                     s->edge_list, s->d_changed, ekeys, evals, ecap, ctl);
      if ((e = cudaMemcpy(&host, ctl, sizeof(host), cudaMemcpyDeviceToHost))) break;
      if (host.overflow) {
        std::fprintf(stderr, "Frontier queue overflow.  Please increase queue-sizing factor.\n");
        e = cudaErrorLaunchOutOfResources;
        break;
      }
      const int esize = host.next_len;
      if ((e = cudaMemsetAsync(ctl, 0, sizeof(gas::Control)))) break;
      gas::contract_kernel<Program><<<grid, gas::NT>>>(esize, ekeys, evals, it, s->vertex_list, s->edge_list, gtmp,
                                                       visited, vnext, vcap, ctl);
      if ((e = cudaMemcpy(&host, ctl, sizeof(host), cudaMemcpyDeviceToHost))) break;
      if (host.overflow) {
        e = cudaErrorLaunchOutOfResources;
        break;
      }
      if ((e = cudaGetLastError())) break;
      fsize = host.next_len;
      int *t = vcur;
      vcur = vnext;
      vnext = t;
      iteration[0]++;
    }
    cudaFree(ctl);
    return e;
  }

  bool debug_ = false;
  double queue_sizing_ = 1.5;
};

}  // namespace GASengine
