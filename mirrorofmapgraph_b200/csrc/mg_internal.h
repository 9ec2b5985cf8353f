// mg_internal.h -- shared host-side definitions of the engine (not installed).
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "mapgraph_b200.h"

// Thread-local error detail behind mg_last_error().
void mg_set_error(const char *fmt, ...);

#ifdef __CUDACC__
#include <cuda_runtime.h>

#define MG_CUDA_TRY(expr)                                                                        \
  do {                                                                                           \
    cudaError_t _e = (expr);                                                                     \
    if (_e != cudaSuccess) {                                                                     \
      mg_set_error("%s:%d: %s failed: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e));  \
      return _e == cudaErrorMemoryAllocation ? MG_ERR_OOM : MG_ERR_CUDA;                         \
    }                                                                                            \
  } while (0)

#define MG_TRY(expr)                 \
  do {                               \
    mg_status _s = (expr);           \
    if (_s != MG_OK) return _s;      \
  } while (0)

// Device control block of one run: frontier sizes, level, direction and the
// counters the engine reports. Lives in device memory; a mapped/pinned mirror is
// read back once at the end of a run.
struct DevCtl {
  int32_t qlen[2];           // frontier sizes: [cur & 1] is the input of the current level
  int32_t level;             // current iteration
  int32_t dir;               // BFS: 0 push, 1 pull
  int32_t done;              // 1 when the loop must stop
  int32_t status;            // mg_status raised on the device (queue overflow, ...)
  int32_t iter_cap;          // stop after this many iterations
  uint32_t blocks_done;      // last-block-done counter of the current kernel
  int32_t cur;               // ping-pong selector of the frontier queues
  int32_t nf_next;           // vertices in the next frontier
  int64_t mf_next;           // out-edges of the next frontier (push/pull heuristic)
  int64_t visited_deg;       // sum of out-degrees of every vertex reached so far
  int64_t edges_inspected;   // edges read by the expansion kernels
  int64_t vertices_expanded; // frontier vertices processed
  int64_t vertices_updated;  // vertices whose value changed
  double dsum[4];            // FP64 reductions (PageRank residual, dangling mass, ...)
  double dprev[4];           // FP64 values of the previous iteration
  int32_t levels_pull;       // levels run bottom-up
  int32_t overflow;          // set by a kernel whose frontier append ran past capacity
  int32_t body_iters;        // WHILE-body executions so far (loop guard)
  int32_t big_len;           // vertices deferred to the grid-strided bin this level
  // SSSP near-far: vertices at distance >= thr wait in a far pile (ping-pong
  // far_cur) until the near frontier runs dry; then the pile is split at a new
  // threshold (split set between the relaxation and split kernels).
  int64_t thr;
  int32_t far_len[2];
  int32_t far_cur;
  int32_t split;
  int32_t far_min;
  int32_t splits;
  int64_t mf_front;          // out-edges of the current frontier (BFS)
  // persistent kernels: per-level counters in a ring of three (frontier out-edges,
  // frontier sizes), and the grid barrier (arrivals, generation)
  int64_t pm[3];
  int32_t pq[3];
  int32_t pb[3];  // deferred big vertices per level (persistent BFS)
  int32_t tile_next;  // next frontier tile of the dynamic schedule (SSSP rounds; reset at level end)
  int32_t trace_len;  // per-level trace records written by this run (mg_graph_trace)
  uint32_t bar_count;
  uint32_t bar_gen;
};

// Padding of the device graph arrays. Offsets arrays hold n + 1 + MG_OFF_PAD
// entries (the pad is INT_MAX) and edge arrays m + MG_EDGE_PAD entries (the pad is
// 0), so 16-byte-aligned bulk copies that round a range outwards stay inside the
// allocation, and an offset read one past the end compares as "no more edges".
constexpr int64_t MG_OFF_PAD = 7;
constexpr int64_t MG_EDGE_PAD = 8;

// Reusable device workspace of a graph, grown on demand.
struct Workspace {
  void *ptr = nullptr;
  size_t bytes = 0;
};

// Default traversal tuning (mg_tuning_defaults).
inline mg_tuning tuning_defaults() {
  mg_tuning t;
  std::memset(&t, 0, sizeof(t));
  t.sssp_heavy = 256;
  t.sssp_heavy_small = 32;
  t.sssp_ctas_per_sm = 4;
  t.sssp_batch_heavy = 32;
  t.bfs_cta_th = 512;
  t.bfs_grid_th = 4096;
  t.bfs_defer_warp = 1;
  t.bfs_persist_max = 1 << 16;
  t.bfs_persist_edges = 1 << 17;
  t.bfs_alpha = 14;
  t.bfs_beta = 24;
  t.bfs_sparse_degree = 8;
  t.bfs_ctas_per_sm = 4;
  t.bfs_tail_max = 512;
  t.bfs_tail_edges = 16384;
  t.cc_rounds = 1;
  return t;
}

struct mg_graph {
  int device = 0;
  int64_t n = 0, m = 0;
  uint32_t flags = 0;
  mg_dtype vtype = MG_DTYPE_NONE;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  // CSR
  int32_t *ro = nullptr, *ci = nullptr;
  void *vals = nullptr;
  // CSC (aliases the CSR when symmetric)
  int32_t *co = nullptr, *ri = nullptr, *perm = nullptr;
  void *cvals = nullptr;
  bool has_csc = false, csc_owned = false;
  // cached checks of the edge values
  bool pending_validation = false;  // MG_GRAPH_ASYNC_UPLOAD: checked before the first use
  bool weights_checked = false;
  int32_t min_weight = 0;
  double mean_weight = 0.0;
  // ragged batch
  std::vector<int64_t> vbase;
  // workspaces: ws_main per-run state, ws_aux graph build scratch, ws_out staged
  // results of host-output calls, ws_plan per-graph plans that outlive one call
  Workspace ws_main, ws_aux, ws_out;
  void *plan_csc = nullptr;  // PageRank gather plan over the CSC (pagerank.cu)
  void *plan_csr = nullptr;  // the same over the CSR (adjoint)
  DevCtl *ctl = nullptr;       // device control block
  DevCtl *ctl_host = nullptr;  // pinned host mirror
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  void *cache = nullptr;       // cached executable loop graphs (engine.cu)
  mg_tuning tune = tuning_defaults();  // traversal thresholds and launch shapes (mg_graph_set_tuning)
  int64_t host_iters = 0;              // body calls of the last host-driven loop (run_loop)
};

// Every device allocation of the library goes through here: cudaMallocAsync on
// stream s, unless the allocation-failure test hook (mg_debug_fail_alloc) says
// this one fails, in which case it returns cudaErrorMemoryAllocation without
// allocating.
cudaError_t mg_malloc_async(void **p, size_t bytes, cudaStream_t s);
// Barrier test hook (mg_debug_barrier_skew): extra arrivals the persistent
// kernels' grid barriers wait for (0 normally) and their poll budget then.
int32_t debug_barrier_extra();
unsigned long long debug_barrier_limit();

// Device memory of a graph's workspaces and plans, taken from the device's
// stream-ordered pool on the graph's stream: freed blocks stay in the pool, so a
// new graph of the same size reuses them without a driver allocation or a
// device-wide synchronisation.
mg_status dev_alloc(mg_graph *g, void **p, size_t bytes);
void dev_free(mg_graph *g, void *p);

// Per-level trace records live in the control block's allocation, behind the
// DevCtl and its 64 spare bytes, so kernels reach them from the DevCtl pointer.
constexpr size_t MG_TRACE_OFF = (sizeof(DevCtl) + 64 + 15) & ~(size_t)15;
__host__ __device__ inline mg_level_record *trace_of(DevCtl *c) {
  return reinterpret_cast<mg_level_record *>(reinterpret_cast<char *>(c) + MG_TRACE_OFF);
}
__device__ inline void trace_level(DevCtl *c, int32_t level, int32_t dir, int64_t frontier, int64_t edges,
                                   double value) {
  if (level < 0 || level >= MG_TRACE_LEVELS) return;
  mg_level_record r;
  r.level = level;
  r.direction = dir;
  r.frontier = frontier;
  r.frontier_edges = edges;
  r.value = value;
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  r.time_ns = t;
  trace_of(c)[level] = r;
  if (level + 1 > c->trace_len) c->trace_len = level + 1;
}

// Grows a workspace to at least `bytes` (contents are not preserved).
mg_status ws_reserve(mg_graph *g, Workspace &w, size_t bytes);

// Carves aligned sub-buffers out of a workspace.
struct Carve {
  char *base;
  size_t off = 0;
  explicit Carve(void *p) : base((char *)p) {}
  template <typename T>
  T *take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T *p = (T *)(base + off);
    off += count * sizeof(T);
    return p;
  }
  static size_t need(std::initializer_list<size_t> sizes) {
    size_t off = 0;
    for (size_t s : sizes) off = ((off + 255) & ~(size_t)255) + s;
    return off + 256;
  }
};

// Makes the graph's device current; returns MG_ERR_CUDA on failure.
mg_status graph_enter(mg_graph *g);

// Checks, before any launch, that a caller's pointer that kernels will read or
// write is device memory of the graph's device (or managed memory): a host
// pointer passed where device memory is required returns MG_ERR_ARG instead of
// faulting the GPU. A null pointer passes (callers check their own required
// arguments). `fn` and `what` name the entry point and the argument in the error.
mg_status check_device_ptr(const mg_graph *g, const void *p, const char *fn, const char *what);

// Copies a device int32 array into a host or device destination.
mg_status copy_out(mg_graph *g, void *dst, const void *src, size_t bytes, int device_output);
#endif  // __CUDACC__
