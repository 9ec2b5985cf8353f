// cc.cu -- connected components (struct cc, Algorithms/CC/cc.h:32-349).
//
// The reference propagates minimum labels: every vertex starts with its own id
// (SequenceKernel, cc.h:118-120) and each iteration pushes a neighbour's smaller
// label through atomicMin, over CSR and CSC (the driver forces directed = 0,
// Algorithms/CC/cc.cu:289), until nothing changes. The fixed point labels every
// vertex with the smallest id in its weakly connected component.
//
// Here the same labels come from one pass of union-find over the edge list:
// hooking always links the larger root under the smaller one with atomicCAS, so
// parent pointers only decrease and every root is its component's minimum; a
// final pass compresses each vertex to its root. Each edge is read once (each
// undirected edge once for symmetric graphs), no iteration loop runs, and the
// result equals the reference's bit for bit.
#include <algorithm>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"

namespace mg {

constexpr int CC_NT = 256;
constexpr int CC_CTA_TH = 1024;

// Root of x with path halving. Parent entries are read from L2 (ld.cg): they are
// rewritten concurrently, and every value ever stored is an ancestor, so a
// racing read is still a valid step towards the root.
__device__ __forceinline__ int32_t uf_find(int32_t *p, int32_t x) {
  int32_t par = __ldcg(p + x);
  while (par != x) {
    const int32_t gp = __ldcg(p + par);
    if (gp != par) __stcg(p + x, gp);
    x = par;
    par = gp;
  }
  return x;
}

__device__ __forceinline__ void uf_union(int32_t *p, int32_t a, int32_t b) {
  int32_t ra = uf_find(p, a), rb = uf_find(p, b);
  while (ra != rb) {
    const int32_t hi = max(ra, rb), lo = min(ra, rb);
    const int32_t old = atomicCAS(p + hi, hi, lo);
    if (old == hi) return;
    // hi was hooked meanwhile; continue from its new root.
    ra = uf_find(p, old);
    rb = uf_find(p, lo);
  }
}

__global__ void cc_init_kernel(int32_t *p, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int32_t)i;
}

// One pass over all vertices in tiles of CC_NT; every edge (v, u) is united.
// With `half` set (symmetric input) only edges with u < v are used: the reverse
// copy of every edge is in the CSR too.
__global__ void __launch_bounds__(CC_NT) cc_hook_kernel(const int32_t *__restrict__ ro,
                                                        const int32_t *__restrict__ ci, int64_t n, int32_t *p,
                                                        int half, unsigned long long *insp_out) {
  __shared__ ExpandSmem<CC_NT> sm;
  __shared__ int64_t s_sum[CC_NT / 32 + 1];
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * CC_NT; tile < n; tile += (int64_t)gridDim.x * CC_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < n ? (int32_t)i : -1;
    expand_tile<CC_NT, CC_CTA_TH>(sm, ro, v, insp, [&](int32_t sv, int32_t k) {
      const int32_t u = ci[k];
      if (half && u >= sv) return;
      if (u == sv) return;
      uf_union(p, sv, u);
    });
  }
  const int64_t b = block_sum<CC_NT>(insp, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd(insp_out, (unsigned long long)b);
}

__global__ void cc_compress_kernel(int32_t *p, int32_t *label, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t r = (int32_t)i;
    int32_t par = __ldcg(p + r);
    while (par != r) {
      r = par;
      par = __ldcg(p + r);
    }
    label[i] = r;
  }
}

}  // namespace mg

extern "C" mg_status mg_cc(mg_graph *g, int32_t *label, const mg_opts *opts, mg_stats *stats) {
  using namespace mg;
  if (!g || !label) {
    mg_set_error("mg_cc: null argument");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  MG_TRY(graph_enter(g));
  const int64_t n = g->n;
  const size_t need = Carve::need({sizeof(int32_t) * (size_t)n, sizeof(int32_t) * (size_t)n});
  MG_TRY(ws_reserve(g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  int32_t *parent = cv.take<int32_t>(n);
  int32_t *lab_ws = cv.take<int32_t>(n);
  int32_t *out = o.device_output ? label : lab_ws;
  cudaStream_t s = g->stream;
  const bool half = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  unsigned long long *insp = reinterpret_cast<unsigned long long *>(&g->ctl->edges_inspected);
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  const int grid = g->num_sms * 8;
  cc_init_kernel<<<grid, 256, 0, s>>>(parent, n);
  cc_hook_kernel<<<g->num_sms * 4, CC_NT, 0, s>>>(g->ro, g->ci, n, parent, half ? 1 : 0, insp);
  cc_compress_kernel<<<grid, 256, 0, s>>>(parent, out, n);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  if (!o.device_output) MG_TRY(copy_out(g, label, out, sizeof(int32_t) * n, 0));
  MG_TRY(fetch_ctl(g));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = 1;
    stats->edges_traversed = g->m;
    stats->edges_inspected = g->ctl_host->edges_inspected;
    stats->bytes_compulsory = 4 * g->m + 4 * (n + 1) + 4 * n /* parent init */ + 8 * n /* compress */;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
  }
  return MG_OK;
}
