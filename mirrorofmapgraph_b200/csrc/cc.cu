// cc.cu -- connected components (struct cc, Algorithms/CC/cc.h:32-349).
//
// The reference propagates minimum labels: every vertex starts with its own id
// (SequenceKernel, cc.h:118-120) and each iteration pushes a neighbour's smaller
// label through atomicMin, over CSR and CSC (the driver forces directed = 0,
// Algorithms/CC/cc.cu:289), until nothing changes. The fixed point labels every
// vertex with the smallest id in its weakly connected component.
//
// Here the same labels come from union-find, where hooking always links the
// larger root under the smaller one with atomicCAS: parent pointers only
// decrease, so every root is its component's minimum and the final labels equal
// the reference's bit for bit. The edge work follows the sampling scheme of
// Afforest (Sutton et al., IPDPS 2018):
//   1. mg_tuning.cc_rounds rounds (1 by default) link every vertex to its first
//      neighbours, then compress;
//   2. one CTA samples 1024 vertices and takes the most frequent root c (on
//      power-law graphs, the giant component);
//   3. only vertices outside c process their remaining edges (and, without a
//      symmetric adjacency, their in-edges too); then compress.
// Any edge with both endpoints skipped joins two members of c's tree already, so
// the result does not depend on the sample.
#include <algorithm>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"

namespace mg {

constexpr int CC_NT = 256;
constexpr int CC_CTA_TH = 1024;
constexpr int CC_SAMPLES = 1024;

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

// Sampling rounds r0 .. r1 - 1: v is united with its r-th neighbour in each
// (the union-find result does not depend on the order of the unions).
__global__ void cc_sample_link_kernel(const int32_t *__restrict__ ro, const int32_t *__restrict__ ci, int64_t n,
                                      int32_t *p, int r0, int r1) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = ro[v], e = ro[v + 1];
    for (int r = r0; r < r1 && b + r < e; r++) {
      const int32_t u = ci[b + r];
      if (u != v) uf_union(p, (int32_t)v, u);
    }
  }
}

__global__ void cc_compress_kernel(int32_t *p, int32_t *label, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t r = (int32_t)i;
    int32_t par = __ldcg(p + r);
    while (par != r) {
      r = par;
      par = __ldcg(p + r);
    }
    if (label) label[i] = r;
    else __stcg(p + i, r);
  }
}

// Most frequent root among CC_SAMPLES hashed vertices (one CTA of CC_SAMPLES
// threads); writes it to *out.
__global__ void __launch_bounds__(CC_SAMPLES) cc_mode_kernel(const int32_t *p, int64_t n, int32_t *out) {
  __shared__ int32_t s[CC_SAMPLES];
  __shared__ unsigned long long best;
  const int t = threadIdx.x;
  uint64_t h = (uint64_t)t * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  h ^= h >> 31;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 29;
  s[t] = __ldcg(p + (int64_t)(h % (uint64_t)n));
  if (t == 0) best = 0ull;
  __syncthreads();
  for (int size = 2; size <= CC_SAMPLES; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const int j = t ^ stride;
      if (j > t) {
        const bool up = (t & size) == 0;
        const int32_t a = s[t], b = s[j];
        if ((a > b) == up) {
          s[t] = b;
          s[j] = a;
        }
      }
      __syncthreads();
    }
  }
  if (t == 0 || s[t] != s[t - 1]) {
    int len = 1;
    while (t + len < CC_SAMPLES && s[t + len] == s[t]) len++;
    // larger count first, then the smaller root
    const unsigned long long key = ((unsigned long long)len << 32) | (unsigned)(INT_MAX - s[t]);
    atomicMax(&best, key);
  }
  __syncthreads();
  if (t == 0) *out = INT_MAX - (int32_t)(best & 0xffffffffu);
}

// Phase 3: every vertex whose root is not c unites all its remaining edges
// (from index `skip` of its CSR row; all in-edges too when `both`).
__global__ void __launch_bounds__(CC_NT) cc_finish_kernel(const int32_t *__restrict__ ro,
                                                          const int32_t *__restrict__ ci,
                                                          const int32_t *__restrict__ co,
                                                          const int32_t *__restrict__ ri, int64_t n, int32_t *p,
                                                          const int32_t *cptr, int skip, int both,
                                                          unsigned long long *insp_out) {
  __shared__ ExpandSmem<CC_NT> sm;
  __shared__ int64_t s_sum[CC_NT / 32 + 1];
  const int32_t c = *cptr;
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * CC_NT; tile < n; tile += (int64_t)gridDim.x * CC_NT) {
    const int64_t i = tile + threadIdx.x;
    int32_t v = i < n ? (int32_t)i : -1;
    if (v >= 0 && __ldcg(p + v) == c) v = -1;
    expand_tile<CC_NT, CC_CTA_TH>(sm, ro, v, insp, [&](int32_t sv, int32_t k) {
      if (k - __ldg(ro + sv) < skip) return;
      const int32_t u = ci[k];
      if (u != sv) uf_union(p, sv, u);
    });
    if (both)
      expand_tile<CC_NT, CC_CTA_TH>(sm, co, v, insp, [&](int32_t sv, int32_t k) {
        const int32_t u = ri[k];
        if (u != sv) uf_union(p, sv, u);
      });
  }
  const int64_t b = block_sum<CC_NT>(insp, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd(insp_out, (unsigned long long)b);
}

// Without a usable transpose: every edge once.
__global__ void __launch_bounds__(CC_NT) cc_all_edges_kernel(const int32_t *__restrict__ ro,
                                                             const int32_t *__restrict__ ci, int64_t n, int32_t *p,
                                                             unsigned long long *insp_out) {
  __shared__ ExpandSmem<CC_NT> sm;
  __shared__ int64_t s_sum[CC_NT / 32 + 1];
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * CC_NT; tile < n; tile += (int64_t)gridDim.x * CC_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < n ? (int32_t)i : -1;
    expand_tile<CC_NT, CC_CTA_TH>(sm, ro, v, insp, [&](int32_t sv, int32_t k) {
      const int32_t u = ci[k];
      if (u != sv) uf_union(p, sv, u);
    });
  }
  const int64_t b = block_sum<CC_NT>(insp, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd(insp_out, (unsigned long long)b);
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
  if (o.device_output) MG_TRY(check_device_ptr(g, label, "mg_cc", "label"));
  const int64_t n = g->n;
  const size_t need = Carve::need({sizeof(int32_t) * (size_t)n, sizeof(int32_t) * (size_t)n, 64});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  int32_t *parent = cv.take<int32_t>(n);
  int32_t *lab_ws = cv.take<int32_t>(n);
  int32_t *cmode = cv.take<int32_t>(16);
  int32_t *out = o.device_output ? label : lab_ws;
  cudaStream_t s = g->stream;
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool sampling = symmetric || g->has_csc;
  unsigned long long *insp = reinterpret_cast<unsigned long long *>(&g->ctl->edges_inspected);
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  const int grid = g->num_sms * 8;
  int64_t launches = 0;
  cc_init_kernel<<<grid, 256, 0, s>>>(parent, n);
  launches++;
  // Neighbour-sampling rounds before the giant component is picked: R-MAT s22
  // 0.33 / 0.41 / 0.48 ms with 1 / 2 / 3 rounds. With none, only the sampled
  // root's own self-loops are skipped, so every count gives the same labels.
  const int32_t rounds = g->tune.cc_rounds;
  if (n > 0 && sampling) {
    // one launch per round: every vertex's first link lands before any second
    // (two rounds in one pass measured 0.51 against 0.41 ms on R-MAT s22)
    for (int r = 0; r < rounds; r++) cc_sample_link_kernel<<<grid, 256, 0, s>>>(g->ro, g->ci, n, parent, r, r + 1);
    cc_compress_kernel<<<grid, 256, 0, s>>>(parent, nullptr, n);
    cc_mode_kernel<<<1, CC_SAMPLES, 0, s>>>(parent, n, cmode);
    cc_finish_kernel<<<g->num_sms * 4, CC_NT, 0, s>>>(g->ro, g->ci, g->co, g->ri, n, parent, cmode, rounds,
                                                      symmetric ? 0 : 1, insp);
    launches += rounds + 3;
  } else if (n > 0) {
    cc_all_edges_kernel<<<g->num_sms * 4, CC_NT, 0, s>>>(g->ro, g->ci, n, parent, insp);
    launches++;
  }
  cc_compress_kernel<<<grid, 256, 0, s>>>(parent, out, n);
  launches++;
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  if (!o.device_output) MG_TRY(copy_out(g, label, out, sizeof(int32_t) * n, 0));
  MG_TRY(fetch_ctl(g));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = 1;
    stats->edges_traversed = g->m;
    stats->edges_inspected = g->ctl_host->edges_inspected + (sampling ? (int64_t)rounds * n : 0);
    // offsets and sampled neighbours, the remaining edges actually read, parent
    // init / compress passes
    stats->bytes_compulsory = 4 * (n + 1) + 4 * stats->edges_inspected + 16 * n;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->launches = launches;
  }
  return MG_OK;
}
