// part.cu -- one rank's share of a BFS over a 1-D vertex partition.
//
// A graph too large for one GPU is split into contiguous vertex ranges, one per
// rank (the layout the reference's unused multi-GPU scaffolding describes,
// GASengine/csr_problem.cuh:339-365). Rank r keeps the out-edges (CSR rows) and
// the in-edges (CSC rows) of its vertices [lo, hi) with global vertex ids, plus
// three replicated arrays of n entries: the visited bitmap, the frontier bitmap
// and the depths. A level is
//   step   push: the owned frontier vertices' out-edges mark unvisited targets in
//          a rank-local bitmap of n bits (any owner); pull: every owned unvisited
//          vertex with an in-neighbour in the frontier marks itself;
//   gather the caller all-gathers the ranks' bitmaps (one collective per level;
//          NCCL over NVLink between GPUs, a shared buffer between partitions on
//          one GPU);
//   merge  OR of the world's bitmaps minus the visited set = the next frontier;
//          every rank folds the same words, so the replicated state stays equal
//          on every rank without another exchange, and the push/pull choice
//          (Beamer's rule, as in bfs.cu) comes out the same everywhere.
// Depths follow the reference's BFS (Algorithms/BFS/bfs.h:28-262): a vertex's
// depth is the first level whose frontier reaches it, whatever the direction.
#include <algorithm>
#include <cstddef>
#include <cstring>

#include "common.cuh"
#include "expand.cuh"
#include "mg_internal.h"
#define MG_PRB_NO_PLAN_KERNELS
#include "pr_binned.cuh"

namespace mg {

constexpr int PART_NT = 256;
constexpr int PART_CTA_TH = 256;
constexpr int PART_PULL_SERIAL = 8;
constexpr int64_t PART_ALPHA = 14, PART_BETA = 24;

// Per-level counters (zeroed before every merge) and run totals.
struct PartCtl {
  unsigned long long nf;    // vertices of the new frontier
  unsigned long long mf;    // their out-edges (global out-degree)
  int32_t qlen;             // owned vertices of the new frontier (push queue)
  int32_t big_len;          // deferred big vertices of a push step
  unsigned long long insp;  // edges read by this rank's steps (run total)
  double resid;             // PageRank: L1 change of the last merge
  double dang;              // PageRank: dangling mass of the current iterate
  unsigned blocks_done;     // PageRank step: CTAs finished (the last resets the schedule)
};

__global__ void part_clear_kernel(uint32_t *vis, uint32_t *fr, int32_t *depth, int64_t nwords, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    depth[i] = -1;
    if (i < nwords) {
      vis[i] = 0u;
      fr[i] = 0u;
    }
  }
}

__global__ void part_seed_kernel(const int32_t *srcs, int32_t nsrc, uint32_t *vis, uint32_t *fr, int32_t *depth,
                                 const int32_t *deg, int64_t lo, int64_t hi, int32_t *q, PartCtl *ctl) {
  __shared__ int64_t s_sum[1024 / 32 + 1];
  int64_t nf = 0, mf = 0;
  for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
    const int32_t s = srcs[i];
    const uint32_t bit = 1u << (s & 31);
    if (!(atomicOr(&vis[s >> 5], bit) & bit)) {
      atomicOr(&fr[s >> 5], bit);
      depth[s] = 0;
      nf += 1;
      mf += deg[s];
      if (s >= lo && s < hi) q[atomicAdd(&ctl->qlen, 1)] = s;
    }
  }
  const int64_t tf = block_sum<1024>(nf, s_sum);
  const int64_t tm = block_sum<1024>(mf, s_sum);
  if (threadIdx.x == 0) {
    ctl->nf = (unsigned long long)tf;
    ctl->mf = (unsigned long long)tm;
  }
}

struct PartPush {
  const uint32_t *vis;
  uint32_t *bits;
};

__device__ __forceinline__ void part_mark(const PartPush &x, int32_t u) {
  const uint32_t bit = 1u << (u & 31);
  const int32_t w = u >> 5;
  if ((x.vis[w] & bit) || (x.bits[w] & bit)) return;
  atomicOr(&x.bits[w], bit);
}

// Push: the owned frontier queue (global ids) expanded over the local CSR rows
// (row v - lo); vertices of GRID_TH or more edges go to part_push_big_kernel.
__global__ void __launch_bounds__(PART_NT) part_push_kernel(const int32_t *ro, const int32_t *ci, int64_t lo,
                                                            const int32_t *q, int32_t qlen, const uint32_t *vis,
                                                            uint32_t *bits, int32_t *big_v, PartCtl *ctl) {
  __shared__ ExpandSmem<PART_NT> sm;
  __shared__ int64_t s_sum[PART_NT / 32 + 1];
  const PartPush x{vis, bits};
  const BigList big{big_v, &ctl->big_len, defer_threshold<PART_NT>(qlen, PART_CTA_TH)};
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * PART_NT; tile < qlen; tile += (int64_t)gridDim.x * PART_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < qlen ? (int32_t)(q[i] - lo) : -1;
    expand_tile<PART_NT, PART_CTA_TH>(sm, ro, v, insp, [&](int32_t, int32_t k) { part_mark(x, ci[k]); }, &big);
  }
  const int64_t bins = block_sum<PART_NT>(insp, s_sum);
  if (threadIdx.x == 0 && bins) atomicAdd(&ctl->insp, (unsigned long long)bins);
}

__global__ void __launch_bounds__(PART_NT) part_push_big_kernel(const int32_t *ro, const int32_t *ci,
                                                                const uint32_t *vis, uint32_t *bits, int32_t *big_v,
                                                                PartCtl *ctl) {
  __shared__ BigSmem<PART_NT> sm;
  const PartPush x{vis, bits};
  expand_big<PART_NT>(sm, ro, BigList{big_v, &ctl->big_len}, [&](int32_t, int32_t k) { part_mark(x, ci[k]); });
}

// Pull: a warp per 32 owned vertices (lo is a multiple of 32, so a warp owns one
// whole word of the output bitmap). Each lane scans its vertex's first in-edges;
// longer rows are then scanned by the whole warp, one row at a time, until a
// frontier in-neighbour turns up.
__global__ void __launch_bounds__(PART_NT) part_pull_kernel(const int32_t *co, const int32_t *ri, int64_t lo,
                                                            int64_t hi, const uint32_t *vis, const uint32_t *fr,
                                                            uint32_t *bits, PartCtl *ctl) {
  __shared__ int64_t s_sum[PART_NT / 32 + 1];
  const int lane = lane_id();
  const int64_t w0 = lo >> 5, w1 = (hi + 31) >> 5;
  const int64_t wstride = ((int64_t)gridDim.x * PART_NT) >> 5;
  int64_t insp = 0;
  for (int64_t w = w0 + (((int64_t)blockIdx.x * PART_NT + threadIdx.x) >> 5); w < w1; w += wstride) {
    const uint32_t vw = vis[w];
    if (vw == FULL) continue;
    const int64_t v = (w << 5) + lane;
    const bool need = v < hi && !((vw >> lane) & 1u);
    bool found = false;
    int32_t beg = 0, end = 0;
    if (need) {
      beg = co[v - lo];
      end = co[v - lo + 1];
    }
    const int32_t lim = min(end, beg + PART_PULL_SERIAL);
    for (int32_t e = beg; e < lim; e++) {
      insp++;
      const int32_t u = ri[e];
      if ((fr[u >> 5] >> (u & 31)) & 1u) {
        found = true;
        break;
      }
    }
    unsigned pend = __ballot_sync(FULL, need && !found && lim < end);
    while (pend) {
      const int l = __ffs(pend) - 1;
      pend &= pend - 1;
      const int32_t b = __shfl_sync(FULL, lim, l), en = __shfl_sync(FULL, end, l);
      bool f = false;
      for (int32_t e0 = b; e0 < en; e0 += 32) {
        const int32_t e = e0 + lane;
        bool hit = false;
        if (e < en) {
          const int32_t u = ri[e];
          hit = (fr[u >> 5] >> (u & 31)) & 1u;
          insp++;
        }
        if (__any_sync(FULL, hit)) {
          f = true;
          break;
        }
      }
      if (lane == l) found = f;
    }
    const unsigned fm = __ballot_sync(FULL, found);
    if (lane == 0 && fm) bits[w] = fm;
  }
  const int64_t bins = block_sum<PART_NT>(insp, s_sum);
  if (threadIdx.x == 0 && bins) atomicAdd(&ctl->insp, (unsigned long long)bins);
}

// Merge: next = (OR over ranks) & ~visited, word by word over all n bits; depths
// and the visited/frontier bitmaps are updated for every vertex, the owned new
// frontier vertices are queued for the next push step.
__global__ void __launch_bounds__(PART_NT) part_merge_kernel(const uint32_t *gathered, int32_t world, int64_t nwords,
                                                             uint32_t *vis, uint32_t *fr, int32_t *depth,
                                                             const int32_t *deg, int32_t level, int64_t lo,
                                                             int64_t hi, int32_t *q, PartCtl *ctl) {
  __shared__ int64_t s_sum[PART_NT / 32 + 1];
  const int lane = lane_id();
  int64_t nf = 0, mf = 0;
  const int64_t stride = (int64_t)gridDim.x * PART_NT;
  // Whole warps walk the words so that the owned-vertex append stays warp-uniform.
  const int64_t wend = (nwords + 31) & ~(int64_t)31;
  for (int64_t w = (int64_t)blockIdx.x * PART_NT + threadIdx.x; w < wend; w += stride) {
    uint32_t x = 0u;
    if (w < nwords) {
      for (int32_t r = 0; r < world; r++) x |= gathered[(int64_t)r * nwords + w];
      const uint32_t old = vis[w];
      x &= ~old;
      fr[w] = x;
      if (x) {
        vis[w] = old | x;
        nf += __popc(x);
        for (uint32_t y = x; y; y &= y - 1) {
          const int64_t v = (w << 5) + (__ffs(y) - 1);
          depth[v] = level + 1;
          mf += deg[v];
        }
      }
    }
    // Owned vertices of the new frontier (words [lo/32, ceil(hi/32)) are owned
    // whole): one queue reservation per warp.
    const uint32_t own = ((w << 5) >= lo && (w << 5) < hi) ? x : 0u;
    const int32_t cnt = __popc(own);
    const int32_t incl = warp_inclusive_scan(cnt);
    const int32_t wtot = __shfl_sync(FULL, incl, 31);
    if (wtot) {
      int32_t base = 0;
      if (lane == 31) base = atomicAdd(&ctl->qlen, wtot);
      base = __shfl_sync(FULL, base, 31) + incl - cnt;
      for (uint32_t y = own; y; y &= y - 1) q[base++] = (int32_t)((w << 5) + (__ffs(y) - 1));
    }
  }
  const int64_t bnf = block_sum<PART_NT>(nf, s_sum);
  const int64_t bmf = block_sum<PART_NT>(mf, s_sum);
  if (threadIdx.x == 0) {
    if (bnf) atomicAdd(&ctl->nf, (unsigned long long)bnf);
    if (bmf) atomicAdd(&ctl->mf, (unsigned long long)bmf);
  }
}

// Offsets 0..m non-decreasing over `rows` rows (bit 0), ids in [0, nv) (bit 1).
__global__ void part_validate_kernel(const int32_t *ro, const int32_t *ci, int64_t rows, int64_t m, int64_t nv,
                                     int32_t *bad) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int32_t b = 0;
  for (int64_t i = tid; i <= rows; i += stride) {
    const int32_t r = ro[i];
    if (i == 0 && r != 0) b |= 1;
    if (i == rows && r != (int32_t)m) b |= 1;
    if (i < rows && ro[i + 1] < r) b |= 1;
  }
  for (int64_t i = tid; i < m; i += stride)
    if ((uint32_t)ci[i] >= (uint64_t)nv) b |= 2;
  if (b) atomicOr(bad, b);
}

__global__ void part_sum_kernel(const int32_t *v, int64_t n, unsigned long long *sum) {
  __shared__ int64_t s_sum[256 / 32 + 1];
  int64_t t = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) t += v[i];
  const int64_t b = block_sum<256>(t, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd(sum, (unsigned long long)b);
}

// PageRank over the partition (normalised, uniform teleport t = 1/n; the rule of
// mg_pagerank's MG_PR_NORMALIZED): x' = alpha (P^T x + d t) + (1 - alpha) t.
// Every rank keeps x and y = x / outdeg for all n vertices; a step computes x' of
// its own rows from y with the degree-binned gather over its in-edges, the
// ranks all-gather the slices, and the merge (identical on every rank) forms y,
// the L1 change and the dangling mass d with fixed-order FP64 sums, so every
// rank takes the same stop decision.
struct PartPrRow {
  float *slice;
  double alpha, tn, d;
  __device__ __forceinline__ void operator()(int32_t r, Comp v) const {
    const double acc = (double)v.hi + (double)v.lo;
    slice[r] = (float)(alpha * (acc + d * tn) + (1.0 - alpha) * tn);
  }
};

__global__ void __launch_bounds__(PRB_NT, PRB_MIN_BLOCKS) part_pr_kernel(PrbArgs p, const float *y, float *slice,
                                                                         double alpha, double tn, PartCtl *ctl) {
  const PartPrRow up{slice, alpha, tn, __ldcg(&ctl->dang)};
  prb_run<false>(p, [&](int32_t col) { return __ldg(y + col); }, up,
                 [&](int64_t, int32_t row, Comp v) { up(row, v); });
  if (last_block(&ctl->blocks_done) && threadIdx.x == 0) {
    *p.grab = 0;
    ctl->blocks_done = 0;
  }
}

__global__ void __launch_bounds__(256) part_pr_init_kernel(int64_t n, double tn, const int32_t *deg, float *x,
                                                           float *y, double *part) {
  __shared__ double s_red[256 / 32 + 1];
  double d = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    x[v] = (float)tn;
    const int32_t k = deg[v];
    if (k > 0) {
      y[v] = (float)(tn / k);
    } else {
      y[v] = 0.f;
      d += (double)(float)tn;
    }
  }
  d = block_sum<256>(d, s_red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = 0.0;
    part[2 * blockIdx.x + 1] = d;
  }
}

__global__ void __launch_bounds__(256) part_pr_merge_kernel(int64_t n, const float *xo, const float *xn,
                                                            const int32_t *deg, float *y, double *part) {
  __shared__ double s_red[256 / 32 + 1];
  double r = 0.0, d = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const float x = xn[v];
    r += fabs((double)x - (double)xo[v]);
    const int32_t k = deg[v];
    if (k > 0) {
      y[v] = (float)((double)x / k);
    } else {
      y[v] = 0.f;
      d += (double)x;
    }
  }
  r = block_sum<256>(r, s_red);
  d = block_sum<256>(d, s_red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r;
    part[2 * blockIdx.x + 1] = d;
  }
}

// Fixed-order sum of the per-CTA partials (the same on every rank).
__global__ void __launch_bounds__(256) part_pr_reduce_kernel(const double *part, int32_t grid, PartCtl *ctl) {
  __shared__ double s_red[256 / 32 + 1];
  double r = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < grid; i += 256) {
    r += part[2 * i];
    d += part[2 * i + 1];
  }
  r = block_sum<256>(r, s_red);
  d = block_sum<256>(d, s_red);
  if (threadIdx.x == 0) {
    ctl->resid = r;
    ctl->dang = d;
  }
}

__global__ void part_outdeg_kernel(const int32_t *ro, int64_t rows, int32_t *deg) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) deg[i] = ro[i + 1] - ro[i];
}

}  // namespace mg

struct mg_part {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t n = 0, lo = 0, hi = 0, nwords = 0, m_out = 0, m_in = 0, m_total = 0;
  int32_t *ro = nullptr, *ci = nullptr, *co = nullptr, *ri = nullptr, *deg = nullptr;
  bool in_aliases_out = false;
  // run state
  uint32_t *vis = nullptr, *fr = nullptr;
  int32_t *depth = nullptr, *q = nullptr, *big_v = nullptr, *srcs = nullptr;
  int32_t src_cap = 0;
  mg::PartCtl *ctl = nullptr, *ctl_host = nullptr;
  // PageRank state
  mg::BinPlan prb;
  bool prb_ok = false;
  float *xo = nullptr, *xn = nullptr, *y = nullptr;
  double *ppart = nullptr;
  int32_t pgrid = 0;
  bool pr_begun = false, pr_stepped = false, pr_done = true;
  int32_t pr_level = 0, pr_max_iter = 50;
  double alpha = 0.85, tol = 1e-6, tn = 0.0, resid = 0.0;
  bool begun = false, done = true, stepped = false;
  int32_t level = 0, dir = 0, mode = MG_DIR_AUTO, iter_cap = 0, qlen = 0;
  int64_t nf = 0, mf = 0, vdeg = 0, levels_pull = 0, steps = 0;
  double ms = 0.0;
};

namespace {

mg_status part_alloc(mg_part *p, void **ptr, size_t bytes) {
  cudaError_t e = mg_malloc_async(ptr, std::max<size_t>(bytes, 4), p->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    mg_set_error("mg_part: device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MG_ERR_OOM : MG_ERR_CUDA;
  }
  return MG_OK;
}

void part_free(mg_part *p) {
  if (!p) return;
  cudaSetDevice(p->device);
  auto fr = [&](void *q) {
    if (q && p->stream) cudaFreeAsync(q, p->stream);
  };
  fr(p->ro);
  fr(p->ci);
  if (!p->in_aliases_out) {
    fr(p->co);
    fr(p->ri);
  }
  fr(p->deg);
  fr(p->vis);
  fr(p->fr);
  fr(p->depth);
  fr(p->q);
  fr(p->big_v);
  fr(p->srcs);
  fr(p->ctl);
  fr(p->xo);
  fr(p->xn);
  fr(p->y);
  fr(p->ppart);
  if (p->prb_ok && p->stream) bin_plan_release(p->stream, p->prb);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->ctl_host) cudaFreeHost(p->ctl_host);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  if (p->stream) cudaStreamDestroy(p->stream);
  cudaGetLastError();
  delete p;
}

mg_status upload(mg_part *p, int32_t **dst, const int32_t *src, int64_t count, int64_t pad, cudaMemcpyKind kind) {
  MG_TRY(part_alloc(p, (void **)dst, sizeof(int32_t) * (size_t)(count + pad)));
  if (count > 0) MG_CUDA_TRY(cudaMemcpyAsync(*dst, src, sizeof(int32_t) * (size_t)count, kind, p->stream));
  if (pad > 0) MG_CUDA_TRY(cudaMemsetAsync(*dst + count, 0, sizeof(int32_t) * (size_t)pad, p->stream));
  return MG_OK;
}

}  // namespace

extern "C" mg_status mg_part_create(int64_t n, int64_t lo, int64_t hi, const int32_t *out_offsets,
                                    const int32_t *out_idx, const int32_t *in_offsets, const int32_t *in_idx,
                                    const int32_t *out_degree, uint32_t flags, mg_part **out) {
  if (!out || !out_offsets || (!in_offsets && !(flags & MG_GRAPH_SYMMETRIC))) {
    mg_set_error("mg_part_create: null argument");
    return MG_ERR_ARG;
  }
  *out = nullptr;
  if (n <= 0 || n > INT32_MAX - 64 || lo < 0 || hi < lo || hi > n || (lo & 31) != 0 || ((hi & 31) != 0 && hi != n)) {
    mg_set_error("mg_part_create: need 0 <= lo <= hi <= n < 2^31, lo a multiple of 32, hi a multiple of 32 or n");
    return MG_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    mg_set_error("mg_part_create: no CUDA device");
    return MG_ERR_NO_DEVICE;
  }
  const bool dev_in = (flags & MG_GRAPH_DEVICE_INPUT) != 0;
  const cudaMemcpyKind kind = dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const int64_t rows = hi - lo;
  // Edge counts come from the offsets' last entries (host reads; device input is
  // read back once).
  int32_t ends[2] = {0, 0};
  auto last = [&](const int32_t *off, int32_t *v) -> mg_status {
    if (dev_in) {
      MG_CUDA_TRY(cudaMemcpy(v, off + rows, sizeof(int32_t), cudaMemcpyDeviceToHost));
    } else {
      *v = off[rows];
    }
    return MG_OK;
  };
  int32_t first[2] = {0, 0};
  auto head = [&](const int32_t *off, int32_t *v) -> mg_status {
    if (dev_in) {
      MG_CUDA_TRY(cudaMemcpy(v, off, sizeof(int32_t), cudaMemcpyDeviceToHost));
    } else {
      *v = off[0];
    }
    return MG_OK;
  };
  MG_TRY(last(out_offsets, &ends[0]));
  MG_TRY(head(out_offsets, &first[0]));
  const bool sym = (flags & MG_GRAPH_SYMMETRIC) != 0;
  if (!sym) {
    MG_TRY(last(in_offsets, &ends[1]));
    MG_TRY(head(in_offsets, &first[1]));
  }
  if (first[0] != 0 || ends[0] < 0 || (!sym && (first[1] != 0 || ends[1] < 0)) || (ends[0] > 0 && !out_idx) ||
      (!sym && ends[1] > 0 && !in_idx)) {
    mg_set_error("mg_part_create: offsets must start at 0 and end at the edge count (with its index array)");
    return MG_ERR_ARG;
  }
  mg_part *p = new mg_part();
  p->n = n;
  p->lo = lo;
  p->hi = hi;
  p->nwords = (n + 31) / 32;
  p->m_out = ends[0];
  p->m_in = sym ? ends[0] : ends[1];
  p->in_aliases_out = sym;
  auto fail = [&](mg_status st) {
    part_free(p);
    return st;
  };
  if (cudaGetDevice(&p->device) != cudaSuccess) return fail(MG_ERR_CUDA);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  p->num_sms = sms > 0 ? sms : 148;
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&p->ev0) != cudaSuccess || cudaEventCreate(&p->ev1) != cudaSuccess) {
    cudaGetLastError();
    mg_set_error("mg_part_create: stream or event creation failed");
    return fail(MG_ERR_CUDA);
  }
  mg_status st;
  if ((st = upload(p, &p->ro, out_offsets, rows + 1, 8, kind)) != MG_OK) return fail(st);
  if ((st = upload(p, &p->ci, out_idx, p->m_out, 8, kind)) != MG_OK) return fail(st);
  if (sym) {
    p->co = p->ro;
    p->ri = p->ci;
  } else {
    if ((st = upload(p, &p->co, in_offsets, rows + 1, 8, kind)) != MG_OK) return fail(st);
    if ((st = upload(p, &p->ri, in_idx, p->m_in, 8, kind)) != MG_OK) return fail(st);
  }
  if (out_degree) {
    if ((st = upload(p, &p->deg, out_degree, n, 8, kind)) != MG_OK) return fail(st);
  } else if (rows == n) {
    // One partition holds everything: the degrees are its own rows'.
    if ((st = part_alloc(p, (void **)&p->deg, sizeof(int32_t) * (size_t)(n + 8))) != MG_OK) return fail(st);
    mg::part_outdeg_kernel<<<p->num_sms * 4, 256, 0, p->stream>>>(p->ro, n, p->deg);
  } else {
    mg_set_error("mg_part_create: out_degree (n entries) is needed when the partition does not hold every vertex");
    return fail(MG_ERR_ARG);
  }
  // Every id must be a vertex and the offsets a valid CSR (checked on the device).
  {
    int32_t *bad = nullptr;
    if ((st = part_alloc(p, (void **)&bad, sizeof(int32_t) * 2)) != MG_OK) return fail(st);
    cudaMemsetAsync(bad, 0, sizeof(int32_t) * 2, p->stream);
    mg::part_validate_kernel<<<p->num_sms * 8, 256, 0, p->stream>>>(p->ro, p->ci, rows, p->m_out, n, bad);
    if (!sym) mg::part_validate_kernel<<<p->num_sms * 8, 256, 0, p->stream>>>(p->co, p->ri, rows, p->m_in, n, bad);
    int32_t hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, p->stream);
    cudaFreeAsync(bad, p->stream);
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) {
      mg_set_error("mg_part_create: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(MG_ERR_CUDA);
    }
    if (hbad) {
      mg_set_error("mg_part_create: %s", (hbad & 1) ? "offsets are not a valid CSR (0..m, non-decreasing)"
                                                    : "vertex id out of range [0, n)");
      return fail(MG_ERR_ARG);
    }
  }
  // Total edges of the graph, for the direction rule.
  {
    unsigned long long *sum = nullptr;
    if ((st = part_alloc(p, (void **)&sum, sizeof(unsigned long long))) != MG_OK) return fail(st);
    cudaMemsetAsync(sum, 0, sizeof(unsigned long long), p->stream);
    mg::part_sum_kernel<<<p->num_sms * 4, 256, 0, p->stream>>>(p->deg, n, sum);
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, p->stream);
    cudaFreeAsync(sum, p->stream);
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) {
      mg_set_error("mg_part_create: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(MG_ERR_CUDA);
    }
    p->m_total = (int64_t)h;
  }
  if ((st = part_alloc(p, (void **)&p->vis, sizeof(uint32_t) * (size_t)p->nwords)) != MG_OK) return fail(st);
  if ((st = part_alloc(p, (void **)&p->fr, sizeof(uint32_t) * (size_t)p->nwords)) != MG_OK) return fail(st);
  if ((st = part_alloc(p, (void **)&p->depth, sizeof(int32_t) * (size_t)n)) != MG_OK) return fail(st);
  if ((st = part_alloc(p, (void **)&p->q, sizeof(int32_t) * (size_t)std::max<int64_t>(rows, 1))) != MG_OK)
    return fail(st);
  if ((st = part_alloc(p, (void **)&p->big_v, sizeof(int32_t) * mg::BIG_CAP)) != MG_OK) return fail(st);
  if ((st = part_alloc(p, (void **)&p->ctl, sizeof(mg::PartCtl))) != MG_OK) return fail(st);
  if (cudaMallocHost((void **)&p->ctl_host, sizeof(mg::PartCtl)) != cudaSuccess) {
    cudaGetLastError();
    mg_set_error("mg_part_create: pinned host allocation failed");
    return fail(MG_ERR_OOM);
  }
  if (cudaStreamSynchronize(p->stream) != cudaSuccess) {
    mg_set_error("mg_part_create: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(MG_ERR_CUDA);
  }
  *out = p;
  return MG_OK;
}

extern "C" mg_status mg_part_destroy(mg_part *p) {
  part_free(p);
  return MG_OK;
}

extern "C" mg_status mg_part_stream(const mg_part *p, void **stream) {
  if (!p || !stream) {
    mg_set_error("mg_part_stream: null argument");
    return MG_ERR_ARG;
  }
  *stream = (void *)p->stream;
  return MG_OK;
}

extern "C" mg_status mg_part_words(const mg_part *p, int64_t *words) {
  if (!p || !words) {
    mg_set_error("mg_part_words: null argument");
    return MG_ERR_ARG;
  }
  *words = p->nwords;
  return MG_OK;
}

static void fill_level(const mg_part *p, mg_part_level *lv) {
  if (!lv) return;
  std::memset(lv, 0, sizeof(*lv));
  lv->frontier = p->nf;
  lv->frontier_edges = p->mf;
  lv->level = p->level;
  lv->done = p->done ? 1 : 0;
  lv->direction = p->dir == 1 ? MG_DIR_PULL : MG_DIR_PUSH;
}

extern "C" mg_status mg_part_bfs_begin(mg_part *p, const int32_t *srcs, int32_t nsrc, const mg_opts *opts,
                                       mg_part_level *level) {
  using namespace mg;
  if (!p || !srcs || nsrc <= 0) {
    mg_set_error("mg_part_bfs_begin: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (o.direction < MG_DIR_AUTO || o.direction > MG_DIR_PULL) {
    mg_set_error("mg_part_bfs_begin: invalid direction %d", o.direction);
    return MG_ERR_ARG;
  }
  for (int32_t i = 0; i < nsrc; i++) {
    if (srcs[i] < 0 || srcs[i] >= p->n) {
      mg_set_error("mg_part_bfs_begin: source %d out of range [0, %lld)", srcs[i], (long long)p->n);
      return MG_ERR_ARG;
    }
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  if (nsrc > p->src_cap) {
    if (p->srcs) cudaFreeAsync(p->srcs, p->stream);
    p->srcs = nullptr;
    p->src_cap = 0;
    MG_TRY(part_alloc(p, (void **)&p->srcs, sizeof(int32_t) * (size_t)nsrc));
    p->src_cap = nsrc;
  }
  cudaStream_t s = p->stream;
  MG_CUDA_TRY(cudaMemcpyAsync(p->srcs, srcs, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaEventRecord(p->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(p->ctl, 0, sizeof(PartCtl), s));
  part_clear_kernel<<<p->num_sms * 8, 256, 0, s>>>(p->vis, p->fr, p->depth, p->nwords, p->n);
  part_seed_kernel<<<1, 1024, 0, s>>>(p->srcs, nsrc, p->vis, p->fr, p->depth, p->deg, p->lo, p->hi, p->q, p->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(PartCtl), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  // AUTO on sparse graphs stays top-down, as in mg_bfs (mean out-degree <= 8)
  p->mode = (o.direction == MG_DIR_AUTO && p->m_total <= 8 * p->n) ? MG_DIR_PUSH : o.direction;
  p->iter_cap = o.iter_num > 0 ? (int32_t)std::min<int64_t>(o.iter_num, p->n + 1) : (int32_t)(p->n + 1);
  p->level = 0;
  p->dir = 0;
  p->nf = (int64_t)p->ctl_host->nf;
  p->mf = (int64_t)p->ctl_host->mf;
  p->vdeg = p->mf;
  p->qlen = p->ctl_host->qlen;
  p->levels_pull = 0;
  p->steps = 0;
  p->done = p->nf == 0 || p->iter_cap <= 0;
  p->begun = true;
  p->stepped = false;
  fill_level(p, level);
  return MG_OK;
}

extern "C" mg_status mg_part_bfs_step(mg_part *p, uint32_t *bits) {
  using namespace mg;
  if (!p || !bits) {
    mg_set_error("mg_part_bfs_step: null argument");
    return MG_ERR_ARG;
  }
  if (!p->begun || p->done || p->stepped) {
    mg_set_error("mg_part_bfs_step: no level pending (call mg_part_bfs_begin, then step and merge in turn)");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  MG_CUDA_TRY(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * (size_t)p->nwords, s));
  if (p->dir == 0) {
    if (p->qlen > 0) {
      const int grid = p->num_sms * 4;
      MG_CUDA_TRY(cudaMemsetAsync(&p->ctl->big_len, 0, sizeof(int32_t), s));
      part_push_kernel<<<grid, PART_NT, 0, s>>>(p->ro, p->ci, p->lo, p->q, p->qlen, p->vis, bits, p->big_v, p->ctl);
      part_push_big_kernel<<<p->num_sms * 4, PART_NT, 0, s>>>(p->ro, p->ci, p->vis, bits, p->big_v, p->ctl);
    }
  } else if (p->hi > p->lo) {
    const int64_t warps = ((p->hi + 31) >> 5) - (p->lo >> 5);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, (int64_t)p->num_sms * 8));
    part_pull_kernel<<<grid, PART_NT, 0, s>>>(p->co, p->ri, p->lo, p->hi, p->vis, p->fr, bits, p->ctl);
  }
  MG_CUDA_TRY(cudaGetLastError());
  p->stepped = true;
  p->steps++;
  return MG_OK;
}

extern "C" mg_status mg_part_bfs_merge(mg_part *p, const uint32_t *gathered, int32_t world, mg_part_level *level) {
  using namespace mg;
  if (!p || !gathered || world <= 0) {
    mg_set_error("mg_part_bfs_merge: null argument or world <= 0");
    return MG_ERR_ARG;
  }
  if (!p->stepped) {
    mg_set_error("mg_part_bfs_merge: no step to merge");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  MG_CUDA_TRY(cudaMemsetAsync(p->ctl, 0, offsetof(PartCtl, big_len), s));
  const int64_t warps = (p->nwords + 31) / 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, (int64_t)p->num_sms * 8));
  part_merge_kernel<<<grid, PART_NT, 0, s>>>(gathered, world, p->nwords, p->vis, p->fr, p->depth, p->deg, p->level,
                                             p->lo, p->hi, p->q, p->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(PartCtl), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  const PartCtl &h = *p->ctl_host;
  p->stepped = false;
  p->level += 1;
  p->nf = (int64_t)h.nf;
  p->mf = (int64_t)h.mf;
  p->vdeg += p->mf;
  p->qlen = h.qlen;
  p->done = p->nf == 0 || p->level >= p->iter_cap;
  if (!p->done) {
    // Beamer's rule on replicated counts: every rank takes the same direction.
    if (p->mode == MG_DIR_PULL) p->dir = 1;
    else if (p->mode == MG_DIR_PUSH) p->dir = 0;
    else if (p->dir == 0) p->dir = p->mf > (p->m_total - p->vdeg) / PART_ALPHA ? 1 : 0;
    else p->dir = p->nf * PART_BETA < p->n ? 0 : 1;
    if (p->dir == 1) p->levels_pull++;
  }
  fill_level(p, level);
  return MG_OK;
}

extern "C" mg_status mg_part_bfs_result(mg_part *p, int32_t *depth, int32_t device_output, mg_stats *stats) {
  using namespace mg;
  if (!p || !depth) {
    mg_set_error("mg_part_bfs_result: null argument");
    return MG_ERR_ARG;
  }
  if (!p->begun) {
    mg_set_error("mg_part_bfs_result: no run (call mg_part_bfs_begin first)");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  MG_CUDA_TRY(cudaEventRecord(p->ev1, s));
  MG_CUDA_TRY(cudaMemcpyAsync(depth, p->depth, sizeof(int32_t) * (size_t)p->n,
                              device_output ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(PartCtl), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = p->level;
    stats->edges_traversed = p->vdeg;
    stats->edges_inspected = (int64_t)p->ctl_host->insp;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p->ev0, p->ev1);
    stats->kernel_ms = ms;
    stats->status_detail = (int32_t)p->levels_pull;
    stats->launches = 2 + 3 * p->steps;
  }
  return MG_OK;
}

// ---------------------------------------------------------------------------
// PageRank over the partition.

static void fill_pr_level(const mg_part *p, mg_part_level *lv) {
  if (!lv) return;
  std::memset(lv, 0, sizeof(*lv));
  lv->level = p->pr_level;
  lv->done = p->pr_done ? 1 : 0;
  lv->residual = p->resid;
}

extern "C" mg_status mg_part_pr_begin(mg_part *p, const mg_pr_opts *opts, mg_part_level *level) {
  using namespace mg;
  if (!p) {
    mg_set_error("mg_part_pr_begin: null argument");
    return MG_ERR_ARG;
  }
  mg_pr_opts o;
  std::memset(&o, 0, sizeof(o));
  o.mode = MG_PR_NORMALIZED;
  if (opts) o = *opts;
  if (o.mode != MG_PR_NORMALIZED || o.weighted) {
    mg_set_error("mg_part_pr_begin: the partitioned PageRank runs MG_PR_NORMALIZED, unweighted");
    return MG_ERR_UNSUPPORTED;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  const int64_t rows = p->hi - p->lo;
  if (!p->prb_ok) {
    MG_TRY(bin_plan_build(s, p->co, rows, p->prb));
    p->prb_ok = true;
  }
  p->pgrid = p->num_sms * 4;
  const size_t vb = sizeof(float) * (size_t)(p->n + 8);
  if (!p->xo) MG_TRY(part_alloc(p, (void **)&p->xo, vb));
  if (!p->xn) MG_TRY(part_alloc(p, (void **)&p->xn, vb));
  if (!p->y) MG_TRY(part_alloc(p, (void **)&p->y, vb));
  if (!p->ppart) MG_TRY(part_alloc(p, (void **)&p->ppart, sizeof(double) * 2 * (size_t)p->pgrid));
  p->alpha = o.alpha > 0 ? o.alpha : 0.85;
  p->tol = o.tol > 0 ? o.tol : 1e-6;
  p->pr_max_iter = o.max_iter > 0 ? o.max_iter : 50;
  p->tn = 1.0 / (double)p->n;
  MG_CUDA_TRY(cudaEventRecord(p->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(p->ctl, 0, sizeof(PartCtl), s));
  part_pr_init_kernel<<<p->pgrid, 256, 0, s>>>(p->n, p->tn, p->deg, p->xo, p->y, p->ppart);
  part_pr_reduce_kernel<<<1, 256, 0, s>>>(p->ppart, p->pgrid, p->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  p->pr_level = 0;
  p->resid = 0.0;
  p->pr_done = false;
  p->pr_begun = true;
  p->pr_stepped = false;
  fill_pr_level(p, level);
  return MG_OK;
}

extern "C" mg_status mg_part_pr_step(mg_part *p, float *slice) {
  using namespace mg;
  if (!p || !slice) {
    mg_set_error("mg_part_pr_step: null argument");
    return MG_ERR_ARG;
  }
  if (!p->pr_begun || p->pr_done || p->pr_stepped) {
    mg_set_error("mg_part_pr_step: no iteration pending (call mg_part_pr_begin, then step and merge in turn)");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  PrbArgs a;
  std::memset(&a, 0, sizeof(a));
  a.off = p->co;
  a.idx = p->ri;
  a.wts = nullptr;
  a.rows = p->prb.rows;
  a.hrows = p->prb.hrows;
  a.hbase = p->prb.hbase;
  a.hcount = p->prb.hcount;
  a.hpart = p->prb.hpart;
  a.hcontrib = p->prb.hcontrib;
  a.grab = p->prb.grab;
  for (int b = 0; b <= PRB_BINS; b++) {
    a.boff[b] = p->prb.boff[b];
    a.wstart[b] = p->prb.wstart[b];
  }
  a.nheavy = p->prb.nheavy;
  if (p->hi > p->lo)
    part_pr_kernel<<<p->num_sms * PRB_MIN_BLOCKS, PRB_NT, 0, p->stream>>>(a, p->y, slice, p->alpha, p->tn, p->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  p->pr_stepped = true;
  return MG_OK;
}

extern "C" mg_status mg_part_pr_merge(mg_part *p, const float *gathered, int32_t world, int64_t stride,
                                      const int64_t *cuts, mg_part_level *level) {
  using namespace mg;
  if (!p || !gathered || !cuts || world <= 0 || stride < 0) {
    mg_set_error("mg_part_pr_merge: null argument, world <= 0 or stride < 0");
    return MG_ERR_ARG;
  }
  if (!p->pr_stepped) {
    mg_set_error("mg_part_pr_merge: no step to merge");
    return MG_ERR_ARG;
  }
  bool mine = false;
  if (cuts[0] != 0 || cuts[world] != p->n) {
    mg_set_error("mg_part_pr_merge: cuts must run from 0 to n");
    return MG_ERR_ARG;
  }
  for (int32_t r = 0; r < world; r++) {
    if (cuts[r + 1] < cuts[r] || cuts[r + 1] - cuts[r] > stride) {
      mg_set_error("mg_part_pr_merge: cuts must be non-decreasing with slices of at most stride entries");
      return MG_ERR_ARG;
    }
    mine = mine || (cuts[r] == p->lo && cuts[r + 1] == p->hi);
  }
  if (!mine) {
    mg_set_error("mg_part_pr_merge: no slice of the cuts is this partition's [lo, hi)");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  for (int32_t r = 0; r < world; r++) {
    const int64_t len = cuts[r + 1] - cuts[r];
    if (len > 0)
      MG_CUDA_TRY(cudaMemcpyAsync(p->xn + cuts[r], gathered + (size_t)r * stride, sizeof(float) * (size_t)len,
                                  cudaMemcpyDeviceToDevice, s));
  }
  part_pr_merge_kernel<<<p->pgrid, 256, 0, s>>>(p->n, p->xo, p->xn, p->deg, p->y, p->ppart);
  part_pr_reduce_kernel<<<1, 256, 0, s>>>(p->ppart, p->pgrid, p->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(PartCtl), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  std::swap(p->xo, p->xn);
  p->pr_stepped = false;
  p->pr_level += 1;
  p->resid = p->ctl_host->resid;
  p->pr_done = p->resid < p->tol || p->pr_level >= p->pr_max_iter;
  fill_pr_level(p, level);
  return MG_OK;
}

extern "C" mg_status mg_part_pr_result(mg_part *p, float *ranks, int32_t device_output, mg_stats *stats) {
  using namespace mg;
  if (!p || !ranks) {
    mg_set_error("mg_part_pr_result: null argument");
    return MG_ERR_ARG;
  }
  if (!p->pr_begun) {
    mg_set_error("mg_part_pr_result: no run (call mg_part_pr_begin first)");
    return MG_ERR_ARG;
  }
  MG_CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  MG_CUDA_TRY(cudaEventRecord(p->ev1, s));
  MG_CUDA_TRY(cudaMemcpyAsync(ranks, p->xo, sizeof(float) * (size_t)p->n,
                              device_output ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = p->pr_level;
    stats->edges_traversed = p->m_total * p->pr_level;
    stats->edges_inspected = p->m_in * p->pr_level;
    stats->residual = p->resid;
    stats->bytes_compulsory =
        p->pr_level * (4 * (p->hi - p->lo + 1) + 4 * p->m_in + 4 * (p->hi - p->lo) + 16 * p->n);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p->ev0, p->ev1);
    stats->kernel_ms = ms;
    stats->launches = 2 + 3 * (int64_t)p->pr_level;
  }
  return MG_OK;
}
