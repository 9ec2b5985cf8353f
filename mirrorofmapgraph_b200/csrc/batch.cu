// batch.cu -- batched traversals. No reference counterpart: the reference runs
// the whole engine once per source (Algorithms/BFS/bfs.cu:442-456), each run
// with its own context, allocations and per-level host round trips.
//
// mg_bfs_batch: bit-parallel multi-source BFS. Up to 64 sources share one pass
// over the graph. Every vertex carries 64-bit masks: `seen` (sources that have
// reached it), the frontier (sources that reached it in the last level) and, for
// top-down levels, an accumulator of sources arriving in this level. One edge
// read serves all the sources of the group. A level runs either
//   - top-down: the union frontier (vertices with a non-empty frontier mask) is
//     expanded with the degree-binned tile expansion and each edge ORs the
//     sender's frontier mask, minus the sources the receiver has already seen,
//     into the receiver's accumulator; a finishing pass commits the new bits, or
//   - bottom-up: every vertex still missing some source ORs its in-neighbours'
//     frontier masks and stops as soon as every missing source has arrived,
// chosen per level from the out-edges of the union frontier. Depth rows:
// depth[i * n + v] = level at which source i reached v, -1 if never. BFS levels
// are unique, so every row equals a single-source mg_bfs from srcs[i].
//
// mg_bfs_ragged: the members of a ragged batch are disjoint inside the union
// graph, so one multi-source BFS from every member's source (shifted by its
// vertex base) is every member's own BFS, in one device run.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"

namespace mg {

constexpr int MS_NT = 256;
constexpr int MS_CTA_TH = 512;
constexpr int MS_WIDTH = 64;        // sources per bit-parallel group
constexpr int MS_PULL_SERIAL = 8;   // in-edges a lane scans alone before the warp helps
constexpr int64_t MS_ALPHA = 14;    // bottom-up when the union frontier's out-edges exceed m / MS_ALPHA

struct MsArgs {
  const int32_t *ro, *ci;  // out-edges (CSR)
  const int32_t *co, *ri;  // in-edges (CSC; the CSR itself for symmetric graphs)
  uint64_t *seen, *f0, *f1, *acc;
  int32_t *q0, *q1;
  int32_t qcap;
  int32_t *big_v;  // grid-strided bin (BIG_CAP vertices)
  int32_t *depth;  // the group's first depth row (k rows of n)
  int64_t n, m_total;
  uint64_t full;   // mask of the group's sources
  int32_t mode, can_pull, both;
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

__device__ void ms_level_end(const MsArgs &a) {
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nf = vload(&c->qlen[cur ^ 1]);
  const int64_t mf = vload(&c->mf_next);
  const int lvl = vload(&c->level) + 1;
  c->level = lvl;
  c->qlen[cur] = 0;
  c->cur = cur ^ 1;
  c->mf_next = 0;
  c->blocks_done = 0;
  c->big_len = 0;
  const bool over = vload(&c->overflow) != 0;
  const bool done = nf == 0 || lvl >= c->iter_cap || over;
  int dir = 0;
  if (a.mode == MG_DIR_PULL) dir = a.can_pull ? 1 : 0;
  else if (a.mode == MG_DIR_AUTO && a.can_pull) dir = mf * MS_ALPHA > a.m_total ? 1 : 0;
  if (dir == 1 && !done) c->levels_pull += 1;
  c->dir = dir;
  c->nf_next = nf;
  if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
  __threadfence();
  c->done = done ? 1 : 0;
  if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
}

__device__ __forceinline__ bool ms_skip(const MsArgs &a, int want_dir) {
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return true;
  }
  return vload(&c->dir) != want_dir;
}

// Writes depth d of every lane's vertex v for each source bit in its `nw`.
// Called by the whole warp (lanes without a vertex pass nw = 0): the warp walks
// the union of its lanes' bits source by source, so the stores of one source go
// to consecutive vertices of one depth row.
__device__ __forceinline__ void ms_write_depths(int32_t *depth, int64_t n, int64_t v, uint64_t nw, int32_t d) {
  const unsigned lo = __reduce_or_sync(FULL, (unsigned)nw), hi = __reduce_or_sync(FULL, (unsigned)(nw >> 32));
  uint64_t any = ((uint64_t)hi << 32) | lo;
  while (any) {
    const int i = __ffsll((long long)any) - 1;
    any &= any - 1;
    if ((nw >> i) & 1) depth[(int64_t)i * n + v] = d;
  }
}

// Top-down expansion of the union frontier into the accumulators.
__global__ void __launch_bounds__(MS_NT) ms_push_kernel(MsArgs a) {
  __shared__ ExpandSmem<MS_NT, uint64_t> sm;
  __shared__ int64_t s_sum[MS_NT / 32 + 1];
  if (ms_skip(a, 0)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  const uint64_t *fcur = cur ? a.f1 : a.f0;
  const uint64_t *seen = a.seen;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(a.acc);
  const int32_t *ci = a.ci, *ri = a.ri;
  int64_t insp = 0, nexp = 0;
  const BigList big{a.big_v, &c->big_len, defer_threshold<MS_NT>(nin, MS_CTA_TH)};
  auto visit_to = [&](uint64_t f, int32_t w) {
    const uint64_t add = f & ~__ldg(seen + w);
    if (add) atomicOr(acc + w, (unsigned long long)add);
  };
  for (int64_t tile = (int64_t)blockIdx.x * MS_NT; tile < nin; tile += (int64_t)gridDim.x * MS_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < nin ? qin[i] : -1;
    nexp += v >= 0;
    const uint64_t f = v >= 0 ? __ldg(fcur + v) : 0;  // the sender's frontier mask, once per vertex
    expand_tile_p<MS_NT, MS_CTA_TH>(sm, a.ro, v, f, insp,
                                    [&](int32_t, uint64_t fv, int32_t k) { visit_to(fv, ci[k]); }, &big);
    if (a.both)
      expand_tile_p<MS_NT, MS_CTA_TH>(sm, a.co, v, f, insp,
                                      [&](int32_t, uint64_t fv, int32_t k) { visit_to(fv, ri[k]); });
  }
  const int64_t bins = block_sum<MS_NT>(insp, s_sum);
  const int64_t bexp = block_sum<MS_NT>(nexp, s_sum);
  if (threadIdx.x == 0) {
    if (bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
    if (bexp) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)bexp);
  }
}

// Grid-strided bin of a top-down level: the out-edges of the deferred hubs spread
// over every CTA.
__global__ void __launch_bounds__(MS_NT) ms_push_big_kernel(MsArgs a) {
  __shared__ BigSmem<MS_NT> sm;
  if (ms_skip(a, 0)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const uint64_t *fcur = cur ? a.f1 : a.f0;
  const uint64_t *seen = a.seen;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(a.acc);
  const int32_t *ci = a.ci;
  expand_big<MS_NT>(sm, a.ro, BigList{a.big_v, &c->big_len}, [&](int32_t sv, int32_t k) {
    const int32_t w = ci[k];
    const uint64_t add = __ldg(fcur + sv) & ~__ldg(seen + w);
    if (add) atomicOr(acc + w, (unsigned long long)add);
  });
}

// Commits a top-down level: new bits = accumulated & ~seen; rewrites every
// vertex's next-frontier mask and clears the accumulators it read.
__global__ void __launch_bounds__(MS_NT) ms_finish_kernel(MsArgs a) {
  __shared__ int64_t s_sum[MS_NT / 32 + 1];
  if (ms_skip(a, 0)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t d = vload(&c->level) + 1;
  uint64_t *fnext = cur ? a.f0 : a.f1;
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen_out = &c->qlen[cur ^ 1];
  int64_t mf = 0, vdeg = 0;
  const int64_t stride = (int64_t)gridDim.x * MS_NT;
  for (int64_t base = (int64_t)blockIdx.x * MS_NT; base < a.n; base += stride) {
    const int64_t w = base + threadIdx.x;
    uint64_t nw = 0;
    if (w < a.n) {
      const uint64_t ac = a.acc[w];
      if (ac) {
        a.acc[w] = 0;
        const uint64_t s = a.seen[w];
        nw = ac & ~s;
        if (nw) {
          a.seen[w] = s | nw;
          const int64_t deg = a.ro[w + 1] - a.ro[w];
          mf += deg;
          vdeg += deg * __popcll(nw);
        }
      }
      fnext[w] = nw;
    }
    ms_write_depths(a.depth, a.n, w, nw, d);
    warp_append(nw != 0, (int32_t)w, qout, qlen_out, a.qcap, &c->overflow);
  }
  const int64_t bmf = block_sum<MS_NT>(mf, s_sum);
  const int64_t bvd = block_sum<MS_NT>(vdeg, s_sum);
  if (threadIdx.x == 0) {
    if (bmf) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)bmf);
    if (bvd) atomicAdd((unsigned long long *)&c->visited_deg, (unsigned long long)bvd);
  }
  if (last_block(&c->blocks_done) && threadIdx.x == 0) ms_level_end(a);
}

// OR of the frontier masks over edges [beg, end) of one vertex per lane: each
// lane first scans up to MS_PULL_SERIAL edges alone; vertices with more edges
// still missing sources are then scanned by the whole warp, one at a time,
// 32 edges per step, until every missing source has arrived.
__device__ __forceinline__ uint64_t ms_gather(const int32_t *__restrict__ off, const int32_t *__restrict__ idx,
                                              const uint64_t *__restrict__ fcur, bool need, int64_t v, uint64_t miss,
                                              uint64_t acc, int64_t &insp) {
  const int lane = lane_id();
  int32_t beg = 0, end = 0;
  if (need && (acc & miss) != miss) {
    beg = off[v];
    end = off[v + 1];
  }
  const int32_t lim = min(end, beg + MS_PULL_SERIAL);
  for (int32_t e = beg; e < lim; e++) {
    insp++;
    acc |= __ldg(fcur + idx[e]);
    if ((acc & miss) == miss) break;
  }
  unsigned pend = __ballot_sync(FULL, need && (acc & miss) != miss && lim < end);
  while (pend) {
    const int l = __ffs(pend) - 1;
    pend &= pend - 1;
    const int32_t b = __shfl_sync(FULL, lim, l), en = __shfl_sync(FULL, end, l);
    const uint64_t m = __shfl_sync(FULL, miss, l);
    uint64_t got = __shfl_sync(FULL, acc, l);
    for (int32_t e0 = b; e0 < en; e0 += 32) {
      const int32_t e = e0 + lane;
      uint64_t x = 0;
      if (e < en) {
        x = __ldg(fcur + idx[e]);
        insp++;
      }
      const unsigned lo = __reduce_or_sync(FULL, (unsigned)x), hi = __reduce_or_sync(FULL, (unsigned)(x >> 32));
      got |= ((uint64_t)hi << 32) | lo;
      if ((got & m) == m) break;
    }
    if (lane == l) acc = got;
  }
  return acc;
}

// Bottom-up level: every vertex still missing sources gathers its in-neighbours'
// frontier masks; commits the new bits and rewrites the next-frontier masks.
__global__ void __launch_bounds__(MS_NT) ms_pull_kernel(MsArgs a) {
  __shared__ int64_t s_sum[MS_NT / 32 + 1];
  if (ms_skip(a, 1)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t d = vload(&c->level) + 1;
  const uint64_t *fcur = cur ? a.f1 : a.f0;
  uint64_t *fnext = cur ? a.f0 : a.f1;
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen_out = &c->qlen[cur ^ 1];
  int64_t mf = 0, vdeg = 0, insp = 0, nexp = 0;
  const BigList big{a.big_v, &c->big_len};
  const int64_t stride = (int64_t)gridDim.x * MS_NT;
  for (int64_t base = (int64_t)blockIdx.x * MS_NT; base < a.n; base += stride) {
    const int64_t v = base + threadIdx.x;
    const bool in = v < a.n;
    const uint64_t s = in ? a.seen[v] : a.full;
    const uint64_t miss = a.full & ~s;
    bool need = miss != 0;
    nexp += need;
    // In-degrees of GRID_TH and more go to the grid-strided bin (ms_pull_big_kernel).
    if (need && !a.both && a.co[v + 1] - a.co[v] >= GRID_TH && defer_big(big, (int32_t)v, GRID_TH)) need = false;
    uint64_t acc = ms_gather(a.co, a.ri, fcur, need, v, miss, 0, insp);
    if (a.both) acc = ms_gather(a.ro, a.ci, fcur, need, v, miss, acc, insp);
    const uint64_t nw = acc & miss;
    if (in) {
      if (nw) {
        a.seen[v] = s | nw;
        const int64_t deg = a.ro[v + 1] - a.ro[v];
        mf += deg;
        vdeg += deg * __popcll(nw);
      }
      fnext[v] = nw;
    }
    ms_write_depths(a.depth, a.n, v, nw, d);
    warp_append(nw != 0, (int32_t)v, qout, qlen_out, a.qcap, &c->overflow);
  }
  const int64_t bmf = block_sum<MS_NT>(mf, s_sum);
  const int64_t bvd = block_sum<MS_NT>(vdeg, s_sum);
  const int64_t bins = block_sum<MS_NT>(insp, s_sum);
  const int64_t bexp = block_sum<MS_NT>(nexp, s_sum);
  if (threadIdx.x == 0) {
    if (bmf) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)bmf);
    if (bvd) atomicAdd((unsigned long long *)&c->visited_deg, (unsigned long long)bvd);
    if (bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
    if (bexp) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)bexp);
  }
}

// Grid-strided bin of a bottom-up level: every CTA ORs the frontier masks of an
// equal slice of the deferred hubs' in-edges into their accumulators; the last
// CTA commits the hubs' new bits and closes the level.
__global__ void __launch_bounds__(MS_NT) ms_pull_big_kernel(MsArgs a) {
  __shared__ BigSmem<MS_NT> sm;
  __shared__ int64_t s_sum[MS_NT / 32 + 1];
  if (ms_skip(a, 1)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const uint64_t *fcur = cur ? a.f1 : a.f0;
  const uint64_t *seen = a.seen;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(a.acc);
  const int32_t *ri = a.ri;
  const uint64_t full = a.full;
  int64_t insp = 0;
  expand_big<MS_NT>(sm, a.co, BigList{a.big_v, &c->big_len}, [&](int32_t v, int32_t k) {
    insp++;
    const uint64_t x = __ldg(fcur + ri[k]) & full & ~__ldg(seen + v);
    if (x && (x & ~__ldcg(reinterpret_cast<const uint64_t *>(acc) + v))) atomicOr(acc + v, (unsigned long long)x);
  });
  const int64_t bins = block_sum<MS_NT>(insp, s_sum);
  if (threadIdx.x == 0 && bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
  if (!last_block(&c->blocks_done)) return;
  const int32_t d = vload(&c->level) + 1;
  uint64_t *fnext = cur ? a.f0 : a.f1;
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen_out = &c->qlen[cur ^ 1];
  const int32_t nb = min(vload(&c->big_len), BIG_CAP);
  int64_t mf = 0, vdeg = 0;
  for (int32_t i = threadIdx.x; i < nb; i += MS_NT) {
    const int32_t v = a.big_v[i];
    const uint64_t ac = __ldcg(a.acc + v);
    a.acc[v] = 0;
    const uint64_t s = a.seen[v];
    uint64_t nw = ac & full & ~s;
    fnext[v] = nw;
    if (nw) {
      a.seen[v] = s | nw;
      const int64_t deg = a.ro[v + 1] - a.ro[v];
      mf += deg;
      vdeg += deg * __popcll(nw);
      while (nw) {
        const int j = __ffsll((long long)nw) - 1;
        nw &= nw - 1;
        a.depth[(int64_t)j * a.n + v] = d;
      }
      const int32_t pos = atomicAdd(qlen_out, 1);
      if (pos < a.qcap) qout[pos] = v;
      else c->overflow = 1;
    }
  }
  const int64_t bmf = block_sum<MS_NT>(mf, s_sum);
  const int64_t bvd = block_sum<MS_NT>(vdeg, s_sum);
  if (threadIdx.x == 0) {
    c->mf_next = vload(&c->mf_next) + bmf;
    c->visited_deg = vload(&c->visited_deg) + bvd;
    __threadfence();
    ms_level_end(a);
  }
}

// Masks := 0; the group's depth rows := -1.
__global__ void ms_clear_kernel(MsArgs a, int32_t k) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    a.seen[i] = 0;
    a.f0[i] = 0;
    a.f1[i] = 0;
    a.acc[i] = 0;
  }
  const int64_t total = (int64_t)k * a.n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) a.depth[i] = -1;
}

// Seeds the group's sources (bit i for srcs[i]; equal sources share a vertex).
__global__ void ms_seed_kernel(MsArgs a, const int32_t *srcs, int32_t k, int32_t iter_cap, int32_t dir0) {
  __shared__ int64_t s_sum[1024 / 32 + 1];
  DevCtl *c = a.ctl;
  int64_t mf = 0, vdeg = 0;
  unsigned long long *seen = reinterpret_cast<unsigned long long *>(a.seen);
  unsigned long long *f0 = reinterpret_cast<unsigned long long *>(a.f0);
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    const int32_t s = srcs[i];
    const unsigned long long bit = 1ull << i;
    const int64_t deg = a.ro[s + 1] - a.ro[s];
    atomicOr(seen + s, bit);
    a.depth[(int64_t)i * a.n + s] = 0;
    vdeg += deg;
    if (atomicOr(f0 + s, bit) == 0ull) {
      mf += deg;
      const int pos = atomicAdd(&c->qlen[0], 1);
      if (pos < a.qcap) a.q0[pos] = s;
      else c->overflow = 1;
    }
  }
  const int64_t tm = block_sum<1024>(mf, s_sum);
  const int64_t tv = block_sum<1024>(vdeg, s_sum);
  if (threadIdx.x == 0) {
    c->visited_deg = tv;
    c->mf_next = 0;
    c->level = 0;
    c->cur = 0;
    int dir = dir0;
    if (a.mode == MG_DIR_AUTO && a.can_pull) dir = tm * MS_ALPHA > a.m_total ? 1 : 0;
    c->dir = dir;
    if (dir == 1) c->levels_pull = 1;
    c->iter_cap = iter_cap;
    c->done = (iter_cap <= 0 || c->overflow) ? 1 : 0;
    if (c->overflow) c->status = MG_ERR_QUEUE_OVERFLOW;
  }
}

}  // namespace mg

// Runs the bit-parallel BFS of every group of up to 64 sources into `depth`
// (device, nsrc x n).
static mg_status msbfs_run(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth, const mg_opts &o,
                           mg_stats *stats) {
  using namespace mg;
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool undirected = o.directed == 0 && !symmetric;
  if (undirected && !g->has_csc) {
    mg_set_error("mg_bfs_batch: directed=0 needs the CSC (graph created with MG_GRAPH_NO_CSC)");
    return MG_ERR_UNSUPPORTED;
  }
  const int64_t n = g->n;
  const size_t need = Carve::need({sizeof(uint64_t) * (size_t)n, sizeof(uint64_t) * (size_t)n,
                                   sizeof(uint64_t) * (size_t)n, sizeof(uint64_t) * (size_t)n,
                                   sizeof(int32_t) * (size_t)n, sizeof(int32_t) * (size_t)n,
                                   sizeof(int32_t) * (size_t)BIG_CAP, sizeof(int32_t) * (size_t)nsrc});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  MsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.seen = cv.take<uint64_t>(n);
  a.f0 = cv.take<uint64_t>(n);
  a.f1 = cv.take<uint64_t>(n);
  a.acc = cv.take<uint64_t>(n);
  a.q0 = cv.take<int32_t>(n);
  a.q1 = cv.take<int32_t>(n);
  a.big_v = cv.take<int32_t>(BIG_CAP);
  int32_t *dsrc = cv.take<int32_t>(nsrc);
  a.qcap = (int32_t)n;
  a.ro = g->ro;
  a.ci = g->ci;
  a.co = g->has_csc ? g->co : g->ro;
  a.ri = g->has_csc ? g->ri : g->ci;
  a.n = n;
  a.m_total = g->m;
  a.mode = o.direction;
  a.can_pull = g->has_csc || symmetric;
  a.both = undirected ? 1 : 0;
  a.ctl = g->ctl;
  cudaStream_t s = g->stream;
  const int32_t iter_cap = o.iter_num > 0 ? (int32_t)std::min<int64_t>(o.iter_num, n + 1) : (int32_t)(n + 1);
  const int32_t dir0 = (o.direction == MG_DIR_PULL && a.can_pull) ? 1 : 0;
  MG_CUDA_TRY(cudaMemcpyAsync(dsrc, srcs, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  const int grid = g->num_sms * 4;
  const bool use_graph = o.use_graph >= 0;
  int64_t iters = 0, vdeg = 0, insp = 0, launches = 0, pulls = 0;
  float ms_total = 0.f;
  for (int32_t g0 = 0; g0 < nsrc; g0 += MS_WIDTH) {
    const int32_t k = std::min<int32_t>(MS_WIDTH, nsrc - g0);
    a.depth = depth + (int64_t)g0 * n;
    a.full = k == 64 ? ~0ull : ((1ull << k) - 1);
    MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
    MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
    ms_clear_kernel<<<g->num_sms * 8, 256, 0, s>>>(a, k);
    ms_seed_kernel<<<1, 1024, 0, s>>>(a, dsrc + g0, k, iter_cap, dir0);
    MG_CUDA_TRY(cudaGetLastError());
    struct Sig {
      MsArgs a;
      int grid;
    } sig;
    std::memset(&sig, 0, sizeof(sig));
    sig.a = a;
    sig.grid = grid;
    LoopBody body = [a, grid](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
      MsArgs b = a;
      b.h = h;
      b.use_cond = use_cond;
      ms_push_kernel<<<grid, MS_NT, 0, st>>>(b);
      ms_push_big_kernel<<<grid, MS_NT, 0, st>>>(b);
      ms_finish_kernel<<<grid, MS_NT, 0, st>>>(b);
      ms_pull_kernel<<<grid, MS_NT, 0, st>>>(b);
      ms_pull_big_kernel<<<grid, MS_NT, 0, st>>>(b);
    };
    MG_TRY(run_loop(g, SLOT_MSBFS, &sig, sizeof(sig), use_graph, body, n + 2));
    MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
    MG_TRY(fetch_ctl(g));
    const DevCtl &hc = *g->ctl_host;
    if (hc.status != 0) {
      mg_set_error("mg_bfs_batch: device status %d", hc.status);
      return (mg_status)hc.status;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    ms_total += ms;
    iters = std::max<int64_t>(iters, hc.level);
    vdeg += hc.visited_deg;
    insp += hc.edges_inspected;
    pulls += hc.levels_pull;
    launches += 2 + (use_graph ? 6 * (int64_t)hc.body_iters : 5 * (int64_t)hc.level);
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = iters;
    stats->edges_traversed = vdeg;
    stats->edges_inspected = insp;
    stats->bytes_compulsory = 12 * insp + 40 * n * iters + 4 * (int64_t)nsrc * n;
    stats->kernel_ms = ms_total;
    stats->status_detail = (int32_t)pulls;
    stats->launches = launches;
  }
  return MG_OK;
}

extern "C" mg_status mg_bfs_batch(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth,
                                  const mg_opts *opts, mg_stats *stats) {
  if (!g || !srcs || nsrc <= 0 || !depth) {
    mg_set_error("mg_bfs_batch: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  if (o.direction < MG_DIR_AUTO || o.direction > MG_DIR_PULL) {
    mg_set_error("mg_bfs_batch: invalid direction %d", o.direction);
    return MG_ERR_ARG;
  }
  for (int32_t i = 0; i < nsrc; i++) {
    if (srcs[i] < 0 || srcs[i] >= g->n) {
      mg_set_error("mg_bfs_batch: source %d out of range [0, %lld)", srcs[i], (long long)g->n);
      return MG_ERR_ARG;
    }
  }
  MG_TRY(graph_enter(g));
  if (o.device_output) MG_TRY(check_device_ptr(g, depth, "mg_bfs_batch", "depth"));
  const size_t bytes = sizeof(int32_t) * (size_t)nsrc * (size_t)g->n;
  int32_t *out = depth;
  if (!o.device_output) {
    MG_TRY(ws_reserve(g, g->ws_out, bytes + 256));
    out = (int32_t *)g->ws_out.ptr;
  }
  MG_TRY(msbfs_run(g, srcs, nsrc, out, o, stats));
  if (!o.device_output) {
    MG_TRY(copy_out(g, depth, out, bytes, 0));
    MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  return MG_OK;
}

extern "C" mg_status mg_bfs_ragged(mg_graph *g, const int32_t *srcs, int32_t *depth, const mg_opts *opts,
                                   mg_stats *stats) {
  if (!g || !srcs || !depth) {
    mg_set_error("mg_bfs_ragged: null argument");
    return MG_ERR_ARG;
  }
  if (g->vbase.size() < 2) {
    mg_set_error("mg_bfs_ragged: the graph is not a ragged batch (create it with mg_graph_create_ragged)");
    return MG_ERR_ARG;
  }
  const int32_t ng = (int32_t)g->vbase.size() - 1;
  std::vector<int32_t> global(ng);
  for (int32_t i = 0; i < ng; i++) {
    const int64_t ni = g->vbase[i + 1] - g->vbase[i];
    if (srcs[i] < 0 || srcs[i] >= ni) {
      mg_set_error("mg_bfs_ragged: source %d of member graph %d out of range [0, %lld)", srcs[i], i,
                   (long long)ni);
      return MG_ERR_ARG;
    }
    global[i] = (int32_t)(g->vbase[i] + srcs[i]);
  }
  return mg_bfs(g, global.data(), ng, depth, opts, stats);
}
