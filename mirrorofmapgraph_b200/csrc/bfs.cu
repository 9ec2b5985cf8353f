// bfs.cu -- breadth-first search (struct bfs, Algorithms/BFS/bfs.h:28-262).
//
// Per level one of two kernels does the work and the last CTA to finish closes
// the level (swap queues, pick the next direction, stop or continue):
//
//  push (top-down)  input: vertex queue. Each CTA takes a tile of 256 frontier
//                   vertices and bins them by out-degree: >= CTA_TH edges are
//                   expanded by the whole CTA, >= 32 by one warp, the rest by a
//                   block-wide scan over the remaining degrees (thread-level
//                   bin), so every edge load is coalesced. A neighbour is claimed
//                   with atomicOr on a visited bitmap (1 bit per vertex); the
//                   winner writes depth = level + 1 and appends itself to the
//                   output queue with a warp-aggregated atomic.
//                   This replaces expand_atomic + contract_atomic
//                   (GASengine/vertex_centric/expand_atomic/cta.cuh:268-759,
//                   contract_atomic/cta.cuh:203-612): no edge-sized frontier is
//                   ever materialised, the dedup is exact, and BFS's contract
//                   (label := iteration + 1, bfs.h:229-255) is fused in.
//  pull (bottom-up) every unvisited vertex scans its in-edges for a parent whose
//                   depth equals the current level and stops at the first hit.
//                   A warp owns 32 consecutive vertices, i.e. one bitmap word,
//                   so visited words are updated without atomics.
//
// The direction switch (Beamer's heuristic: go bottom-up when the frontier's
// out-edges exceed 1/14 of the unexplored edges, back when the frontier drops
// below n/24) is evaluated on the device.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"

namespace mg {

constexpr int BFS_NT = 256;
constexpr int BFS_CTA_TH = 512;   // out-degree at or above which a CTA expands the vertex
constexpr int PULL_SERIAL = 8;    // in-edges a lane scans alone before the warp helps
// Beamer's direction rule (mg_tuning.bfs_alpha / bfs_beta, defaults 14 and 24):
// pull when the frontier's out-edges exceed the unvisited vertices' out-edges /
// alpha, back to push when the frontier holds fewer than n / beta vertices. AUTO
// runs top-down only on graphs of mean out-degree <= bfs_sparse_degree (8).

struct BfsArgs {
  const int32_t *ro, *ci;  // out-edges (CSR)
  const int32_t *co, *ri;  // in-edges (CSC; the CSR itself for symmetric graphs)
  int32_t *label;
  uint32_t *vis;
  int32_t *q0, *q1;
  int32_t qcap;
  int32_t mode;      // MG_DIR_*
  int32_t can_pull;  // in-edges available and traversal direction allows it
  int32_t both;      // directed == 0 on a non-symmetric graph: expand CSR and CSC
  int64_t n;
  int64_t m_total;
  int32_t *big_v;  // grid-strided bin of the push direction (BIG_CAP entries)
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
  uint32_t bar_extra;            // test hook (mg_debug_barrier_skew): a barrier that cannot complete
  unsigned long long bar_limit;  // barrier polls before MG_ERR_TIMEOUT
  // tuned thresholds (mg_tuning): CTA-bin and grid-bin out-degrees, the warp-bin
  // deferral rule, the persistent kernel's frontier limits, Beamer's constants
  int32_t cta_th, grid_th, defer_warp;
  int32_t persist_max;
  int64_t persist_edges;
  int64_t alpha, beta;
};

// The graph's tuned BFS thresholds into the kernel arguments.
inline void bfs_tuning(BfsArgs &a, const mg_tuning &t) {
  a.cta_th = t.bfs_cta_th;
  a.grid_th = t.bfs_grid_th;
  a.defer_warp = t.bfs_defer_warp;
  a.persist_max = t.bfs_persist_max;
  a.persist_edges = t.bfs_persist_edges;
  a.alpha = t.bfs_alpha;
  a.beta = t.bfs_beta;
}

__device__ void bfs_level_end(const BfsArgs &a) {
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nf = vload(&c->qlen[cur ^ 1]);
  const int64_t mf = vload(&c->mf_next);
  const int64_t vdeg = vload(&c->visited_deg) + mf;
  const int lvl = vload(&c->level) + 1;
  trace_level(c, lvl - 1, vload(&c->dir) == 1 ? MG_DIR_PULL : MG_DIR_PUSH, vload(&c->qlen[cur]),
              vload(&c->mf_front), 0.0);
  c->visited_deg = vdeg;
  c->mf_front = mf;
  c->level = lvl;
  c->qlen[cur] = 0;
  c->cur = cur ^ 1;
  c->mf_next = 0;
  c->blocks_done = 0;
  c->big_len = 0;
  // the persistent kernel's per-level counters start from zero when it next runs
  for (int k = 0; k < 3; k++) {
    c->pq[k] = 0;
    c->pm[k] = 0;
    c->pb[k] = 0;
  }
  const bool over = vload(&c->overflow) != 0;
  const bool done = nf == 0 || lvl >= c->iter_cap || over;
  int dir = vload(&c->dir);
  if (!done) {
    if (a.mode == MG_DIR_PULL) {
      dir = a.can_pull ? 1 : 0;
    } else if (a.mode == MG_DIR_PUSH || !a.can_pull) {
      dir = 0;
    } else if (dir == 0) {
      if (mf > (a.m_total - vdeg) / a.alpha) dir = 1;
    } else {
      if ((int64_t)nf * a.beta < a.n) dir = 0;
    }
  }
  if (dir == 1 && !done) c->levels_pull += 1;
  c->dir = dir;
  c->nf_next = nf;
  if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
  __threadfence();
  c->done = done ? 1 : 0;
  if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
}

// Early exit shared by both kernels: when the run is already over, make sure
// the WHILE node stops.
__device__ __forceinline__ bool bfs_skip(const BfsArgs &a, int want_dir) {
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return true;
  }
  return vload(&c->dir) != want_dir;
}

// Per-thread state of a push level (plain copies, so nothing is read through
// the kernel-parameter block).
struct PushCtx {
  int32_t *label;
  uint32_t *vis;
  const int32_t *ro;
  int32_t *qout;
  int32_t *qlen_out;
  int32_t *overflow;
  int32_t qcap;
  int32_t level;
  int64_t mf;
  BlockQueue *bq = nullptr;  // staging of discoveries (nullptr: straight to the queue)
};

__device__ __forceinline__ void bfs_visit(PushCtx &x, int32_t u) {
  const uint32_t bit = 1u << (u & 31);
  uint32_t *wp = x.vis + (u >> 5);
  bool disc = false;
  if (!(*wp & bit)) {
    uint32_t old = atomicOr(wp, bit);
    disc = !(old & bit);
  }
  if (disc) {
    x.label[u] = x.level + 1;
    x.mf += x.ro[u + 1] - x.ro[u];
  }
  staged_append(x.bq, disc, u, x.qout, x.qlen_out, x.qcap, x.overflow);
}

__global__ void __launch_bounds__(BFS_NT) bfs_push_kernel(BfsArgs a) {
  __shared__ ExpandSmem<BFS_NT> sm;
  __shared__ BlockQueue bq;
  __shared__ int64_t s_sum[BFS_NT / 32 + 1];
  if (bfs_skip(a, 0)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  PushCtx x{a.label, a.vis, a.ro, cur ? a.q0 : a.q1, &c->qlen[cur ^ 1], &c->overflow, a.qcap, vload(&c->level), 0};
  bq_init(bq);
  x.bq = &bq;
  int64_t insp = 0, nexp = 0;
  const BigList big{a.big_v, &c->big_len, defer_threshold<BFS_NT>(nin, a.cta_th, a.grid_th, a.defer_warp)};
  for (int64_t tile = (int64_t)blockIdx.x * BFS_NT; tile < nin; tile += (int64_t)gridDim.x * BFS_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < nin ? qin[i] : -1;
    nexp += v >= 0;
    const int32_t *ci = a.ci, *ri = a.ri;
    expand_tile<BFS_NT, BFS_CTA_TH>(sm, a.ro, v, insp, [&](int32_t, int32_t k) { bfs_visit(x, ci[k]); }, &big, -1,
                                    a.cta_th);
    if (a.both)
      expand_tile<BFS_NT, BFS_CTA_TH>(sm, a.co, v, insp, [&](int32_t, int32_t k) { bfs_visit(x, ri[k]); }, nullptr,
                                      -1, a.cta_th);
  }
  bq_flush(bq, x.qout, x.qlen_out, x.qcap, x.overflow);
  const int64_t bmf = block_sum<BFS_NT>(x.mf, s_sum);
  const int64_t bins = block_sum<BFS_NT>(insp, s_sum);
  const int64_t bexp = block_sum<BFS_NT>(nexp, s_sum);
  if (threadIdx.x == 0) {
    if (bmf) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)bmf);
    if (bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
    if (bexp) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)bexp);
  }
}

// Persistent push levels for small frontiers (high-diameter graphs such as
// lattices, where a BFS has thousands of levels of a few thousand vertices and
// per-level launches dominate). One cooperative launch runs level after level,
// with a grid barrier between the expansion and the level end, while the level is
// a push level with at most bfs_persist_max frontier vertices and bfs_persist_edges
// frontier out-edges; it then returns and the per-level kernels continue from the
// same control block. Vertices of GRID_TH or more edges are deferred as in the
// per-level push and expanded by the whole grid after a second barrier, which
// only levels that deferred one take.
constexpr unsigned long long PERSIST_WAIT = 1ull << 22;  // barrier polls (seconds at most) before giving up

__global__ void __launch_bounds__(BFS_NT) bfs_persist_kernel(BfsArgs a) {
  // The tile pass and the grid-strided pass are separated by a grid barrier.
  __shared__ union {
    ExpandSmem<BFS_NT> e;
    BigSmem<BFS_NT> b;
  } sm;
  __shared__ BlockQueue bq;
  __shared__ int64_t s_sum[BFS_NT / 32 + 1];
  DevCtl *c = a.ctl;
  // Entry state, as the seed kernel or the last per-level kernel left it; every
  // block reads the same values and then takes the same decisions level by level.
  const int32_t l0 = vload(&c->level);
  int32_t lvl = l0, sel = vload(&c->cur);
  int32_t nin = vload(&c->qlen[sel]);
  int64_t mf = vload(&c->mf_front), vdeg = vload(&c->visited_deg);
  const int32_t iter_cap = vload(&c->iter_cap);
  if (vload(&c->done) || vload(&c->dir) != 0 || nin > a.persist_max || mf > a.persist_edges) return;
  bq_init(bq);
  for (;;) {
    // Per-level counters rotate over three slots: this level appends to `out`;
    // `zero` is the slot the next level appends to (nobody touches it now).
    const int out = (lvl - l0 + 1) % 3, zero = (lvl - l0 + 2) % 3;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->pq[zero] = 0;
      c->pm[zero] = 0;
      c->pb[zero] = 0;
    }
    const int32_t *qin = sel ? a.q1 : a.q0;
    PushCtx x{a.label, a.vis, a.ro, sel ? a.q0 : a.q1, &c->pq[out], &c->overflow, a.qcap, lvl, 0};
    x.bq = &bq;
    const BigList big{a.big_v, &c->pb[out], defer_threshold<BFS_NT>(nin, a.cta_th, a.grid_th, a.defer_warp)};
    const int32_t *ci = a.ci, *ri = a.ri;
    int64_t insp = 0, nexp = 0;
    for (int64_t tile = (int64_t)blockIdx.x * BFS_NT; tile < nin; tile += (int64_t)gridDim.x * BFS_NT) {
      const int64_t i = tile + threadIdx.x;
      const int32_t v = i < nin ? qin[i] : -1;
      nexp += v >= 0;
      expand_tile<BFS_NT, BFS_CTA_TH>(sm.e, a.ro, v, insp, [&](int32_t, int32_t k) { bfs_visit(x, ci[k]); }, &big,
                                      -1, a.cta_th);
      if (a.both)
        expand_tile<BFS_NT, BFS_CTA_TH>(sm.e, a.co, v, insp, [&](int32_t, int32_t k) { bfs_visit(x, ri[k]); },
                                        nullptr, -1, a.cta_th);
    }
    bq_flush(bq, x.qout, x.qlen_out, x.qcap, x.overflow);
    const int64_t bmf = block_sum<BFS_NT>(x.mf, s_sum);
    const int64_t bins = block_sum<BFS_NT>(insp, s_sum);
    const int64_t bexp = block_sum<BFS_NT>(nexp, s_sum);
    if (threadIdx.x == 0) {
      if (bmf) atomicAdd((unsigned long long *)&c->pm[out], (unsigned long long)bmf);
      if (bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
      if (bexp) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)bexp);
    }
    if (!grid_barrier(&c->bar_count, &c->bar_gen, a.bar_limit, a.bar_extra)) {
      if (threadIdx.x == 0) {
        c->status = MG_ERR_TIMEOUT;
        c->done = 1;
      }
      return;
    }
    if (vload(&c->pb[out]) > 0) {
      // The deferred vertices' edges, spread over the whole grid.
      x.mf = 0;
      expand_big<BFS_NT>(sm.b, a.ro, big, [&](int32_t, int32_t k) { bfs_visit(x, ci[k]); });
      bq_flush(bq, x.qout, x.qlen_out, x.qcap, x.overflow);
      const int64_t bmf2 = block_sum<BFS_NT>(x.mf, s_sum);
      if (threadIdx.x == 0 && bmf2) atomicAdd((unsigned long long *)&c->pm[out], (unsigned long long)bmf2);
      if (!grid_barrier(&c->bar_count, &c->bar_gen, a.bar_limit, a.bar_extra)) {
        if (threadIdx.x == 0) {
          c->status = MG_ERR_TIMEOUT;
          c->done = 1;
        }
        return;
      }
    }
    // Level end (bfs_level_end's rules), computed alike in every block.
    if (blockIdx.x == 0 && threadIdx.x == 0) trace_level(c, lvl, MG_DIR_PUSH, nin, mf, 0.0);
    const int32_t nf = vload(&c->pq[out]);
    mf = vload(&c->pm[out]);
    vdeg += mf;
    lvl += 1;
    sel ^= 1;
    const bool over = vload(&c->overflow) != 0;
    const bool done = nf == 0 || lvl >= iter_cap || over;
    int dir = 0;
    if (a.mode == MG_DIR_PULL) dir = a.can_pull ? 1 : 0;
    else if (a.mode == MG_DIR_AUTO && a.can_pull && mf > (a.m_total - vdeg) / a.alpha) dir = 1;
    if (done || dir != 0 || nf > a.persist_max || mf > a.persist_edges) {
      // Hand over to the per-level kernels (or finish) with their control state.
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->level = lvl;
        c->cur = sel;
        c->qlen[sel] = nf;
        c->qlen[sel ^ 1] = 0;
        c->visited_deg = vdeg;
        c->mf_front = mf;
        c->mf_next = 0;
        c->blocks_done = 0;
        c->big_len = 0;
        c->nf_next = nf;
        c->dir = dir;
        if (dir == 1 && !done) c->levels_pull += 1;
        if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
        __threadfence();
        c->done = done ? 1 : 0;
      }
      return;
    }
    nin = nf;
  }
}

// Grid-strided bin of a push level: the deferred hubs' edges spread over every
// CTA; the last CTA closes the level.
__global__ void __launch_bounds__(BFS_NT) bfs_push_big_kernel(BfsArgs a) {
  __shared__ BigSmem<BFS_NT> sm;
  __shared__ BlockQueue bq;
  __shared__ int64_t s_sum[BFS_NT / 32 + 1];
  if (bfs_skip(a, 0)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  PushCtx x{a.label, a.vis, a.ro, cur ? a.q0 : a.q1, &c->qlen[cur ^ 1], &c->overflow, a.qcap, vload(&c->level), 0};
  bq_init(bq);
  x.bq = &bq;
  const int32_t *ci = a.ci;
  expand_big<BFS_NT>(sm, a.ro, BigList{a.big_v, &c->big_len}, [&](int32_t, int32_t k) { bfs_visit(x, ci[k]); });
  bq_flush(bq, x.qout, x.qlen_out, x.qcap, x.overflow);
  const int64_t bmf = block_sum<BFS_NT>(x.mf, s_sum);
  if (threadIdx.x == 0 && bmf) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)bmf);
  if (last_block(&c->blocks_done) && threadIdx.x == 0) bfs_level_end(a);
}

__global__ void __launch_bounds__(BFS_NT) bfs_pull_kernel(BfsArgs a) {
  __shared__ int64_t s_sum[BFS_NT / 32 + 1];
  if (bfs_skip(a, 1)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t level = vload(&c->level);
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen_out = &c->qlen[cur ^ 1];
  const int lane = lane_id();
  const int64_t nwords = (a.n + 31) >> 5;
  const int64_t wstride = ((int64_t)gridDim.x * BFS_NT) >> 5;
  int64_t mf = 0, insp = 0, nexp = 0;
  for (int64_t w = ((int64_t)blockIdx.x * BFS_NT + threadIdx.x) >> 5; w < nwords; w += wstride) {
    const uint32_t vw = a.vis[w];
    if (vw == FULL) continue;
    const int64_t v = (w << 5) + lane;
    const bool need = v < a.n && !((vw >> lane) & 1u);
    bool found = false;
    int32_t beg = 0, end = 0;
    if (need) {
      beg = a.co[v];
      end = a.co[v + 1];
      nexp++;
    }
    const int32_t lim = min(end, beg + PULL_SERIAL);
    for (int32_t e = beg; e < lim; e++) {
      insp++;
      if (a.label[a.ri[e]] == level) {
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
        const bool hit = e < en && a.label[a.ri[e]] == level;
        insp += e < en;
        if (__any_sync(FULL, hit)) {
          f = true;
          break;
        }
      }
      if (lane == l) found = f;
    }
    const unsigned fm = __ballot_sync(FULL, found);
    if (fm) {
      if (lane == 0) a.vis[w] = vw | fm;
      if (found) {
        a.label[v] = level + 1;
        mf += a.ro[v + 1] - a.ro[v];
      }
      warp_append(found, (int32_t)v, qout, qlen_out, a.qcap, &c->overflow);
    }
  }
  const int64_t bmf = block_sum<BFS_NT>(mf, s_sum);
  const int64_t bins = block_sum<BFS_NT>(insp, s_sum);
  const int64_t bexp = block_sum<BFS_NT>(nexp, s_sum);
  if (threadIdx.x == 0) {
    if (bmf) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)bmf);
    if (bins) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)bins);
    if (bexp) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)bexp);
  }
  if (last_block(&c->blocks_done) && threadIdx.x == 0) bfs_level_end(a);
}

// labels := -1, visited := 0.
__global__ void bfs_clear_kernel(int32_t *label, uint32_t *vis, int64_t n) {
  const int64_t nw = (n + 31) >> 5;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    label[i] = -1;
    if (i < nw) vis[i] = 0;
  }
}

// Seeds the sources (duplicates collapse) and initialises the control block.
__global__ void bfs_seed_kernel(BfsArgs a, const int32_t *srcs, int32_t nsrc, int32_t iter_cap, int32_t dir0) {
  __shared__ int64_t s_sum[1024 / 32 + 1];
  DevCtl *c = a.ctl;
  int64_t mf = 0;
  for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
    const int32_t s = srcs[i];
    const uint32_t bit = 1u << (s & 31);
    const uint32_t old = atomicOr(&a.vis[s >> 5], bit);
    if (!(old & bit)) {
      a.label[s] = 0;
      mf += a.ro[s + 1] - a.ro[s];
      int pos = atomicAdd(&c->qlen[0], 1);
      if (pos < a.qcap) a.q0[pos] = s;
      else c->overflow = 1;
    }
  }
  const int64_t t = block_sum<1024>(mf, s_sum);
  if (threadIdx.x == 0) {
    c->visited_deg = t;
    c->mf_front = t;
    c->level = 0;
    c->cur = 0;
    c->dir = dir0;
    c->iter_cap = iter_cap;
    c->done = (iter_cap <= 0 || c->overflow) ? 1 : 0;
    if (c->overflow) c->status = MG_ERR_QUEUE_OVERFLOW;
  }
}

}  // namespace mg

// Blocks of the persistent kernel: every SM's resident share (0 when the
// occupancy query fails).
static int persist_grid(mg_graph *g) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::bfs_persist_kernel, mg::BFS_NT, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return occ > 0 ? g->num_sms * std::min(occ, 4) : 0;
}

extern "C" mg_status mg_bfs(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth, const mg_opts *opts,
                            mg_stats *stats) {
  using namespace mg;
  if (!g || !srcs || nsrc <= 0 || !depth) {
    mg_set_error("mg_bfs: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  if (o.direction < MG_DIR_AUTO || o.direction > MG_DIR_PULL) {
    mg_set_error("mg_bfs: invalid direction %d", o.direction);
    return MG_ERR_ARG;
  }
  for (int32_t i = 0; i < nsrc; i++) {
    if (srcs[i] < 0 || srcs[i] >= g->n) {
      mg_set_error("mg_bfs: source %d out of range [0, %lld)", srcs[i], (long long)g->n);
      return MG_ERR_ARG;
    }
  }
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool undirected = o.directed == 0 && !symmetric;
  if (undirected && !g->has_csc) {
    mg_set_error("mg_bfs: directed=0 needs the CSC (graph created with MG_GRAPH_NO_CSC)");
    return MG_ERR_UNSUPPORTED;
  }
  MG_TRY(graph_enter(g));
  if (o.device_output) MG_TRY(check_device_ptr(g, depth, "mg_bfs", "depth"));
  const int64_t n = g->n;
  int64_t qcap64 = o.queue_sizing > 0 ? (int64_t)std::ceil(o.queue_sizing * (double)n) : n;
  qcap64 = std::max<int64_t>(1, std::min<int64_t>(qcap64, n));
  const int32_t qcap = (int32_t)qcap64;
  const int64_t nwords = (n + 31) / 32;
  const size_t need = Carve::need({sizeof(int32_t) * (size_t)n, sizeof(uint32_t) * (size_t)nwords,
                                   sizeof(int32_t) * (size_t)qcap, sizeof(int32_t) * (size_t)qcap,
                                   sizeof(int32_t) * (size_t)nsrc, sizeof(int32_t) * (size_t)BIG_CAP});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  int32_t *label_ws = cv.take<int32_t>(n);
  uint32_t *vis = cv.take<uint32_t>(nwords);
  int32_t *q0 = cv.take<int32_t>(qcap);
  int32_t *q1 = cv.take<int32_t>(qcap);
  int32_t *dsrc = cv.take<int32_t>(nsrc);
  int32_t *big_v = cv.take<int32_t>(BIG_CAP);
  int32_t *label = o.device_output ? depth : label_ws;
  cudaStream_t s = g->stream;

  BfsArgs a;
  std::memset(&a, 0, sizeof(a));  // the loop-graph signature compares its bytes
  bfs_tuning(a, g->tune);
  a.ro = g->ro;
  a.ci = g->ci;
  a.co = g->has_csc ? g->co : g->ro;
  a.ri = g->has_csc ? g->ri : g->ci;
  a.label = label;
  a.vis = vis;
  a.q0 = q0;
  a.q1 = q1;
  a.qcap = qcap;
  // AUTO on sparse graphs (mean out-degree <= 8: lattices, road networks) stays
  // top-down: a bottom-up level scans every unvisited vertex and, far from a thin
  // wavefront, finds no early exit (4096^2 lattice: 7.8 ms with Beamer's rule,
  // 6.7 ms top-down only).
  a.mode = (o.direction == MG_DIR_AUTO && g->m <= (int64_t)g->tune.bfs_sparse_degree * g->n) ? MG_DIR_PUSH
                                                                                           : o.direction;
  a.can_pull = g->has_csc && !undirected;
  a.both = undirected ? 1 : 0;
  a.n = n;
  a.m_total = g->m;
  a.big_v = big_v;
  a.ctl = g->ctl;
  a.h = 0;
  a.use_cond = 0;
  a.bar_extra = (uint32_t)debug_barrier_extra();
  a.bar_limit = a.bar_extra ? debug_barrier_limit() : PERSIST_WAIT;

  const int32_t iter_cap = o.iter_num > 0 ? (int32_t)std::min<int64_t>(o.iter_num, n + 1) : (int32_t)(n + 1);
  MG_CUDA_TRY(cudaMemcpyAsync(dsrc, srcs, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  bfs_clear_kernel<<<g->num_sms * 8, 256, 0, s>>>(label, vis, n);
  bfs_seed_kernel<<<1, 1024, 0, s>>>(a, dsrc, nsrc, iter_cap, 0);
  MG_CUDA_TRY(cudaGetLastError());
  // Small push levels first, in one persistent cooperative launch (all blocks
  // resident); a device that cannot co-schedule the grid skips it.
  const int pgrid = persist_grid(g);
  int64_t persist_launches = 0;
  if (pgrid > 0 && o.direction != MG_DIR_PULL) {
    BfsArgs pa = a;
    void *params[] = {&pa};
    if (cudaLaunchCooperativeKernel((const void *)bfs_persist_kernel, dim3(pgrid), dim3(BFS_NT), params, 0, s) ==
        cudaSuccess)
      persist_launches = 1;
    cudaGetLastError();
  }

  const int grid = g->num_sms * g->tune.bfs_ctas_per_sm;
  const bool use_graph = o.use_graph >= 0;
  struct Sig {
    BfsArgs a;
    int grid;
    int32_t tail_max, tail_edges;
  } sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.a = a;
  sig.grid = grid;
  sig.tail_max = g->tune.bfs_tail_max;
  sig.tail_edges = g->tune.bfs_tail_edges;
  // Tail levels: one CTA runs the persistent kernel at the top of every iteration
  // (its grid barrier is the CTA's own), so a run of tiny push levels (at most
  // bfs_tail_max vertices and bfs_tail_edges out-edges) costs one launch instead of
  // a launch sequence per level; on a larger frontier it returns at once and the
  // per-level kernels go on from the same control block.
  BfsArgs ta = a;
  ta.persist_max = g->tune.bfs_tail_max;
  ta.persist_edges = g->tune.bfs_tail_edges;
  const bool tail = ta.persist_max > 0 && ta.persist_edges > 0 && o.direction != MG_DIR_PULL;
  LoopBody body = [a, ta, tail, grid](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
    BfsArgs b = a;
    b.h = h;
    b.use_cond = use_cond;
    if (tail) bfs_persist_kernel<<<1, BFS_NT, 0, st>>>(ta);
    bfs_push_kernel<<<grid, BFS_NT, 0, st>>>(b);
    bfs_push_big_kernel<<<grid, BFS_NT, 0, st>>>(b);
    bfs_pull_kernel<<<grid, BFS_NT, 0, st>>>(b);
  };
  MG_TRY(run_loop(g, SLOT_BFS, &sig, sizeof(sig), use_graph, body, n + 2));
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  if (!o.device_output) MG_TRY(copy_out(g, depth, label, sizeof(int32_t) * n, 0));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = hc.visited_deg;
    stats->edges_inspected = hc.edges_inspected;
    stats->bytes_compulsory = 4 * hc.edges_inspected + 16 * hc.vertices_expanded + 4 * n +
                              (int64_t)hc.levels_pull * ((n + 7) / 8);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->status_detail = hc.levels_pull;
    const int64_t per = 3 + (tail ? 1 : 0);
    stats->launches = 2 + persist_launches + (use_graph ? (per + 1) * (int64_t)hc.body_iters : per * g->host_iters);
  }
  if (hc.status == MG_ERR_TIMEOUT) {
    mg_set_error("mg_bfs: a grid barrier of the persistent levels timed out");
    return MG_ERR_TIMEOUT;
  }
  if (hc.status != 0) {
    mg_set_error("mg_bfs: frontier exceeded queue capacity %d", qcap);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// ---- BFS over a fixed, statically allocated scratch area -------------------
// mg_bfs grows the graph's workspace on demand, which allocates device memory on
// the first call and whenever a call needs more. Some callers cannot allow that:
// a serving process that reserved its device memory up front and must not grow it
// while requests run, code called from inside a memory allocator (which must not
// re-enter the allocator), or a caller that keeps every device allocation under
// its own accounting. This variant takes its frontier queues, visited bitmap,
// source list and deferred-hub list from one file-scope device array of fixed
// size, writes depths straight into the caller's device buffer, and drives the
// level loop from the host (no executable graph is instantiated).
namespace mg {

constexpr int64_t NOALLOC_MAX_N = MG_BFS_NOALLOC_MAX_VERTICES;
constexpr int64_t NOALLOC_MAX_SRC = MG_BFS_NOALLOC_MAX_SOURCES;
constexpr size_t noalloc_round(size_t b) { return (b + 255) & ~(size_t)255; }
// Layout (bytes, each part 256-aligned): visited bitmap, two frontier queues,
// sources, deferred hubs.
constexpr size_t NOALLOC_VIS = 0;
constexpr size_t NOALLOC_Q0 = NOALLOC_VIS + noalloc_round(sizeof(uint32_t) * ((NOALLOC_MAX_N + 31) / 32));
constexpr size_t NOALLOC_Q1 = NOALLOC_Q0 + noalloc_round(sizeof(int32_t) * NOALLOC_MAX_N);
constexpr size_t NOALLOC_SRC = NOALLOC_Q1 + noalloc_round(sizeof(int32_t) * NOALLOC_MAX_N);
constexpr size_t NOALLOC_BIG = NOALLOC_SRC + noalloc_round(sizeof(int32_t) * NOALLOC_MAX_SRC);
constexpr size_t NOALLOC_BYTES = NOALLOC_BIG + noalloc_round(sizeof(int32_t) * BIG_CAP);  // 8,540,160 bytes

// Nothing in it has to start at zero: every call clears the bitmap itself and
// writes the queues, sources and hub list before reading them.
static __device__ __align__(256) uint32_t bfs_noalloc_scratch[NOALLOC_BYTES / sizeof(uint32_t)];

// Waits for a stream when it goes out of scope.
struct StreamDrain {
  cudaStream_t s;
  ~StreamDrain() { cudaStreamSynchronize(s); }
};

// Device address of the scratch array, resolved once per device (the first call
// on a device; later calls reuse the cached address).
static std::mutex noalloc_mu;
static std::vector<char *> noalloc_addr;

static mg_status noalloc_scratch_of(int device, char **out) {
  std::lock_guard<std::mutex> lk(noalloc_mu);
  if ((int)noalloc_addr.size() <= device) noalloc_addr.resize(device + 1, nullptr);
  if (!noalloc_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, bfs_noalloc_scratch);
    if (e != cudaSuccess) {
      mg_set_error("mg_bfs_noalloc: cudaGetSymbolAddress of the scratch array failed on device %d: %s", device,
                   cudaGetErrorString(e));
      return MG_ERR_CUDA;
    }
    noalloc_addr[device] = static_cast<char *>(p);
  }
  *out = noalloc_addr[device];
  return MG_OK;
}

}  // namespace mg

extern "C" mg_status mg_bfs_noalloc(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth,
                                    const mg_opts *opts, mg_stats *stats) {
  using namespace mg;
  if (!g || !srcs || nsrc <= 0 || !depth) {
    mg_set_error("mg_bfs_noalloc: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  if (g->n > NOALLOC_MAX_N) {
    mg_set_error("mg_bfs_noalloc: graph has %lld vertices, the fixed scratch holds at most %lld (use mg_bfs)",
                 (long long)g->n, (long long)NOALLOC_MAX_N);
    return MG_ERR_ARG;
  }
  if (nsrc > NOALLOC_MAX_SRC) {
    mg_set_error("mg_bfs_noalloc: %d sources, the fixed scratch holds at most %lld", nsrc,
                 (long long)NOALLOC_MAX_SRC);
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  if (o.direction < MG_DIR_AUTO || o.direction > MG_DIR_PULL) {
    mg_set_error("mg_bfs_noalloc: invalid direction %d", o.direction);
    return MG_ERR_ARG;
  }
  for (int32_t i = 0; i < nsrc; i++) {
    if (srcs[i] < 0 || srcs[i] >= g->n) {
      mg_set_error("mg_bfs_noalloc: source %d out of range [0, %lld)", srcs[i], (long long)g->n);
      return MG_ERR_ARG;
    }
  }
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool undirected = o.directed == 0 && !symmetric;
  if (undirected && !g->has_csc) {
    mg_set_error("mg_bfs_noalloc: directed=0 needs the CSC (graph created with MG_GRAPH_NO_CSC)");
    return MG_ERR_UNSUPPORTED;
  }
  MG_TRY(graph_enter(g));
  MG_TRY(check_device_ptr(g, depth, "mg_bfs_noalloc", "depth"));
  char *scratch = nullptr;
  MG_TRY(noalloc_scratch_of(g->device, &scratch));
  const int64_t n = g->n;
  int64_t qcap64 = o.queue_sizing > 0 ? (int64_t)std::ceil(o.queue_sizing * (double)n) : n;
  qcap64 = std::max<int64_t>(1, std::min<int64_t>(qcap64, n));
  const int32_t qcap = (int32_t)qcap64;
  int32_t *dsrc = reinterpret_cast<int32_t *>(scratch + NOALLOC_SRC);
  cudaStream_t s = g->stream;

  BfsArgs a;
  std::memset(&a, 0, sizeof(a));  // the loop-graph signature compares its bytes
  bfs_tuning(a, g->tune);
  a.ro = g->ro;
  a.ci = g->ci;
  a.co = g->has_csc ? g->co : g->ro;
  a.ri = g->has_csc ? g->ri : g->ci;
  a.label = depth;
  a.vis = reinterpret_cast<uint32_t *>(scratch + NOALLOC_VIS);
  a.q0 = reinterpret_cast<int32_t *>(scratch + NOALLOC_Q0);
  a.q1 = reinterpret_cast<int32_t *>(scratch + NOALLOC_Q1);
  a.qcap = qcap;
  // AUTO on sparse graphs (mean out-degree <= 8: lattices, road networks) stays
  // top-down: a bottom-up level scans every unvisited vertex and, far from a thin
  // wavefront, finds no early exit (4096^2 lattice: 7.8 ms with Beamer's rule,
  // 6.7 ms top-down only).
  a.mode = (o.direction == MG_DIR_AUTO && g->m <= (int64_t)g->tune.bfs_sparse_degree * g->n) ? MG_DIR_PUSH
                                                                                           : o.direction;
  a.can_pull = g->has_csc && !undirected;
  a.both = undirected ? 1 : 0;
  a.n = n;
  a.m_total = g->m;
  a.big_v = reinterpret_cast<int32_t *>(scratch + NOALLOC_BIG);
  a.ctl = g->ctl;
  a.h = 0;
  a.use_cond = 0;
  a.bar_extra = (uint32_t)debug_barrier_extra();
  a.bar_limit = a.bar_extra ? debug_barrier_limit() : PERSIST_WAIT;

  const int32_t iter_cap = o.iter_num > 0 ? (int32_t)std::min<int64_t>(o.iter_num, n + 1) : (int32_t)(n + 1);
  // From the first queued copy on, every return (errors included) waits for the
  // stream: the queued work uses the shared scratch array, and a caller that
  // serialises its calls must find the array idle when a call returns.
  StreamDrain drain{s};
  MG_CUDA_TRY(cudaMemcpyAsync(dsrc, srcs, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  bfs_clear_kernel<<<g->num_sms * 8, 256, 0, s>>>(depth, a.vis, n);
  bfs_seed_kernel<<<1, 1024, 0, s>>>(a, dsrc, nsrc, iter_cap, 0);
  MG_CUDA_TRY(cudaGetLastError());
  const int grid = g->num_sms * g->tune.bfs_ctas_per_sm;
  LoopBody body = [a, grid](cudaStream_t st, cudaGraphConditionalHandle, int) {
    bfs_push_kernel<<<grid, BFS_NT, 0, st>>>(a);
    bfs_push_big_kernel<<<grid, BFS_NT, 0, st>>>(a);
    bfs_pull_kernel<<<grid, BFS_NT, 0, st>>>(a);
  };
  MG_TRY(run_loop(g, SLOT_BFS, nullptr, 0, false, body, n + 2));
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = hc.visited_deg;
    stats->edges_inspected = hc.edges_inspected;
    stats->bytes_compulsory = 4 * hc.edges_inspected + 16 * hc.vertices_expanded + 4 * n +
                              (int64_t)hc.levels_pull * ((n + 7) / 8);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->status_detail = hc.levels_pull;
    stats->launches = 2 + 3 * (int64_t)hc.level;
  }
  if (hc.status != 0) {
    mg_set_error("mg_bfs_noalloc: frontier exceeded queue capacity %d", qcap);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// ---- predecessors of a BFS result ------------------------------------------
// The reference's pred_extract (Algorithms/BFS/predextract.cuh:246-373): over the
// in-edges of every vertex v, the candidate of edge (u, v) is u when
// label[v] - label[u] == 1 and -1 otherwise (gather_edge, :143-155), reduced by max
// (ReduceFunctor, :211-219). Unreached vertices get -1; a source (label 0) gets
// its largest unreached in-neighbour, as in the reference, where the comment calls
// that value arbitrary (Algorithms/BFS/bfs.cu:461). Vertices without in-edges get
// -1. Each lane takes one vertex; in-degrees above 32 are scanned by the warp.
namespace mg {

__global__ void __launch_bounds__(256) bfs_pred_kernel(const int32_t *__restrict__ co, const int32_t *__restrict__ ri,
                                                       const int32_t *__restrict__ label, int64_t n,
                                                       int32_t *__restrict__ pred) {
  const int lane = lane_id();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const int64_t v = base + threadIdx.x;
    const bool in = v < n;
    const int32_t lv = in ? label[v] : -1;
    const int32_t beg = in ? co[v] : 0, end = in ? co[v + 1] : 0;
    const bool scan = in && lv != -1;  // unreached vertices never match (label -2 does not exist)
    int32_t best = -1;
    const bool small = end - beg <= 32;
    if (scan && small)
      for (int32_t e = beg; e < end; e++) {
        const int32_t u = ri[e];
        if (lv - label[u] == 1) best = max(best, u);
      }
    unsigned pend = __ballot_sync(FULL, scan && !small);
    while (pend) {
      const int l = __ffs(pend) - 1;
      pend &= pend - 1;
      const int32_t b = __shfl_sync(FULL, beg, l), en = __shfl_sync(FULL, end, l), lbl = __shfl_sync(FULL, lv, l);
      int32_t m = -1;
      for (int32_t e = b + lane; e < en; e += 32) {
        const int32_t u = ri[e];
        if (lbl - label[u] == 1) m = max(m, u);
      }
      m = __reduce_max_sync(FULL, m);
      if (lane == l) best = m;
    }
    if (in) pred[v] = best;
  }
}

}  // namespace mg

extern "C" mg_status mg_bfs_predecessors(mg_graph *g, const int32_t *depth, int32_t *pred, const mg_opts *opts) {
  using namespace mg;
  if (!g || !depth || !pred) {
    mg_set_error("mg_bfs_predecessors: null argument");
    return MG_ERR_ARG;
  }
  const int dev_io = opts ? opts->device_output : 0;
  if (!g->has_csc) {
    mg_set_error("mg_bfs_predecessors: the gather over in-edges needs the CSC (graph created with MG_GRAPH_NO_CSC)");
    return MG_ERR_UNSUPPORTED;
  }
  MG_TRY(graph_enter(g));
  if (dev_io) {
    MG_TRY(check_device_ptr(g, depth, "mg_bfs_predecessors", "depth"));
    MG_TRY(check_device_ptr(g, pred, "mg_bfs_predecessors", "pred"));
  }
  const int64_t n = g->n;
  cudaStream_t s = g->stream;
  const int32_t *dlabel = depth;
  int32_t *dpred = pred;
  if (!dev_io) {
    MG_TRY(ws_reserve(g, g->ws_out, Carve::need({sizeof(int32_t) * (size_t)n, sizeof(int32_t) * (size_t)n})));
    Carve cv(g->ws_out.ptr);
    int32_t *l = cv.take<int32_t>(n);
    dpred = cv.take<int32_t>(n);
    MG_CUDA_TRY(cudaMemcpyAsync(l, depth, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    dlabel = l;
  }
  if (n > 0) bfs_pred_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->co, g->ri, dlabel, n, dpred);
  MG_CUDA_TRY(cudaGetLastError());
  if (!dev_io) MG_CUDA_TRY(cudaMemcpyAsync(pred, dpred, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  return MG_OK;
}
