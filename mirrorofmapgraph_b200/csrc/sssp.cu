// sssp.cu -- single-source shortest paths (struct sssp, Algorithms/SSSP/sssp.h:33-409).
//
// The reference runs a push Bellman-Ford in five phases per iteration: apply
// (min of dist and gathered candidate), post-apply (commit, reset gather_tmp),
// expand (emit neighbour + candidate distance for every improving edge into an
// edge-sized queue), contract (atomicMin into gather_tmp, cull duplicates)
// (sssp.h:242-402, GASengine/enactor_vertex_centric.cuh:2561-2822).
//
// Here one kernel per iteration does all of it: each frontier vertex's edges are
// expanded with the degree-binned tile expansion; an improving edge lowers
// dist[u] directly with atomicMin, and the thread whose atomicMin won the
// improvement claims u's bit in the next frontier's bitmap and appends it with a
// warp-aggregated atomic. No edge-sized queue exists and duplicates never enter
// the frontier. Distances are unique fixed points, so the result equals the
// reference's bit for bit for any schedule.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"

namespace mg {

constexpr int SSSP_NT = 256;
constexpr int SSSP_CH = 256;  // edges per chunk of a heavy frontier vertex
constexpr int SSSP_U = 4;     // edge slots of 32 a warp holds in flight
constexpr int SSSP_WS = 128;  // next-frontier stage per warp (shared memory)

struct SsspArgs {
  const int32_t *ro, *ci, *w;   // CSR with weights (w == nullptr: unit weights)
  const int32_t *co, *ri, *cw;  // CSC with permuted weights (directed == 0 only)
  int32_t *dist;
  uint32_t *inq0, *inq1;        // next-frontier dedup bitmaps (ping-pong)
  int32_t *q0, *q1;
  int32_t qcap;
  int32_t both;
  int64_t n;
  int2 *chunks;      // {item, first edge | 1 << 31 for a CSC edge} of the heavy vertices' chunks
  int32_t chunk_cap;
  int32_t heavy;        // out-degree from which a frontier vertex is cut into chunks
  int32_t heavy_small;  // the same for a frontier of fewer vertices than the grid has lanes
  int32_t vmask;   // item -> vertex mask: -1 for one instance; batched runs keep the
                   // instance number in the bits above it (item = instance << s | v)
  int32_t delta;   // near-far bucket width (0: plain frontier Bellman-Ford)
  int32_t *far0, *far1;  // far piles (ping-pong)
  uint32_t *infar;       // bit per item: in the current far pile
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

// Per-warp staging of next-frontier appends in shared memory: one global atomic
// per SSSP_WS items instead of one per warp-wide append (a round of R-MAT s22 adds
// two million vertices to one queue).
struct WarpStage {
  int32_t *buf;
  int32_t n;  // entries held (the same in every lane)
};

// Every lane of the warp calls it.
__device__ __forceinline__ void ws_flush(WarpStage &st, int32_t *queue, int32_t *len, int32_t cap,
                                         int32_t *overflow) {
  __syncwarp();
  if (st.n == 0) return;
  int32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(len, st.n);
  base = __shfl_sync(FULL, base, 0);
  for (int32_t i = lane_id(); i < st.n; i += 32) {
    const int32_t pos = base + i;
    if (pos < cap) queue[pos] = st.buf[i];
    else *overflow = 1;
  }
  __syncwarp();
  st.n = 0;
}

// Appends item where pred; every lane of the warp calls it.
__device__ __forceinline__ void ws_push(WarpStage &st, bool pred, int32_t item, int32_t *queue, int32_t *len,
                                        int32_t cap, int32_t *overflow) {
  const unsigned pm = __ballot_sync(FULL, pred);
  if (pm == 0) return;
  const int32_t cnt = __popc(pm);
  if (st.n + cnt > SSSP_WS) ws_flush(st, queue, len, cap, overflow);
  if (pred) st.buf[st.n + __popc(pm & lanemask_lt())] = item;
  st.n += cnt;
}

struct RelaxCtx {
  int32_t *dist;
  uint32_t *inq_next;
  const int32_t *ro;
  int32_t *qout, *qlen_out, *overflow;
  int32_t qcap;
  int32_t vmask;
  int64_t updates;
  // near-far: improvements to a distance >= thr go to the far pile instead
  int32_t delta;
  int64_t thr;
  uint32_t *infar;
  int32_t *far_out, *far_len_out;
};

// Relaxes SSSP_U edges per lane: edge r goes to item u[r] (-1: none) with weight
// w[r] from a vertex at distance dv[r]. The loads, the atomicMins and the bitmap
// claims of the SSSP_U edges are each issued together, so a lane waits for one
// memory round trip per step rather than per edge. Every lane of the warp calls it.
__device__ __forceinline__ void relax_group(RelaxCtx &x, WarpStage &st, const int32_t (&u)[SSSP_U],
                                            const int32_t (&w)[SSSP_U], const int32_t (&dv)[SSSP_U]) {
  int32_t cd[SSSP_U], nd[SSSP_U], old[SSSP_U];
  bool tr[SSSP_U];
#pragma unroll
  for (int r = 0; r < SSSP_U; r++) cd[r] = u[r] >= 0 ? __ldcg(x.dist + u[r]) : INT_MIN;
#pragma unroll
  for (int r = 0; r < SSSP_U; r++) {
    const int64_t s = (int64_t)dv[r] + (int64_t)w[r];
    tr[r] = u[r] >= 0 && s < (int64_t)cd[r];
    nd[r] = (int32_t)min(s, (int64_t)INT_MAX);
  }
  if (x.delta <= 0) {
    // Plain rounds: an edge that improves on the distance read before the
    // atomicMin marks its head in the next-frontier bitmap, and neither atomic's
    // old value is waited for (the frontier is compacted from the bitmap after the
    // round). A mark from an improvement that a concurrent smaller one overtook
    // only expands that vertex once more.
#pragma unroll
    for (int r = 0; r < SSSP_U; r++) {
      if (tr[r]) {
        red_min(x.dist + u[r], nd[r]);
        red_or(x.inq_next + (u[r] >> 5), 1u << (u[r] & 31));
        x.updates++;
      }
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < SSSP_U; r++) old[r] = tr[r] ? atomicMin(x.dist + u[r], nd[r]) : INT_MIN;
  uint32_t ob[SSSP_U];
  bool nearq[SSSP_U];
#pragma unroll
  for (int r = 0; r < SSSP_U; r++) {
    const bool win = tr[r] && nd[r] < old[r];
    nearq[r] = (int64_t)nd[r] < x.thr;
    ob[r] = 0xffffffffu;  // no claim: reads as "already queued"
    if (win) ob[r] = atomicOr((nearq[r] ? x.inq_next : x.infar) + (u[r] >> 5), 1u << (u[r] & 31));
  }
#pragma unroll
  for (int r = 0; r < SSSP_U; r++) {
    if (tr[r] && nd[r] < old[r]) x.updates++;
    const bool fresh = u[r] >= 0 && !(ob[r] & (1u << (u[r] & 31)));
    ws_push(st, fresh && nearq[r], u[r], x.qout, x.qlen_out, x.qcap, x.overflow);
    warp_append(fresh && !nearq[r], u[r], x.far_out, x.far_len_out, x.qcap, x.overflow);
  }
}

__device__ __forceinline__ RelaxCtx relax_ctx(const SsspArgs &a, DevCtl *c, int cur) {
  const int fc = a.delta > 0 ? vload(&c->far_cur) : 0;
  return RelaxCtx{a.dist, (cur || a.delta <= 0) ? a.inq0 : a.inq1, a.ro, cur ? a.q0 : a.q1, &c->qlen[cur ^ 1],
                  &c->overflow, a.qcap,
                  a.vmask, 0, a.delta, vload(&c->thr), a.infar, fc ? a.far1 : a.far0, &c->far_len[fc]};
}

// The edges of the warp's 32 vertices (lane l brings vertex item v, its distance
// dv, its first edge beg and deg edges), concatenated and walked 32 x SSSP_U at a
// time: edge slot j belongs to the last lane whose exclusive degree prefix is <= j
// (binary search over the lanes' prefixes by shuffles).
__device__ __forceinline__ void warp_walk(RelaxCtx &x, WarpStage &st, int32_t v, int32_t dv, int32_t beg,
                                          int32_t deg, const int32_t *__restrict__ adj,
                                          const int32_t *__restrict__ wt, int32_t hi) {
  const int lane = lane_id();
  const int32_t inc = warp_inclusive_scan(deg);
  const int32_t tot = __shfl_sync(FULL, inc, 31);
  const int32_t ex = inc - deg;
  const int32_t kb = beg - ex;  // edge index of slot j of this lane's vertex: kb + j
  for (int32_t b0 = 0; b0 < tot; b0 += 32 * SSSP_U) {
    int32_t u[SSSP_U], w[SSSP_U], d[SSSP_U];
#pragma unroll
    for (int r = 0; r < SSSP_U; r++) {
      const int32_t j = b0 + r * 32 + lane;
      int l = 0;
#pragma unroll
      for (int sft = 16; sft > 0; sft >>= 1)
        if (__shfl_sync(FULL, ex, l + sft) <= j) l += sft;
      const int32_t k = __shfl_sync(FULL, kb, l) + j;
      const int32_t sv = __shfl_sync(FULL, v, l);
      d[r] = __shfl_sync(FULL, dv, l);
      const bool ok = j < tot;
      u[r] = ok ? ((sv & hi) | adj[k]) : -1;
      w[r] = ok ? (wt ? wt[k] : 1) : 0;
    }
    relax_group(x, st, u, w, d);
  }
}

// Cuts the lanes' vertices of at least `th` edges into chunks of SSSP_CH edges and
// appends them to the chunk list ({item, first edge | flag}); returns the number
// of edges this lane still has to walk itself (0 when chunked). A warp whose chunks
// do not fit walks all its vertices (the slots it took are marked empty).
__device__ __forceinline__ int32_t warp_chunks(const SsspArgs &a, int32_t *clen, int32_t v, int32_t beg,
                                               int32_t deg, int32_t th, int32_t flag) {
  const int lane = lane_id();
  const int32_t nch = (v >= 0 && deg >= th) ? (deg + SSSP_CH - 1) / SSSP_CH : 0;
  const int32_t inc = warp_inclusive_scan(nch);
  const int32_t tot = __shfl_sync(FULL, inc, 31);
  if (tot == 0) return deg;
  int32_t base = 0;
  if (lane == 0) base = atomicAdd(clen, tot);
  base = __shfl_sync(FULL, base, 0);
  const int32_t ex = inc - nch;
  if (base + tot > a.chunk_cap) {
    for (int32_t j = base + lane; j < a.chunk_cap; j += 32) a.chunks[j] = make_int2(-1, 0);
    return deg;
  }
  for (int32_t j0 = 0; j0 < tot; j0 += 32) {
    const int32_t j = j0 + lane;
    int l = 0;
#pragma unroll
    for (int sft = 16; sft > 0; sft >>= 1)
      if (__shfl_sync(FULL, ex, l + sft) <= j) l += sft;
    const int32_t sv = __shfl_sync(FULL, v, l);
    const int32_t sb = __shfl_sync(FULL, beg, l);
    const int32_t se = __shfl_sync(FULL, ex, l);
    if (j < tot) a.chunks[base + j] = make_int2(sv, (sb + (j - se) * SSSP_CH) | flag);
  }
  return nch ? 0 : deg;
}

__device__ void sssp_level_end(const SsspArgs &a) {
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nf = vload(&c->qlen[cur ^ 1]);
  const int lvl = vload(&c->level) + 1;
  trace_level(c, lvl - 1, MG_DIR_PUSH, vload(&c->qlen[cur]), vload(&c->mf_next), 0.0);
  c->mf_next = 0;
  c->level = lvl;
  c->qlen[cur] = 0;
  c->cur = cur ^ 1;
  c->blocks_done = 0;
  c->big_len = 0;
  c->tile_next = 0;
  const bool over = vload(&c->overflow) != 0;
  // near-far: an empty near frontier with vertices waiting in the far pile is a
  // split (the far kernels refill the near frontier), not the end
  const int32_t nfar = a.delta > 0 ? vload(&c->far_len[vload(&c->far_cur)]) : 0;
  const bool split = nf == 0 && nfar > 0 && !over;
  const bool done = (nf == 0 && !split) || lvl >= c->iter_cap || over;
  c->split = (split && !done) ? 1 : 0;
  if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
  __threadfence();
  c->done = done ? 1 : 0;
  if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
}

// Adds a block's counters to the control block.
__device__ __forceinline__ void sssp_counters(DevCtl *c, int64_t *s_sum, int64_t reach, int64_t insp, int64_t nexp,
                                              int64_t upd) {
  const int64_t b0 = block_sum<SSSP_NT>(reach, s_sum);
  const int64_t b1 = block_sum<SSSP_NT>(insp, s_sum);
  const int64_t b2 = block_sum<SSSP_NT>(nexp, s_sum);
  const int64_t b3 = block_sum<SSSP_NT>(upd, s_sum);
  if (threadIdx.x == 0) {
    if (b0) atomicAdd((unsigned long long *)&c->mf_next, (unsigned long long)b0);
    if (b1) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)b1);
    if (b2) atomicAdd((unsigned long long *)&c->vertices_expanded, (unsigned long long)b2);
    if (b3) atomicAdd((unsigned long long *)&c->vertices_updated, (unsigned long long)b3);
  }
}

// Relaxation round, pass 1: each warp takes 32 frontier items, cuts the heavy ones
// into chunks for pass 2 and walks the edges of the others itself.
__global__ void __launch_bounds__(SSSP_NT, 4) sssp_relax_kernel(SsspArgs a) {
  __shared__ int32_t s_stage[SSSP_NT / 32][SSSP_WS];
  __shared__ int64_t s_sum[SSSP_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  uint32_t *inq_cur = cur ? a.inq1 : a.inq0;
  RelaxCtx x = relax_ctx(a, c, cur);
  WarpStage st{s_stage[warp_id()], 0};
  const int32_t hi = ~a.vmask;  // instance bits of an item
  const int64_t nw = (int64_t)gridDim.x * (SSSP_NT / 32);
  const int64_t gw = (int64_t)blockIdx.x * (SSSP_NT / 32) + warp_id();
  // A frontier of fewer vertices than the grid has lanes leaves most warps without
  // a vertex of their own: hand every vertex of heavy_small edges or more to pass 2.
  const int32_t th = (int64_t)nin < nw * 32 ? a.heavy_small : a.heavy;
  int64_t insp = 0, nexp = 0;
  for (int64_t base = gw * 32; base < nin; base += nw * 32) {
    const int64_t i = base + lane_id();
    const int32_t v = i < nin ? qin[i] : -1;
    int32_t beg = 0, deg = 0, dv = 0, cb = 0, cdeg = 0;
    if (v >= 0) {
      // Near-far rounds: the whole bitmap of the current frontier is cleared here,
      // one word at a time (nothing sets bits in it during this round). Plain
      // rounds have one bitmap, cleared by the compaction.
      if (a.delta > 0) inq_cur[v >> 5] = 0u;
      nexp++;
      beg = a.ro[v & a.vmask];
      deg = a.ro[(v & a.vmask) + 1] - beg;
      dv = vload(a.dist + v);
      if (a.both) {
        cb = a.co[v & a.vmask];
        cdeg = a.co[(v & a.vmask) + 1] - cb;
      }
      insp += deg + cdeg;
    }
    deg = warp_chunks(a, &c->big_len, v, beg, deg, th, 0);
    warp_walk(x, st, v, dv, beg, deg, a.ci, a.w, hi);
    if (a.both) {
      cdeg = warp_chunks(a, &c->big_len, v, cb, cdeg, th, INT_MIN);
      warp_walk(x, st, v, dv, cb, cdeg, a.ri, a.cw, hi);
    }
  }
  ws_flush(st, x.qout, x.qlen_out, x.qcap, x.overflow);
  // the round's frontier out-edges (its inspected edges) go to the trace record
  sssp_counters(c, s_sum, insp, insp, nexp, x.updates);
}

// Pass 2: every warp of the grid relaxes chunks of the heavy vertices' edges; the
// last CTA closes the round.
__global__ void __launch_bounds__(SSSP_NT, 4) sssp_chunk_kernel(SsspArgs a) {
  __shared__ int32_t s_stage[SSSP_NT / 32][SSSP_WS];
  __shared__ int64_t s_sum[SSSP_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  RelaxCtx x = relax_ctx(a, c, cur);
  WarpStage st{s_stage[warp_id()], 0};
  const int32_t hi = ~a.vmask;
  const int lane = lane_id();
  const int32_t nch = min(vload(&c->big_len), a.chunk_cap);
  const int32_t nw = gridDim.x * (SSSP_NT / 32);
  for (int32_t ch = blockIdx.x * (SSSP_NT / 32) + warp_id(); ch < nch; ch += nw) {
    const int2 e = a.chunks[ch];
    if (e.x < 0) continue;
    const bool rev = e.y < 0;
    const int32_t k0 = e.y & INT_MAX;
    const int32_t *off = rev ? a.co : a.ro;
    const int32_t *adj = rev ? a.ri : a.ci;
    const int32_t *wt = rev ? a.cw : a.w;
    const int32_t end = min(k0 + SSSP_CH, off[(e.x & a.vmask) + 1]);
    const int32_t dv = vload(a.dist + e.x);
    const int32_t base = e.x & hi;
    for (int32_t b = k0; b < end; b += 32 * SSSP_U) {
      int32_t u[SSSP_U], w[SSSP_U], d[SSSP_U];
#pragma unroll
      for (int r = 0; r < SSSP_U; r++) {
        const int32_t k = b + r * 32 + lane;
        const bool ok = k < end;
        u[r] = ok ? (base | adj[k]) : -1;
        w[r] = ok ? (wt ? wt[k] : 1) : 0;
        d[r] = dv;
      }
      relax_group(x, st, u, w, d);
    }
  }
  ws_flush(st, x.qout, x.qlen_out, x.qcap, x.overflow);
  sssp_counters(c, s_sum, 0, 0, 0, x.updates);
  if (a.delta > 0 && last_block(&c->blocks_done) && threadIdx.x == 0) sssp_level_end(a);
}

// Plain rounds, pass 3: the next frontier, compacted in item order from the
// bitmap the round marked (one word per thread, one queue atomic per CTA), the
// words cleared for the next round; the last CTA ends the round. Near-far rounds
// append to the queue as they relax and end in pass 2.
__global__ void __launch_bounds__(SSSP_NT) sssp_compact_kernel(SsspArgs a) {
  __shared__ int32_t s_red[SSSP_NT / 32 + 1];
  __shared__ int32_t s_base;
  DevCtl *c = a.ctl;
  if (a.delta > 0 || vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0 && vload(&c->done)) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen = &c->qlen[cur ^ 1];
  uint32_t *bm = a.inq0;
  const int64_t nwords = (a.n + 31) >> 5;
  for (int64_t t0 = (int64_t)blockIdx.x * SSSP_NT; t0 < nwords; t0 += (int64_t)gridDim.x * SSSP_NT) {
    const int64_t w = t0 + threadIdx.x;
    uint32_t m = 0u;
    if (w < nwords) {
      m = bm[w];
      if (m) bm[w] = 0u;
    }
    int32_t tot;
    int32_t pos = block_exclusive_scan<SSSP_NT>((int32_t)__popc(m), s_red, &tot);
    if (threadIdx.x == 0) s_base = tot ? atomicAdd(qlen, tot) : 0;
    __syncthreads();
    pos += s_base;
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      if (pos < a.qcap) qout[pos] = (int32_t)(w * 32 + b);
      else c->overflow = 1;
      pos++;
    }
    __syncthreads();
  }
  if (last_block(&c->blocks_done) && threadIdx.x == 0) sssp_level_end(a);
}

// The TEPS numerator of a run: out-degrees of every reached item's vertex.
__global__ void sssp_reach_kernel(const int32_t *__restrict__ dist, int64_t nitems, int32_t vmask,
                                  const int32_t *__restrict__ ro, DevCtl *c) {
  __shared__ int64_t s_sum[256 / 32 + 1];
  int64_t t = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nitems; i += (int64_t)gridDim.x * blockDim.x)
    if (dist[i] != INT_MAX) t += ro[(i & vmask) + 1] - ro[i & vmask];
  const int64_t b = block_sum<256>(t, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd((unsigned long long *)&c->visited_deg, (unsigned long long)b);
}

// Near-far split, pass 1: the smallest distance still waiting at or above the
// threshold (entries below it are stale: their vertex was improved into the near
// frontier since).
__global__ void __launch_bounds__(SSSP_NT) sssp_far_min_kernel(SsspArgs a) {
  DevCtl *c = a.ctl;
  if (vload(&c->done) || !vload(&c->split)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0 && vload(&c->done)) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int fc = vload(&c->far_cur);
  const int32_t len = min(vload(&c->far_len[fc]), a.qcap);
  const int32_t *far = fc ? a.far1 : a.far0;
  const int64_t thr = vload(&c->thr);
  int32_t mn = INT_MAX;
  for (int32_t i = blockIdx.x * SSSP_NT + threadIdx.x; i < len; i += gridDim.x * SSSP_NT) {
    const int32_t d = vload(a.dist + far[i]);
    if ((int64_t)d >= thr) mn = min(mn, d);
  }
  mn = __reduce_min_sync(FULL, mn);
  if (lane_id() == 0 && mn != INT_MAX) atomicMin(&c->far_min, mn);
}

// Pass 2: new threshold max(thr, far_min) + delta; waiting vertices below it
// join the near frontier, the rest move to the other far pile, stale entries are
// dropped. The last CTA switches the piles.
__global__ void __launch_bounds__(SSSP_NT) sssp_far_split_kernel(SsspArgs a) {
  DevCtl *c = a.ctl;
  if (vload(&c->done) || !vload(&c->split)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0 && vload(&c->done)) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const int fc = vload(&c->far_cur);
  const int32_t len = min(vload(&c->far_len[fc]), a.qcap);
  const int32_t *far = fc ? a.far1 : a.far0;
  int32_t *far_keep = fc ? a.far0 : a.far1;
  const int64_t thr = vload(&c->thr);
  const int32_t fmin = vload(&c->far_min);
  const int64_t thr_new = (fmin == INT_MAX ? thr : max(thr, (int64_t)fmin)) + a.delta;
  int32_t *qnear = cur ? a.q1 : a.q0;
  uint32_t *inq_near = cur ? a.inq1 : a.inq0;
  const int32_t ntile = (len + SSSP_NT - 1) / SSSP_NT;
  for (int32_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int32_t i = t * SSSP_NT + threadIdx.x;
    bool to_near = false, keep = false;
    int32_t u = 0;
    if (i < len) {
      u = far[i];
      const int64_t d = vload(a.dist + u);
      const uint32_t bit = 1u << (u & 31);
      if (d < thr_new) {
        atomicAnd(a.infar + (u >> 5), ~bit);
        if (d >= thr) to_near = !(atomicOr(inq_near + (u >> 5), bit) & bit);
      } else {
        keep = true;
      }
    }
    warp_append(to_near, u, qnear, &c->qlen[cur], a.qcap, &c->overflow);
    warp_append(keep, u, far_keep, &c->far_len[fc ^ 1], a.qcap, &c->overflow);
  }
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->blocks_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  c->blocks_done = 0;
  c->thr = thr_new;
  c->far_len[fc] = 0;
  c->far_cur = fc ^ 1;
  c->far_min = INT_MAX;
  c->splits += 1;
  const bool over = vload(&c->overflow) != 0;
  const int32_t nn = vload(&c->qlen[cur]);
  const int32_t nk = vload(&c->far_len[fc ^ 1]);
  // Nothing moved but vertices still wait: split again at the next pass.
  c->split = (nn == 0 && nk > 0 && !over) ? 1 : 0;
  const bool done = (nn == 0 && nk == 0) || over;
  if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
  __threadfence();
  c->done = done ? 1 : 0;
  if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
}

__global__ void sssp_clear_kernel(int32_t *dist, uint32_t *b0, uint32_t *b1, uint32_t *b2, int64_t n) {
  const int64_t nw = (n + 31) >> 5;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dist[i] = INT_MAX;
    if (i < nw) {
      b0[i] = 0;
      b1[i] = 0;
      if (b2) b2[i] = 0;
    }
  }
}

__global__ void sssp_seed_kernel(SsspArgs a, const int32_t *srcs, int32_t nsrc, int32_t iter_cap) {
  DevCtl *c = a.ctl;
  for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
    const int32_t s = srcs[i];
    const uint32_t bit = 1u << (s & 31);
    // duplicates: near-far rounds clear this bitmap as they expand the seeds; plain
    // rounds mark the next frontier in inq0 and leave inq1 to the seeds
    if (!(atomicOr(&(a.delta > 0 ? a.inq0 : a.inq1)[s >> 5], bit) & bit)) {
      a.dist[s] = 0;
      const int pos = atomicAdd(&c->qlen[0], 1);
      if (pos < a.qcap) a.q0[pos] = s;
      else c->overflow = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    c->iter_cap = iter_cap;
    c->thr = a.delta > 0 ? (int64_t)a.delta : INT64_MAX;
    c->far_min = INT_MAX;
    c->done = c->overflow ? 1 : 0;
    if (c->overflow) c->status = MG_ERR_QUEUE_OVERFLOW;
  }
}

// Minimum and sum of the int32 edge weights (out[0] min, out[1..2] the sum as
// an unsigned 64-bit count of non-negative values).
__global__ void min_i32_kernel(const int32_t *__restrict__ v, int64_t m, int *__restrict__ out) {
  int mn = INT_MAX;
  unsigned long long sum = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    mn = min(mn, v[i]);
    sum += v[i] > 0 ? (unsigned long long)v[i] : 0ull;
  }
  mn = __reduce_min_sync(FULL, mn);
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
  if (lane_id() == 0) {
    if (mn != INT_MAX) atomicMin(out, mn);
    if (sum) atomicAdd(reinterpret_cast<unsigned long long *>(out + 2), sum);
  }
}

// ---- Batched SSSP with interleaved distances -------------------------------
// Up to 32 instances form a group: a vertex's 32 distances are one 128-byte row
// (lane i of a warp holds instance i), and a 32-bit mask per row says which
// instances improved the vertex in the last round. Frontier items are
// (group, vertex) pairs, item = group << shift | vertex. A warp takes an item and
// walks its edges once for every instance of the group: the instances active at
// the item load their distance to the edge's head from one row, lower it with
// atomicMin, and the warp ORs the ballot of the winners into the head's next mask;
// the OR that finds the mask empty queues the head. Heavy items are cut into
// chunks (carrying the mask) that every warp of the grid takes.
constexpr int MSS_CH = 128;  // edges per chunk of a heavy item
constexpr int MSS_U = 8;     // edges a warp holds in flight

struct MssArgs {
  const int32_t *ro, *ci, *w;   // CSR (w == nullptr: unit weights)
  const int32_t *co, *ri, *cw;  // CSC (directed == 0 on an asymmetric graph)
  int32_t *D;                   // rows of 32 distances, row (g, v) at g * n + v
  uint32_t *m0, *m1;            // active-instance masks per row (ping-pong)
  int32_t *q0, *q1;
  int32_t qcap;
  int4 *chunks;                 // {item, first edge | 1 << 31 for a CSC edge, mask, 0}
  int32_t chunk_cap;
  int32_t heavy;
  int64_t n;
  int32_t shift, vmask;
  int32_t both;
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

// Relaxes edges [k0, k1) of adj/wt from the vertex whose row this lane's instance
// reads as dv (act: the lane's instance improved that vertex last round). An edge
// that improves on the distance read before the atomicMin sets the instance's bit
// in the head's next mask; neither atomic's old value is waited for (the frontier
// is compacted from the masks after the round), so a warp keeps one memory round
// trip per MSS_U edges. A bit set by an improvement that a concurrent smaller one
// overtook only re-expands that vertex once more.
//
// The edges are staged MSS_CH at a time in the warp's shared buffer `se` as
// (head, weight) pairs, read back two per 16-byte broadcast load; slots past the
// end hold (0, INT_MAX), an edge that can never improve a distance. Inactive lanes
// compare against 0. Every lane of the warp calls it with the same edge range.
__device__ __forceinline__ void mss_edges(const MssArgs &a, int2 *se, uint32_t *mnext, int64_t gbase, bool act,
                                          int32_t dv, const int32_t *__restrict__ adj,
                                          const int32_t *__restrict__ wt, int32_t k0, int32_t k1, int64_t &updates) {
  const int lane = lane_id();
  int32_t *Dl = a.D + (gbase << 5) + lane;  // this lane's column of the group's rows
  uint32_t *mg = mnext + gbase;
  for (int32_t b = k0; b < k1; b += MSS_CH) {
    const int32_t cnt = min(MSS_CH, k1 - b);
#pragma unroll
    for (int q = 0; q < MSS_CH / 32; q++) {
      const int32_t j = q * 32 + lane;
      se[j] = j < cnt ? make_int2(adj[b + j], wt ? wt[b + j] : 1) : make_int2(0, INT_MAX);
    }
    __syncwarp();
    for (int32_t e0 = 0; e0 < cnt; e0 += MSS_U) {
      int32_t u[MSS_U], w[MSS_U], cu[MSS_U];
#pragma unroll
      for (int r = 0; r < MSS_U; r += 2) {
        const int4 p = *reinterpret_cast<const int4 *>(se + e0 + r);
        u[r] = p.x;
        w[r] = p.y;
        u[r + 1] = p.z;
        w[r + 1] = p.w;
      }
#pragma unroll
      for (int r = 0; r < MSS_U; r++) cu[r] = act ? __ldcg(Dl + ((uint32_t)u[r] << 5)) : 0;
      uint32_t myb = 0;
      int32_t myv = 0;
#pragma unroll
      for (int r = 0; r < MSS_U; r++) {
        const int32_t nd = (int32_t)min((uint32_t)dv + (uint32_t)w[r], (uint32_t)INT_MAX);
        const bool tr = nd < cu[r];
        if (tr) red_min(Dl + ((uint32_t)u[r] << 5), nd);
        const uint32_t bits = __ballot_sync(FULL, tr);
        if (lane == r) {
          myb = bits;
          myv = u[r];
        }
      }
      if (myb) {
        updates += __popc(myb);
        red_or(mg + myv, myb);
      }
    }
    __syncwarp();
  }
}

__device__ void mss_level_end(const MssArgs &a) {
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const int32_t nf = vload(&c->qlen[cur ^ 1]);
  const int lvl = vload(&c->level) + 1;
  trace_level(c, lvl - 1, MG_DIR_PUSH, vload(&c->qlen[cur]), 0, 0.0);
  c->level = lvl;
  c->qlen[cur] = 0;
  c->cur = cur ^ 1;
  c->blocks_done = 0;
  c->big_len = 0;
  const bool over = vload(&c->overflow) != 0;
  const bool done = nf == 0 || lvl >= c->iter_cap || over;
  if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
  __threadfence();
  c->done = done ? 1 : 0;
  if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
}

// Pass 1: each warp reads 32 frontier items' headers (one per lane), cuts the
// heavy ones into chunks and walks the others item by item.
__global__ void __launch_bounds__(SSSP_NT, 4) mss_relax_kernel(MssArgs a) {
  __shared__ __align__(16) int2 s_edges[SSSP_NT / 32][MSS_CH + MSS_U];
  __shared__ int64_t s_sum[SSSP_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  uint32_t *mcur = cur ? a.m1 : a.m0, *mnext = cur ? a.m0 : a.m1;
  const int lane = lane_id();
  const int64_t nw = (int64_t)gridDim.x * (SSSP_NT / 32);
  int64_t insp = 0, nexp = 0, upd = 0;
  for (int64_t base = ((int64_t)blockIdx.x * (SSSP_NT / 32) + warp_id()) * 32; base < nin; base += nw * 32) {
    const int64_t i = base + lane;
    const int32_t it = i < nin ? qin[i] : -1;
    int64_t row = 0;
    uint32_t mask = 0;
    int32_t beg = 0, deg = 0, cb = 0, cdeg = 0;
    if (it >= 0) {
      const int32_t v = it & a.vmask;
      row = (int64_t)(it >> a.shift) * a.n + v;
      mask = mcur[row];
      mcur[row] = 0u;  // this array collects the round after next; nothing else writes it now
      beg = a.ro[v];
      deg = a.ro[v + 1] - beg;
      if (a.both) {
        cb = a.co[v];
        cdeg = a.co[v + 1] - cb;
      }
      insp += deg + cdeg;
      nexp++;
    }
    // heavy items: chunks for pass 2, forward then reverse edges
    for (int dir = 0; dir < (a.both ? 2 : 1); dir++) {
      const int32_t db = dir ? cb : beg, dd = dir ? cdeg : deg;
      const int32_t nch = (it >= 0 && dd >= a.heavy) ? (dd + MSS_CH - 1) / MSS_CH : 0;
      const int32_t inc = warp_inclusive_scan(nch);
      const int32_t tot = __shfl_sync(FULL, inc, 31);
      if (tot == 0) continue;
      int32_t cbase = 0;
      if (lane == 0) cbase = atomicAdd(&c->big_len, tot);
      cbase = __shfl_sync(FULL, cbase, 0);
      if (cbase + tot > a.chunk_cap) {  // no room: this warp walks its heavy items itself
        for (int32_t j = cbase + lane; j < a.chunk_cap; j += 32) a.chunks[j] = make_int4(-1, 0, 0, 0);
        continue;
      }
      const int32_t ex = inc - nch;
      for (int32_t j0 = 0; j0 < tot; j0 += 32) {
        const int32_t j = j0 + lane;
        int l = 0;
#pragma unroll
        for (int sft = 16; sft > 0; sft >>= 1)
          if (__shfl_sync(FULL, ex, l + sft) <= j) l += sft;
        const int32_t sit = __shfl_sync(FULL, it, l);
        const int32_t sb = __shfl_sync(FULL, db, l);
        const int32_t se = __shfl_sync(FULL, ex, l);
        const uint32_t sm = __shfl_sync(FULL, mask, l);
        if (j < tot) a.chunks[cbase + j] = make_int4(sit, (sb + (j - se) * MSS_CH) | (dir ? INT_MIN : 0), (int)sm, 0);
      }
      if (nch) {
        if (dir) cdeg = 0;
        else deg = 0;
      }
    }
    // light items, one at a time by the whole warp
    unsigned todo = __ballot_sync(FULL, deg + cdeg > 0);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const int32_t sit = __shfl_sync(FULL, it, j);
      const int64_t srow = __shfl_sync(FULL, row, j);
      const uint32_t sm = __shfl_sync(FULL, mask, j);
      const int64_t gbase = (int64_t)(sit >> a.shift) * a.n;
      const bool act = (sm >> lane) & 1u;
      const int32_t dv = act ? __ldcg(a.D + (srow << 5) + lane) : INT_MAX;
      const int32_t sb = __shfl_sync(FULL, beg, j), sd = __shfl_sync(FULL, deg, j);
      int2 *se = s_edges[warp_id()];
      if (sd) mss_edges(a, se, mnext, gbase, act, dv, a.ci, a.w, sb, sb + sd, upd);
      if (a.both) {
        const int32_t scb = __shfl_sync(FULL, cb, j), scd = __shfl_sync(FULL, cdeg, j);
        if (scd) mss_edges(a, se, mnext, gbase, act, dv, a.ri, a.cw, scb, scb + scd, upd);
      }
    }
  }
  sssp_counters(c, s_sum, 0, insp, nexp, upd);
}

// Pass 2: chunks of the heavy items, a warp per chunk.
__global__ void __launch_bounds__(SSSP_NT, 4) mss_chunk_kernel(MssArgs a) {
  __shared__ __align__(16) int2 s_edges[SSSP_NT / 32][MSS_CH + MSS_U];
  __shared__ int64_t s_sum[SSSP_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  uint32_t *mnext = cur ? a.m0 : a.m1;
  const int lane = lane_id();
  int64_t upd = 0;
  const int32_t nch = min(vload(&c->big_len), a.chunk_cap);
  const int32_t nw = gridDim.x * (SSSP_NT / 32);
  for (int32_t ch = blockIdx.x * (SSSP_NT / 32) + warp_id(); ch < nch; ch += nw) {
    const int4 e = a.chunks[ch];
    if (e.x < 0) continue;
    const bool rev = e.y < 0;
    const int32_t k0 = e.y & INT_MAX;
    const int32_t v = e.x & a.vmask;
    const int64_t gbase = (int64_t)(e.x >> a.shift) * a.n;
    const int32_t *off = rev ? a.co : a.ro;
    const int32_t end = min(k0 + MSS_CH, off[v + 1]);
    const bool act = ((uint32_t)e.z >> lane) & 1u;
    const int32_t dv = act ? __ldcg(a.D + ((gbase + v) << 5) + lane) : INT_MAX;
    mss_edges(a, s_edges[warp_id()], mnext, gbase, act, dv, rev ? a.ri : a.ci, rev ? a.cw : a.w, k0, end, upd);
  }
  sssp_counters(c, s_sum, 0, 0, 0, upd);
}

// Pass 3: the next frontier, compacted in row order from the masks the round set
// (rows of MSS_CT consecutive masks per tile, one queue atomic per tile); the last
// CTA ends the round.
constexpr int MSS_CT = SSSP_NT * 4;
__global__ void __launch_bounds__(SSSP_NT) mss_compact_kernel(MssArgs a, int64_t rows) {
  __shared__ int32_t s_red[SSSP_NT / 32 + 1];
  __shared__ int32_t s_base;
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const uint32_t *mnext = cur ? a.m0 : a.m1;
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen = &c->qlen[cur ^ 1];
  for (int64_t t0 = (int64_t)blockIdx.x * MSS_CT; t0 < rows; t0 += (int64_t)gridDim.x * MSS_CT) {
    const int64_t r0 = t0 + (int64_t)threadIdx.x * 4;
    uint32_t mk[4] = {0u, 0u, 0u, 0u};
    if (r0 + 3 < rows) {
      const uint4 q = *reinterpret_cast<const uint4 *>(mnext + r0);
      mk[0] = q.x;
      mk[1] = q.y;
      mk[2] = q.z;
      mk[3] = q.w;
    } else {
      for (int k = 0; k < 4; k++)
        if (r0 + k < rows) mk[k] = mnext[r0 + k];
    }
    const int32_t cnt = (mk[0] != 0u) + (mk[1] != 0u) + (mk[2] != 0u) + (mk[3] != 0u);
    int32_t tot;
    int32_t ex = block_exclusive_scan<SSSP_NT>(cnt, s_red, &tot);
    if (threadIdx.x == 0) s_base = tot ? atomicAdd(qlen, tot) : 0;
    __syncthreads();
    ex += s_base;
    for (int k = 0; k < 4; k++) {
      if (mk[k] == 0u) continue;
      const int64_t row = r0 + k;
      const int32_t g = (int32_t)(row / a.n);
      const int32_t v = (int32_t)(row - (int64_t)g * a.n);
      if (ex < a.qcap) qout[ex] = (g << a.shift) | v;
      else c->overflow = 1;
      ex++;
    }
    __syncthreads();
  }
  if (last_block(&c->blocks_done) && threadIdx.x == 0) mss_level_end(a);
}

// Rows := INT_MAX, masks := 0.
__global__ void mss_clear_kernel(MssArgs a, int64_t rows) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows * 32; i += stride) {
    a.D[i] = INT_MAX;
    if (i < rows) {
      a.m0[i] = 0u;
      a.m1[i] = 0u;
    }
  }
}

// Instance i (group i / 32, lane i % 32) starts at srcs[i]; items of equal
// (group, vertex) share a queue entry.
__global__ void mss_seed_kernel(MssArgs a, const int32_t *srcs, int32_t nsrc, int32_t iter_cap) {
  DevCtl *c = a.ctl;
  for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
    const int32_t s = srcs[i];
    const int32_t g = i >> 5;
    const int64_t row = (int64_t)g * a.n + s;
    a.D[(row << 5) + (i & 31)] = 0;
    if (atomicOr(a.m0 + row, 1u << (i & 31)) == 0u) {
      const int pos = atomicAdd(&c->qlen[0], 1);
      if (pos < a.qcap) a.q0[pos] = (g << a.shift) | s;
      else c->overflow = 1;
    }
  }
  if (threadIdx.x == 0) {
    c->iter_cap = iter_cap;
    c->done = c->overflow ? 1 : 0;
    if (c->overflow) c->status = MG_ERR_QUEUE_OVERFLOW;
  }
}

// Rows -> nsrc x n distance rows (a 32 x 32 transpose per block of 32 vertices
// and one group), and the TEPS numerator: out-degrees of every instance's reached
// vertices.
__global__ void __launch_bounds__(1024) mss_unpack_kernel(MssArgs a, int32_t *dist, int32_t nsrc, int32_t groups) {
  __shared__ int32_t t[32][33];
  __shared__ int64_t s_sum[1024 / 32 + 1];
  const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
  const int64_t vtiles = (a.n + 31) >> 5;
  int64_t reach = 0;
  for (int64_t tile = blockIdx.x; tile < vtiles * groups; tile += gridDim.x) {
    const int32_t g = (int32_t)(tile / vtiles);
    const int64_t v0 = (tile % vtiles) << 5;
    const int64_t v = v0 + wy;
    __syncthreads();
    t[wy][lane] = v < a.n ? a.D[(((int64_t)g * a.n + v) << 5) + lane] : INT_MAX;
    __syncthreads();
    // thread (wy, lane): instance g * 32 + wy, vertex v0 + lane
    const int32_t inst = g * 32 + wy;
    const int64_t vv = v0 + lane;
    if (inst < nsrc && vv < a.n) {
      const int32_t d = t[lane][wy];
      dist[(int64_t)inst * a.n + vv] = d;
      if (d != INT_MAX) reach += a.ro[vv + 1] - a.ro[vv];
    }
  }
  const int64_t b = block_sum<1024>(reach, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd((unsigned long long *)&a.ctl->visited_deg, (unsigned long long)b);
}

}  // namespace mg

// Checks once per graph that int32 weights are non-negative (cached).
static mg_status check_weights_nonnegative(mg_graph *g) {
  if (g->vtype != MG_DTYPE_I32 || g->m == 0 || g->weights_checked) return MG_OK;
  int *d = reinterpret_cast<int *>(reinterpret_cast<char *>(g->ctl) + sizeof(DevCtl));
  int h[4] = {INT_MAX, 0, 0, 0};
  MG_CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
  mg::min_i32_kernel<<<g->num_sms * 4, 256, 0, g->stream>>>((const int32_t *)g->vals, g->m, d);
  MG_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  unsigned long long sum = 0;
  std::memcpy(&sum, h + 2, sizeof(sum));
  g->weights_checked = true;
  g->min_weight = h[0];
  g->mean_weight = (double)sum / (double)g->m;
  return MG_OK;
}

// Checks what every SSSP call needs from the graph and the options.
static mg_status sssp_check(mg_graph *g, const int32_t *srcs, int32_t nsrc, const mg_opts &o, const char *who) {
  for (int32_t i = 0; i < nsrc; i++) {
    if (srcs[i] < 0 || srcs[i] >= g->n) {
      mg_set_error("%s: source %d out of range [0, %lld)", who, srcs[i], (long long)g->n);
      return MG_ERR_ARG;
    }
  }
  if (g->vtype == MG_DTYPE_F32) {
    mg_set_error("%s: float edge values are not supported (int32 distances)", who);
    return MG_ERR_UNSUPPORTED;
  }
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  if (o.directed == 0 && !symmetric && !g->has_csc) {
    mg_set_error("%s: directed=0 needs the CSC", who);
    return MG_ERR_UNSUPPORTED;
  }
  MG_TRY(check_weights_nonnegative(g));
  if (g->vtype == MG_DTYPE_I32 && g->min_weight < 0) {
    mg_set_error("%s: negative edge weight %d", who, g->min_weight);
    return MG_ERR_ARG;
  }
  return MG_OK;
}

// Runs SSSP over `nitems` frontier items into `dist` (device, nitems entries),
// seeded from the items `seeds`. One instance: items are vertices (vmask -1).
// Batched: item = instance << s | vertex with vmask = 2^s - 1, so every instance
// relaxes its own copy of the distances over the shared CSR.
static mg_status sssp_core(mg_graph *g, const int32_t *seeds, int32_t nseed, int32_t *dist, int64_t nitems,
                           int32_t vmask, const mg_opts &o, mg_stats *stats) {
  using namespace mg;
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool both = o.directed == 0 && !symmetric;
  const int64_t n = g->n;
  int64_t qcap64 = o.queue_sizing > 0 ? (int64_t)std::ceil(o.queue_sizing * (double)nitems) : nitems;
  const int32_t qcap = (int32_t)std::max<int64_t>(1, std::min<int64_t>(qcap64, nitems));
  const int64_t nwords = (nitems + 31) / 32;
  // Schedule. Near-far with bucket width delta when asked for (delta > 0), or by
  // default on sparse graphs (mean out-degree <= 8, e.g. lattices), where plain
  // frontier Bellman-Ford re-relaxes every edge many times over its long paths:
  // there delta = 8 x the mean weight. Plain Bellman-Ford on denser graphs (R-MAT:
  // fewer, wider rounds win) and whenever an iteration cap is set (the cap counts
  // the reference's relaxation rounds) or delta < 0.
  int32_t delta = -1;
  if (o.iter_num <= 0 && g->vtype == MG_DTYPE_I32) {
    if (o.delta > 0) {
      delta = o.delta;
    } else if (o.delta == 0 && n > 0 && (double)g->m <= 8.0 * (double)n) {
      delta = (int32_t)std::max(1.0, std::min(1e9, std::round(8.0 * g->mean_weight)));
    }
  }
  const size_t far_items = delta > 0 ? (size_t)qcap : 0;
  // Chunk list: a round's heavy vertices hold at most (edges / SSSP_CH + vertices of
  // heavy_small edges or more) chunks; each instance's frontier holds a vertex once,
  // so its edges are at most m per direction. Past the capacity a warp walks its
  // heavy vertices itself.
  const mg_tuning &tn = g->tune;
  const int32_t heavy = std::max(1, tn.sssp_heavy);
  const int32_t heavy_small = std::max(1, std::min(tn.sssp_heavy_small, heavy));
  const double inst = (double)nitems / (double)std::max<int64_t>(1, n);
  const double dirs = both ? 2.0 : 1.0;
  const double cbound = inst * dirs * (double)g->m * (1.0 / SSSP_CH + 1.0 / heavy) + 65536.0;
  const int32_t chunk_cap = (int32_t)std::max(
      1.0, std::min(cbound, tn.sssp_chunk_cap > 0 ? (double)tn.sssp_chunk_cap : (double)(1 << 23)));
  const size_t need = Carve::need({sizeof(uint32_t) * (size_t)nwords, sizeof(uint32_t) * (size_t)nwords,
                                   sizeof(int32_t) * (size_t)qcap, sizeof(int32_t) * (size_t)qcap,
                                   sizeof(int32_t) * (size_t)nseed, sizeof(int2) * (size_t)chunk_cap,
                                   sizeof(int32_t) * far_items, sizeof(int32_t) * far_items,
                                   sizeof(uint32_t) * (delta > 0 ? (size_t)nwords : 0)});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  SsspArgs a;
  std::memset(&a, 0, sizeof(a));  // the loop-graph signature compares its bytes
  a.inq0 = cv.take<uint32_t>(nwords);
  a.inq1 = cv.take<uint32_t>(nwords);
  a.q0 = cv.take<int32_t>(qcap);
  a.q1 = cv.take<int32_t>(qcap);
  int32_t *dsrc = cv.take<int32_t>(nseed);
  a.chunks = cv.take<int2>(chunk_cap);
  a.chunk_cap = chunk_cap;
  a.heavy = heavy;
  a.heavy_small = heavy_small;
  a.delta = delta > 0 ? delta : 0;
  a.far0 = delta > 0 ? cv.take<int32_t>(far_items) : nullptr;
  a.far1 = delta > 0 ? cv.take<int32_t>(far_items) : nullptr;
  a.infar = delta > 0 ? cv.take<uint32_t>(nwords) : nullptr;
  a.ro = g->ro;
  a.ci = g->ci;
  a.w = g->vtype == MG_DTYPE_I32 ? (const int32_t *)g->vals : nullptr;
  a.co = g->has_csc ? g->co : g->ro;
  a.ri = g->has_csc ? g->ri : g->ci;
  a.cw = g->vtype == MG_DTYPE_I32 ? (const int32_t *)(g->has_csc ? g->cvals : g->vals) : nullptr;
  a.dist = dist;
  a.qcap = qcap;
  a.both = both ? 1 : 0;
  a.n = nitems;
  a.vmask = vmask;
  a.ctl = g->ctl;
  a.h = 0;
  a.use_cond = 0;
  cudaStream_t s = g->stream;
  // Bellman-Ford rounds of every instance are bounded by its vertex count; the
  // near-far schedule adds rounds that find nothing new (a bucket's last round),
  // so its bound is looser.
  const int64_t rounds = delta > 0 ? std::min<int64_t>(4 * n + 64, INT_MAX - 64) : n + 1;
  const int32_t iter_cap = o.iter_num > 0 ? (int32_t)std::min<int64_t>(o.iter_num, n + 1) : (int32_t)rounds;
  MG_CUDA_TRY(cudaMemcpyAsync(dsrc, seeds, sizeof(int32_t) * nseed, cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  sssp_clear_kernel<<<g->num_sms * 8, 256, 0, s>>>(dist, a.inq0, a.inq1, a.infar, nitems);
  sssp_seed_kernel<<<1, 1024, 0, s>>>(a, dsrc, nseed, iter_cap);
  MG_CUDA_TRY(cudaGetLastError());
  const int grid = g->num_sms * std::max(1, std::min(tn.sssp_ctas_per_sm, 8));
  struct Sig {
    SsspArgs a;
    int grid;
  } sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.a = a;
  sig.grid = grid;
  const int64_t nwords_all = (nitems + 31) / 32;
  const int cgrid =
      (int)std::max<int64_t>(1, std::min<int64_t>((nwords_all + SSSP_NT - 1) / SSSP_NT, g->num_sms * 8));
  LoopBody body = [a, grid, cgrid](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
    SsspArgs b = a;
    b.h = h;
    b.use_cond = use_cond;
    sssp_relax_kernel<<<grid, SSSP_NT, 0, st>>>(b);
    sssp_chunk_kernel<<<grid, SSSP_NT, 0, st>>>(b);
    if (b.delta <= 0) sssp_compact_kernel<<<cgrid, SSSP_NT, 0, st>>>(b);
    if (b.delta > 0) {
      sssp_far_min_kernel<<<grid, SSSP_NT, 0, st>>>(b);
      sssp_far_split_kernel<<<grid, SSSP_NT, 0, st>>>(b);
    }
  };
  MG_TRY(run_loop(g, vmask == -1 ? SLOT_SSSP : SLOT_BSSSP, &sig, sizeof(sig), o.use_graph >= 0, body,
                  (int64_t)iter_cap + 2));
  sssp_reach_kernel<<<g->num_sms * 4, 256, 0, s>>>(dist, nitems, vmask, g->ro, g->ctl);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = hc.visited_deg;
    stats->edges_inspected = hc.edges_inspected;
    stats->bytes_compulsory = (a.w ? 8 : 4) * hc.edges_inspected + 16 * hc.vertices_expanded + 8 * hc.vertices_updated;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    const int64_t per = a.delta > 0 ? 4 : 3;
    stats->launches = 3 + (o.use_graph >= 0 ? (per + 1) * (int64_t)hc.body_iters : per * (int64_t)hc.level);
    stats->status_detail = a.delta > 0 ? a.delta : 0;
  }
  if (hc.status != 0) {
    mg_set_error("mg_sssp: device status %d (queue capacity %d)", hc.status, qcap);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// Runs a (multi-source) SSSP into `dist` (device, n entries).
static mg_status sssp_run(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist, const mg_opts &o,
                          mg_stats *stats) {
  MG_TRY(sssp_check(g, srcs, nsrc, o, "mg_sssp"));
  return sssp_core(g, srcs, nsrc, dist, g->n, -1, o, stats);
}

extern "C" mg_status mg_sssp(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist, const mg_opts *opts,
                             mg_stats *stats) {
  if (!g || !srcs || nsrc <= 0 || !dist) {
    mg_set_error("mg_sssp: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  MG_TRY(graph_enter(g));
  if (o.device_output) MG_TRY(check_device_ptr(g, dist, "mg_sssp", "dist"));
  int32_t *out = dist;
  if (!o.device_output) {
    MG_TRY(ws_reserve(g, g->ws_out, sizeof(int32_t) * (size_t)g->n + 256));
    out = (int32_t *)g->ws_out.ptr;
  }
  MG_TRY(sssp_run(g, srcs, nsrc, out, o, stats));
  if (!o.device_output) {
    MG_TRY(copy_out(g, dist, out, sizeof(int32_t) * g->n, 0));
    MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  return MG_OK;
}

// Batched plain Bellman-Ford over interleaved distance rows (mss_* kernels) into
// `dist` (device, nsrc x n).
static mg_status msssp_run(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist, const mg_opts &o,
                           mg_stats *stats) {
  using namespace mg;
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  const bool both = o.directed == 0 && !symmetric;
  const int64_t n = g->n;
  const int32_t groups = (nsrc + 31) / 32;
  int shift = 0;
  while ((int64_t(1) << shift) < n) shift++;
  if ((int64_t)groups << shift > (int64_t)INT_MAX + 1) {
    mg_set_error("mg_sssp_batch: %d groups of 32 sources over %lld vertices exceed 2^31 frontier items; split the "
                 "sources", groups, (long long)n);
    return MG_ERR_ARG;
  }
  const int64_t rows = (int64_t)groups * n;
  const mg_tuning &tn = g->tune;
  const int32_t heavy = std::max(1, tn.sssp_batch_heavy);
  const double cbound = groups * (both ? 2.0 : 1.0) * (double)g->m * (1.0 / MSS_CH + 1.0 / heavy) + 65536.0;
  const int32_t chunk_cap = (int32_t)std::max(
      1.0, std::min(cbound, tn.sssp_chunk_cap > 0 ? (double)tn.sssp_chunk_cap : (double)(1 << 23)));
  const size_t need = Carve::need({sizeof(int32_t) * 32 * (size_t)rows, sizeof(uint32_t) * (size_t)rows,
                                   sizeof(uint32_t) * (size_t)rows, sizeof(int32_t) * (size_t)rows,
                                   sizeof(int32_t) * (size_t)rows, sizeof(int4) * (size_t)chunk_cap,
                                   sizeof(int32_t) * (size_t)nsrc});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  MssArgs a;
  std::memset(&a, 0, sizeof(a));  // the loop-graph signature compares its bytes
  a.D = cv.take<int32_t>(32 * (size_t)rows);
  a.m0 = cv.take<uint32_t>(rows);
  a.m1 = cv.take<uint32_t>(rows);
  a.q0 = cv.take<int32_t>(rows);
  a.q1 = cv.take<int32_t>(rows);
  a.chunks = cv.take<int4>(chunk_cap);
  int32_t *dsrc = cv.take<int32_t>(nsrc);
  a.qcap = (int32_t)std::min<int64_t>(rows, INT_MAX);
  a.chunk_cap = chunk_cap;
  a.heavy = heavy;
  a.ro = g->ro;
  a.ci = g->ci;
  a.w = g->vtype == MG_DTYPE_I32 ? (const int32_t *)g->vals : nullptr;
  a.co = g->has_csc ? g->co : g->ro;
  a.ri = g->has_csc ? g->ri : g->ci;
  a.cw = g->vtype == MG_DTYPE_I32 ? (const int32_t *)(g->has_csc ? g->cvals : g->vals) : nullptr;
  a.n = n;
  a.shift = shift;
  a.vmask = (int32_t)((int64_t(1) << shift) - 1);
  a.both = both ? 1 : 0;
  a.ctl = g->ctl;
  cudaStream_t s = g->stream;
  MG_CUDA_TRY(cudaMemcpyAsync(dsrc, srcs, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  mss_clear_kernel<<<g->num_sms * 8, 256, 0, s>>>(a, rows);
  mss_seed_kernel<<<1, 1024, 0, s>>>(a, dsrc, nsrc, (int32_t)std::min<int64_t>(n + 1, INT_MAX));
  MG_CUDA_TRY(cudaGetLastError());
  const int grid = g->num_sms * std::max(1, std::min(tn.sssp_ctas_per_sm, 8));
  struct Sig {
    MssArgs a;
    int grid;
  } sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.a = a;
  sig.grid = grid;
  const int cgrid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + MSS_CT - 1) / MSS_CT, g->num_sms * 8));
  LoopBody body = [a, grid, cgrid, rows](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
    MssArgs b = a;
    b.h = h;
    b.use_cond = use_cond;
    mss_relax_kernel<<<grid, SSSP_NT, 0, st>>>(b);
    mss_chunk_kernel<<<grid, SSSP_NT, 0, st>>>(b);
    mss_compact_kernel<<<cgrid, SSSP_NT, 0, st>>>(b, rows);
  };
  MG_TRY(run_loop(g, SLOT_MSSSP, &sig, sizeof(sig), o.use_graph >= 0, body, n + 3));
  mss_unpack_kernel<<<g->num_sms * 2, 1024, 0, s>>>(a, dist, nsrc, groups);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = hc.visited_deg;
    stats->edges_inspected = hc.edges_inspected;
    // per inspected edge: its index and weight, one row read; per expanded item:
    // its mask and offsets; the rows written back once
    stats->bytes_compulsory = (a.w ? 8 : 4) * hc.edges_inspected + 16 * hc.vertices_expanded +
                              128 * hc.vertices_expanded + 4 * (int64_t)nsrc * n;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->launches = 3 + (o.use_graph >= 0 ? 4 * (int64_t)hc.body_iters : 3 * (int64_t)hc.level);
  }
  if (hc.status != 0) {
    mg_set_error("mg_sssp_batch: device status %d", hc.status);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// nsrc independent single-source runs in one device run (no reference
// counterpart; the reference loops the engine per source,
// Algorithms/BFS/bfs.cu:442-456). Instance i relaxes items i << s | v, with
// 2^s >= n; the distance rows are then packed to nsrc x n.
extern "C" mg_status mg_sssp_batch(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist,
                                   const mg_opts *opts, mg_stats *stats) {
  if (!g || !srcs || nsrc <= 0 || !dist) {
    mg_set_error("mg_sssp_batch: null argument or nsrc <= 0");
    return MG_ERR_ARG;
  }
  mg_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  MG_TRY(graph_enter(g));
  if (o.device_output) MG_TRY(check_device_ptr(g, dist, "mg_sssp_batch", "dist"));
  MG_TRY(sssp_check(g, srcs, nsrc, o, "mg_sssp_batch"));
  const int64_t n = g->n;
  // Plain unbounded rounds on graphs where a single run would take them too (mean
  // out-degree above 8, or delta < 0): interleaved distance rows, one edge read for
  // up to 32 instances. Near-far and capped runs: one item per instance and vertex.
  const bool interleaved = o.iter_num <= 0 && n > 0 && (o.delta < 0 || (o.delta == 0 && g->m > 8 * n));
  if (interleaved) {
    int32_t *out = dist;
    if (!o.device_output) {
      MG_TRY(ws_reserve(g, g->ws_out, sizeof(int32_t) * (size_t)nsrc * (size_t)n + 256));
      out = (int32_t *)g->ws_out.ptr;
    }
    MG_TRY(msssp_run(g, srcs, nsrc, out, o, stats));
    if (!o.device_output) {
      MG_TRY(copy_out(g, dist, out, sizeof(int32_t) * (size_t)nsrc * (size_t)n, 0));
      MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    return MG_OK;
  }
  int shift = 0;
  while ((int64_t(1) << shift) < n) shift++;
  const int64_t stride = int64_t(1) << shift;
  if (n == 0 || (int64_t)nsrc * stride > (int64_t)INT_MAX) {
    mg_set_error("mg_sssp_batch: %d instances of %lld (padded to %lld) vertices exceed 2^31 frontier items; "
                 "split the sources", nsrc, (long long)n, (long long)stride);
    return MG_ERR_ARG;
  }
  const int64_t nitems = (int64_t)nsrc * stride;
  std::vector<int32_t> seeds(nsrc);
  for (int32_t i = 0; i < nsrc; i++) seeds[i] = (int32_t)(((int64_t)i << shift) | srcs[i]);
  // Distances are computed into a padded buffer unless the rows are already dense
  // and the output is on the device.
  const bool direct = stride == n && o.device_output;
  int32_t *work = dist;
  if (!direct) {
    MG_TRY(ws_reserve(g, g->ws_out, sizeof(int32_t) * (size_t)nitems + 256));
    work = (int32_t *)g->ws_out.ptr;
  }
  MG_TRY(sssp_core(g, seeds.data(), nsrc, work, nitems, (int32_t)(stride - 1), o, stats));
  if (!direct) {
    MG_CUDA_TRY(cudaMemcpy2DAsync(dist, sizeof(int32_t) * n, work, sizeof(int32_t) * stride, sizeof(int32_t) * n,
                                  nsrc, o.device_output ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  g->stream));
    MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  return MG_OK;
}
