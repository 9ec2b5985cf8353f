// pr_gather.cuh -- load-balanced gather over a CSR-shaped adjacency (rows ->
// edge lists), used by PageRank (rows = CSC columns: in-edges) and by its adjoint
// (rows = CSR rows: out-edges).
//
// Work split (merge path): the n row ends and the m edges form one sequence of
// n + m items; tile t owns items [t*IPC, (t+1)*IPC). Tile coordinates (first row,
// first edge) are precomputed once per graph.
//
// Each CTA is persistent and double-buffered: while it reduces tile k out of one
// shared-memory stage, thread 0 has already issued the TMA bulk copies
// (cp.async.bulk global->shared, completion counted on an mbarrier) of tile k+1
// into the other stage: the tile's row offsets, edge indices, edge weights, and
// up to NR per-row arrays the row update reads (previous iterate, row sums,
// teleport, ...). The ranges are widened to 16-byte boundaries (every array is
// padded for that), so the copies are legal for any tile, and no thread ever
// waits on a dependent global load in the row epilogue. Every mbarrier wait is
// bounded; a wait that runs out makes the CTA leave with a failure the caller
// reports as MG_ERR_TIMEOUT.
//
// Per-row sums are finished in three deterministic steps:
//   - inside a thread, rows that start and end in the thread are complete;
//   - a thread's first completed row adds the carries of the preceding threads
//     of the CTA that were still inside that row (in thread order);
//   - a row begun in an earlier tile is finished by the fix-up kernel, which
//     adds the carries of the preceding tiles (in tile order).
// Sums are compensated: every addend goes through TwoSum into (hi, lo), and
// weighted products through an FMA-based TwoProduct, so the result does not
// depend on how a row is split.
#pragma once

#include <climits>

#include "common.cuh"

namespace mg {

constexpr int PRG_NT = 256;
constexpr int PRG_IPT = 8;
constexpr int PRG_IPC = PRG_NT * PRG_IPT;
constexpr int PRG_STAGE = PRG_IPC + 8;  // widened to 16-byte boundaries on both sides
constexpr int PRG_MAXR = 4;             // per-row arrays a stage can carry
constexpr uint32_t PRG_WAIT_LIMIT = 1u << 24;

struct Comp {
  float hi, lo;
};

__device__ __forceinline__ void two_sum_add(Comp &c, float v) {
  const float s = c.hi + v;
  const float bp = s - c.hi;
  const float err = (c.hi - (s - bp)) + (v - bp);
  c.hi = s;
  c.lo += err;
}

__device__ __forceinline__ void comp_add(Comp &c, const Comp &d) {
  two_sum_add(c, d.hi);
  c.lo += d.lo;
}

// ---- mbarrier / bulk-copy primitives (sm_90+ PTX, single-CTA use) ----------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on phase `parity`; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < PRG_WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Merge-path split of diagonal `diag`: number of row ends among the first
// `diag` items of (row_end[0..nrows), edge ids ebase..ebase+nedges).
__device__ __forceinline__ int merge_split(const int32_t *row_end, int nrows, int32_t ebase, int nedges, int diag) {
  int lo = max(0, diag - nedges), hi = min(diag, nrows);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (row_end[mid] <= ebase + (diag - mid - 1)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

#ifndef MG_PRB_NO_PLAN_KERNELS  // plan building runs in pagerank.cu only
// Tile coordinates over the global sequence: tx[t], ty[t] for t = 0..ntiles.
__global__ void prg_plan_kernel(const int32_t *__restrict__ off, int64_t n, int64_t m, int32_t ntiles,
                                int32_t *__restrict__ tx, int32_t *__restrict__ ty) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t diag = min((int64_t)t * PRG_IPC, n + m);
    int64_t lo = max((int64_t)0, diag - m), hi = min(diag, n);
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)off[mid + 1] <= diag - mid - 1) lo = mid + 1;
      else hi = mid;
    }
    tx[t] = (int32_t)lo;
    ty[t] = (int32_t)(diag - lo);
  }
}
#endif  // MG_PRB_NO_PLAN_KERNELS

// One shared-memory stage: widened copies of the tile's offsets (raw[k] =
// off[xa + k]), edge indices (idx[k] = idx[ya + k]), weights, and per-row arrays
// (rows[j][k] = rowsrc[j][xa + k]); coord = x0, y0, x1, y1, xa.
template <bool WEIGHTED, int NR>
struct PrgStage {
  int32_t raw[PRG_STAGE];
  int32_t idx[PRG_STAGE];
  float w[WEIGHTED ? PRG_STAGE : 4];
  float rows[NR > 0 ? NR : 1][PRG_STAGE];
  int32_t coord[8];
};

template <bool WEIGHTED, int NR>
struct PrgSmem {
  PrgStage<WEIGHTED, NR> st[2];
  uint64_t bar[2];
  int32_t crow[PRG_NT];
  float chi[PRG_NT];
  float clo[PRG_NT];
  float rhi[PRG_IPC];  // per-row sums of the current tile
  float rlo[PRG_IPC];
  int32_t wfirst[PRG_NT / 32];
};

template <bool WEIGHTED, int NR>
constexpr size_t prg_smem_bytes() {
  return sizeof(PrgSmem<WEIGHTED, NR>);
}

// The adjacency a gather runs over, with its plan, carry arrays and the per-row
// arrays to stage (each padded to n + 8 entries, 16-byte aligned).
struct PrgGraph {
  const int32_t *off, *idx;
  const float *wts;
  const int32_t *tx, *ty;
  int32_t ntiles;
  int64_t n;
  int32_t *carry_row, *head_row;
  Comp *carry_val, *head_val;
  const float *rowsrc[PRG_MAXR];
};

// Issues the bulk copies of the tile with coordinates c = (x0, y0, x1, y1) into
// stage s (thread 0 only).
template <bool WEIGHTED, int NR>
__device__ __forceinline__ void prg_issue(PrgSmem<WEIGHTED, NR> &sm, int s, const PrgGraph &g, const int4 c) {
  PrgStage<WEIGHTED, NR> &st = sm.st[s];
  const int32_t x0 = c.x, y0 = c.y, x1 = c.z, y1 = c.w;
  const int32_t ya = y0 & ~3, yb = (y1 + 3) & ~3;
  const int32_t xa = x0 & ~3, xb = (x1 + 2 + 3) & ~3;
  const uint32_t bi = (uint32_t)(yb - ya) * 4u, br = (uint32_t)(xb - xa) * 4u;
  st.coord[0] = x0;
  st.coord[1] = y0;
  st.coord[2] = x1;
  st.coord[3] = y1;
  st.coord[4] = xa;
  fence_proxy_async();
  mbar_arrive_expect_tx(&sm.bar[s], br * (1 + NR) + (WEIGHTED ? 2u : 1u) * bi);
  bulk_g2s(st.raw, g.off + xa, br, &sm.bar[s]);
#pragma unroll
  for (int j = 0; j < NR; j++) bulk_g2s(st.rows[j], g.rowsrc[j] + xa, br, &sm.bar[s]);
  if (bi) {
    bulk_g2s(st.idx, g.idx + ya, bi, &sm.bar[s]);
    if (WEIGHTED) bulk_g2s(st.w, g.wts + ya, bi, &sm.bar[s]);
  }
}

__device__ __forceinline__ int4 prg_coords(const PrgGraph &g, int32_t t) {
  return make_int4(g.tx[t], g.ty[t], g.tx[t + 1], g.ty[t + 1]);
}

// Reduces one staged tile. `gather(col)` returns the neighbour's value;
// `finish(row, Comp, stage)` consumes a completed row whose per-row inputs are in
// the stage.
template <bool WEIGHTED, int NR, typename Gather, typename Finish>
__device__ __forceinline__ void prg_compute(PrgSmem<WEIGHTED, NR> &sm, const PrgStage<WEIGHTED, NR> &st,
                                            const PrgGraph &g, int32_t t, Gather &gather, Finish &finish) {
  const int tid = threadIdx.x;
  const int32_t x0 = st.coord[0], y0 = st.coord[1], x1 = st.coord[2], y1 = st.coord[3];
  const int nrows = x1 - x0, nedges = y1 - y0;
  const int32_t *rend = st.raw + (x0 & 3) + 1;  // rend[i] = off[x0 + i + 1]; past n the pad is INT_MAX
  const int32_t beg0 = st.raw[x0 & 3];          // off[x0]
  const int32_t *sidx = st.idx + (y0 & 3);
  const float *sw = st.w + (y0 & 3);
  const int total = nrows + nedges;
  const int d0 = min(tid * PRG_IPT, total);
  int lx = merge_split(rend, nrows, y0, nedges, d0);
  int ly = d0 - lx;
  // Pass 1: classify the thread's items and issue every neighbour load.
  int e_of[PRG_IPT];
  float v_hi[PRG_IPT], v_lo[PRG_IPT];
  {
    int cx = lx, cy = ly;
#pragma unroll
    for (int k = 0; k < PRG_IPT; k++) {
      e_of[k] = -2;  // past the tile
      if (d0 + k < total) {
        if (cy < nedges && y0 + cy < rend[cx]) {
          e_of[k] = cy;
          cy++;
        } else {
          e_of[k] = -1;  // row end
          cx++;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < PRG_IPT; k++) {
      v_hi[k] = 0.f;
      v_lo[k] = 0.f;
      if (e_of[k] >= 0) {
        const float gv = gather(sidx[e_of[k]]);
        if (WEIGHTED) {
          const float a = sw[e_of[k]];
          v_hi[k] = a * gv;
          v_lo[k] = __fmaf_rn(a, gv, -v_hi[k]);
        } else {
          v_hi[k] = gv;
        }
      }
    }
  }
  // Pass 2: segmented accumulation. Completed rows only record their sums in
  // shared memory; the row update runs afterwards, one row per thread.
  Comp acc{0.f, 0.f};
  bool has_first = false;
  int f_row = 0;
  Comp f_val{0.f, 0.f};
#pragma unroll
  for (int k = 0; k < PRG_IPT; k++) {
    if (e_of[k] >= 0) {
      two_sum_add(acc, v_hi[k]);
      acc.lo += v_lo[k];
    } else if (e_of[k] == -1) {
      if (!has_first) {
        has_first = true;
        f_row = lx;
        f_val = acc;
      } else {
        sm.rhi[lx] = acc.hi;
        sm.rlo[lx] = acc.lo;
      }
      acc.hi = 0.f;
      acc.lo = 0.f;
      lx++;
    }
  }
  // Segmented inclusive scan of the threads' trailing partials keyed by their
  // trailing row (non-decreasing in tid, so equal keys are contiguous): lane
  // shuffles inside each warp, then an 8-step pass across the warps.
  const int lane = tid & 31, wid = tid >> 5;
  Comp p = acc;
  const int key = lx;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float uh = __shfl_up_sync(0xffffffffu, p.hi, o), ul = __shfl_up_sync(0xffffffffu, p.lo, o);
    const int uk = __shfl_up_sync(0xffffffffu, key, o);
    if (lane >= o && uk == key) {
      Comp q{uh, ul};
      comp_add(q, p);
      p = q;
    }
  }
  if (lane == 0) sm.wfirst[wid] = key;
  if (lane == 31) {
    sm.crow[wid] = key;
    sm.chi[wid] = p.hi;
    sm.clo[wid] = p.lo;
  }
  __syncthreads();
  if (tid == 0) {
    // Warp totals become segment totals ending at each warp's last lane.
    for (int w = 1; w < PRG_NT / 32; w++) {
      if (sm.crow[w] == sm.crow[w - 1] && sm.wfirst[w] == sm.crow[w]) {
        Comp q{sm.chi[w - 1], sm.clo[w - 1]};
        comp_add(q, Comp{sm.chi[w], sm.clo[w]});
        sm.chi[w] = q.hi;
        sm.clo[w] = q.lo;
      }
    }
  }
  __syncthreads();
  if (wid > 0 && sm.crow[wid - 1] == key && sm.wfirst[wid] == key) {
    Comp q{sm.chi[wid - 1], sm.clo[wid - 1]};
    comp_add(q, p);
    p = q;
  }
  // p = sum of the run of trailing partials ending at this thread.
  const Comp carry_in = Comp{__shfl_up_sync(0xffffffffu, p.hi, 1), __shfl_up_sync(0xffffffffu, p.lo, 1)};
  const int key_prev = __shfl_up_sync(0xffffffffu, key, 1);
  __syncthreads();
  sm.crow[tid] = key;
  sm.chi[tid] = p.hi;
  sm.clo[tid] = p.lo;
  __syncthreads();
  // A row begun in an earlier tile is finished by the fix-up kernel.
  const bool defer0 = y0 > beg0;
  if (has_first) {
    Comp tot{0.f, 0.f};
    if (tid > 0) {
      const bool cont = lane > 0 ? key_prev == f_row : sm.crow[tid - 1] == f_row;
      if (cont) tot = lane > 0 ? carry_in : Comp{sm.chi[tid - 1], sm.clo[tid - 1]};
    }
    comp_add(tot, f_val);
    if (f_row == 0 && defer0) {
      g.head_row[t] = x0;
      g.head_val[t] = tot;
    } else {
      sm.rhi[f_row] = tot.hi;
      sm.rlo[f_row] = tot.lo;
    }
  }
  if (tid == PRG_NT - 1) {
    g.carry_row[t] = x0 + key;
    g.carry_val[t] = p;
  }
  __syncthreads();
  // Row updates: consecutive threads on consecutive rows (coalesced stores, no
  // divergence from the item walk).
  for (int j = (defer0 ? 1 : 0) + tid; j < nrows; j += PRG_NT) finish(x0 + j, Comp{sm.rhi[j], sm.rlo[j]}, st);
}

// Persistent double-buffered loop over tiles blockIdx.x, +gridDim.x, ...
// Returns false if a bounded wait ran out.
template <bool WEIGHTED, int NR, typename Gather, typename Finish>
__device__ __forceinline__ bool prg_run(PrgSmem<WEIGHTED, NR> &sm, const PrgGraph &g, Gather &&gather,
                                        Finish &&finish) {
  // Thread 0 keeps the coordinates of the next tile to issue in registers,
  // loaded one iteration ahead so the issue never waits on a global load.
  int4 cnext = make_int4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    mbar_init(&sm.bar[0], 1);
    mbar_init(&sm.bar[1], 1);
    fence_barrier_init();
    if ((int32_t)blockIdx.x < g.ntiles) prg_issue<WEIGHTED, NR>(sm, 0, g, prg_coords(g, blockIdx.x));
    if ((int32_t)(blockIdx.x + gridDim.x) < g.ntiles) cnext = prg_coords(g, blockIdx.x + gridDim.x);
  }
  __syncthreads();
  uint32_t phase[2] = {0u, 0u};
  int k = 0;
  for (int32_t t = blockIdx.x; t < g.ntiles; t += gridDim.x, k++) {
    const int s = k & 1;
    const int32_t tn = t + gridDim.x;
    if (threadIdx.x == 0 && tn < g.ntiles) {
      prg_issue<WEIGHTED, NR>(sm, s ^ 1, g, cnext);
      if (tn + (int32_t)gridDim.x < g.ntiles) cnext = prg_coords(g, tn + gridDim.x);
    }
    const bool ok = mbar_wait_bounded(&sm.bar[s], phase[s]);
    if (__syncthreads_or(!ok)) {
      // Give the copy in flight for the next tile a bounded chance to land.
      if (tn < g.ntiles) mbar_wait_bounded(&sm.bar[s ^ 1], phase[s ^ 1]);
      return false;
    }
    phase[s] ^= 1u;
    prg_compute<WEIGHTED, NR>(sm, sm.st[s], g, t, gather, finish);
    __syncthreads();
  }
  return true;
}

// Cross-tile fix-up of the row begun before tile t (if any): adds the carries of
// the preceding tiles that ended inside that row, in tile order.
template <typename Finish>
__device__ __forceinline__ void prg_fixup_tile(int32_t t, const int32_t *__restrict__ carry_row,
                                               const Comp *__restrict__ carry_val, int32_t *__restrict__ head_row,
                                               const Comp *__restrict__ head_val, Finish &&finish) {
  const int32_t r = head_row[t];
  if (r < 0) return;
  int32_t t0 = t;
  while (t0 > 0 && carry_row[t0 - 1] == r) t0--;
  Comp tot{0.f, 0.f};
  for (int32_t q = t0; q < t; q++) comp_add(tot, carry_val[q]);
  comp_add(tot, head_val[t]);
  head_row[t] = -1;
  finish(r, tot);
}

}  // namespace mg
