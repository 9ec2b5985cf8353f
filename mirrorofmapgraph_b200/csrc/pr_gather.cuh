// pr_gather.cuh -- load-balanced gather over a CSR-shaped adjacency (rows ->
// edge lists), used by PageRank (rows = CSC columns: in-edges) and by its adjoint
// (rows = CSR rows: out-edges).
//
// Work split (merge path): the n row ends and the m edges form one sequence of
// n + m items; tile t owns items [t*IPC, (t+1)*IPC). Tile coordinates (first row,
// first edge) are precomputed once per graph. A tile stages its row ends and its
// edge indices (and weights) in shared memory, each thread consumes IPT items,
// and per-row sums are finished in three deterministic steps:
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

struct PrgShared {
  int32_t row_end[PRG_IPC + 1];
  int32_t idx[PRG_IPC];
  float w[PRG_IPC];
  int32_t crow[PRG_NT];
  float chi[PRG_NT];
  float clo[PRG_NT];
  int32_t beg0;
};

// One tile. `val(j)` returns the gathered value of local edge j (the neighbour's
// value, times the edge weight when weighted, as an exact hi/lo pair through
// `prod`). `finish(row, Comp)` consumes a completed row; rows begun in an earlier
// tile are written to the head arrays instead.
template <bool WEIGHTED, typename Gather, typename Finish>
__device__ __forceinline__ void prg_tile(PrgShared &sm, const int32_t *__restrict__ off,
                                         const int32_t *__restrict__ idx, const float *__restrict__ wts, int64_t n,
                                         int32_t t, int32_t x0, int32_t y0, int32_t x1, int32_t y1,
                                         int32_t *__restrict__ carry_row, Comp *__restrict__ carry_val,
                                         int32_t *__restrict__ head_row, Comp *__restrict__ head_val,
                                         Gather &&gather, Finish &&finish) {
  const int tid = threadIdx.x;
  const int nrows = x1 - x0, nedges = y1 - y0;
  for (int i = tid; i < nrows; i += PRG_NT) sm.row_end[i] = off[x0 + i + 1];
  if (tid == 0) {
    sm.row_end[nrows] = (x1 < n) ? off[x1 + 1] : INT_MAX;
    sm.beg0 = off[x0];
  }
  for (int j = tid; j < nedges; j += PRG_NT) {
    sm.idx[j] = idx[y0 + j];
    if (WEIGHTED) sm.w[j] = wts[y0 + j];
  }
  __syncthreads();
  const int total = nrows + nedges;
  const int d0 = min(tid * PRG_IPT, total);
  int lx = merge_split(sm.row_end, nrows, y0, nedges, d0);
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
        if (cy < nedges && y0 + cy < sm.row_end[cx]) {
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
        const float g = gather(sm.idx[e_of[k]]);
        if (WEIGHTED) {
          const float a = sm.w[e_of[k]];
          v_hi[k] = a * g;
          v_lo[k] = __fmaf_rn(a, g, -v_hi[k]);
        } else {
          v_hi[k] = g;
        }
      }
    }
  }
  // Pass 2: segmented accumulation.
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
        finish(x0 + lx, acc);
      }
      acc.hi = 0.f;
      acc.lo = 0.f;
      lx++;
    }
  }
  sm.crow[tid] = lx;
  sm.chi[tid] = acc.hi;
  sm.clo[tid] = acc.lo;
  __syncthreads();
  if (has_first) {
    int t0 = tid;
    while (t0 > 0 && sm.crow[t0 - 1] == f_row) t0--;
    Comp tot{0.f, 0.f};
    for (int q = t0; q < tid; q++) comp_add(tot, Comp{sm.chi[q], sm.clo[q]});
    comp_add(tot, f_val);
    if (f_row == 0 && y0 > sm.beg0) {
      head_row[t] = x0;
      head_val[t] = tot;
    } else {
      finish(x0 + f_row, tot);
    }
  }
  if (tid == PRG_NT - 1) {
    const int r = sm.crow[PRG_NT - 1];
    int t0 = PRG_NT - 1;
    while (t0 > 0 && sm.crow[t0 - 1] == r) t0--;
    Comp tot{0.f, 0.f};
    for (int q = t0; q < PRG_NT; q++) comp_add(tot, Comp{sm.chi[q], sm.clo[q]});
    carry_row[t] = x0 + r;
    carry_val[t] = tot;
  }
  __syncthreads();
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
