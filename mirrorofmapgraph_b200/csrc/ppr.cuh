// ppr.cuh -- batched personalised PageRank: up to 256 teleport vectors solved
// together (no reference counterpart; the reference runs one uniform PageRank
// per engine run, Algorithms/PageRank/PageRank.h:33-409).
//
// Layout: every per-vertex array holds the W = 32 * VPL vectors of a group side
// by side (vertex-major, n x W floats), so one gather of a neighbour's row serves
// all vectors: a warp handles one destination row (or one 2048-edge chunk of a hub
// row), each lane owns VPL of the W columns and reads them with one 16-byte load
// per 4 columns; column indices are read once per 32 edges and shared by shuffle.
// Per column the update is the single-vector one,
//   x'_v = alpha (sum_u a_uv g_u + d t_v) + (1 - alpha) t_v,  g'_v = x'_v / s_v,
// accumulated with compensated FP32 sums; the per-column L1 residual and dangling
// mass are reduced in FP64 in a fixed order (per-CTA partials, per-hub
// contributions, then the last CTA), and the loop stops when every column's
// residual is below tol.
#pragma once

#include "common.cuh"
#include "pr_binned.cuh"

namespace mg {

constexpr int PPR_NT = 256;
constexpr int PPR_MAXW = 256;  // vectors per group

struct PprArgs {
  const int32_t *off, *idx;  // CSC (gathered adjacency)
  const float *wts;          // its edge weights (nullptr: unit)
  const int32_t *rows;       // non-hub rows of the bin plan (bins 0..5), plan order
  int64_t nlight;
  const int32_t *hrows, *hbase;  // hub rows and their first chunk
  int64_t nheavy, nchunks;
  int32_t *hcount;  // arrival counters of the hubs (nheavy)
  int32_t *grab;    // work-item counter of the dynamic schedule (reset by the last CTA)
  Comp *hpart;      // hub chunk partial sums (nchunks x W)
  double *hres;     // per-hub FP64 contributions: residual (W) then dangling (W)
  const float *srow;  // s_u (0: dangling)
  const float *tele;  // n x W
  float *x0, *x1, *g0, *g1;  // n x W ping-pong
  double *dang;   // W: dangling mass of the current iterate
  double *part;   // grid x 2W per-CTA partials
  int64_t n;
  int32_t W;
  double alpha, tol;
  int32_t max_iter;
  int32_t grid;
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

// Column of element e of a lane: blocks of 4 columns at 128 q + 4 lane for
// VPL >= 4, else VPL consecutive columns at VPL * lane.
template <int VPL>
__device__ __forceinline__ int ppr_col(int lane, int e) {
  if (VPL >= 4) return 128 * (e >> 2) + 4 * lane + (e & 3);
  return VPL * lane + e;
}

template <int VPL>
__device__ __forceinline__ void ppr_load(const float *__restrict__ row, int lane, float (&v)[VPL]) {
  if constexpr (VPL >= 4) {
#pragma unroll
    for (int q = 0; q < VPL / 4; q++) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(row + 128 * q) + lane);
      v[4 * q] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  } else if constexpr (VPL == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(row) + lane);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    v[0] = __ldg(row + lane);
  }
}

template <int VPL>
__device__ __forceinline__ void ppr_store(float *row, int lane, const float (&v)[VPL]) {
  if constexpr (VPL >= 4) {
#pragma unroll
    for (int q = 0; q < VPL / 4; q++)
      reinterpret_cast<float4 *>(row + 128 * q)[lane] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else if constexpr (VPL == 2) {
    reinterpret_cast<float2 *>(row)[lane] = make_float2(v[0], v[1]);
  } else {
    row[lane] = v[0];
  }
}

// Compensated sums over edges [b, e) of the gathered rows, all W columns.
template <int VPL, bool WEIGHTED>
__device__ __forceinline__ void ppr_gather(const PprArgs &a, const float *__restrict__ gold, int32_t b, int32_t e,
                                           Comp (&acc)[VPL]) {
  const int lane = threadIdx.x & 31;
  const int64_t W = a.W;
  for (int32_t k0 = b; k0 < e; k0 += 32) {
    const int32_t kk = k0 + lane;
    const int32_t myc = kk < e ? __ldg(a.idx + kk) : 0;
    const float myw = (WEIGHTED && kk < e) ? __ldg(a.wts + kk) : 1.f;
    const int cnt = min(32, e - k0);
    int t = 0;
    for (; t + 4 <= cnt; t += 4) {
      float v[4][VPL];
#pragma unroll
      for (int u = 0; u < 4; u++) ppr_load<VPL>(gold + (int64_t)__shfl_sync(FULL, myc, t + u) * W, lane, v[u]);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const float wu = WEIGHTED ? __shfl_sync(FULL, myw, t + u) : 1.f;
#pragma unroll
        for (int j = 0; j < VPL; j++) {
          if (WEIGHTED) {
            const float p = wu * v[u][j];
            two_sum_add(acc[j], p);
            acc[j].lo += __fmaf_rn(wu, v[u][j], -p);
          } else {
            two_sum_add(acc[j], v[u][j]);
          }
        }
      }
    }
    for (; t < cnt; t++) {
      float v[VPL];
      ppr_load<VPL>(gold + (int64_t)__shfl_sync(FULL, myc, t) * W, lane, v);
      const float wu = WEIGHTED ? __shfl_sync(FULL, myw, t) : 1.f;
#pragma unroll
      for (int j = 0; j < VPL; j++) {
        if (WEIGHTED) {
          const float p = wu * v[j];
          two_sum_add(acc[j], p);
          acc[j].lo += __fmaf_rn(wu, v[j], -p);
        } else {
          two_sum_add(acc[j], v[j]);
        }
      }
    }
  }
}

// Row update of one destination row, all columns; adds |x' - x| and the dangling
// mass of x' into rs / ds.
template <int VPL>
__device__ __forceinline__ void ppr_update(const PprArgs &a, int64_t row, const Comp (&acc)[VPL],
                                           const float *__restrict__ xo, float *xn, float *gn,
                                           const double (&dj)[VPL], double (&rs)[VPL], double (&ds)[VPL]) {
  const int lane = threadIdx.x & 31;
  const int64_t W = a.W;
  const double s = (double)__ldg(a.srow + row);
  float t[VPL], xold[VPL], xnew[VPL], gnew[VPL];
  ppr_load<VPL>(a.tele + row * W, lane, t);
  ppr_load<VPL>(xo + row * W, lane, xold);
#pragma unroll
  for (int j = 0; j < VPL; j++) {
    const double sum = (double)acc[j].hi + (double)acc[j].lo;
    const double nv = a.alpha * (sum + dj[j] * (double)t[j]) + (1.0 - a.alpha) * (double)t[j];
    if (s > 0.0) {
      gnew[j] = (float)(nv / s);
    } else {
      gnew[j] = 0.f;
      ds[j] += nv;
    }
    xnew[j] = (float)nv;
    rs[j] += fabs((double)xnew[j] - (double)xold[j]);
  }
  ppr_store<VPL>(xn + row * W, lane, xnew);
  ppr_store<VPL>(gn + row * W, lane, gnew);
}

// Last CTA of an iteration: per-column FP64 totals in a fixed order, the new
// dangling masses, and the stop decision (every column below tol).
__device__ void ppr_iteration_end(const PprArgs &a, int cur, double *s_max) {
  DevCtl *c = a.ctl;
  double mx = 0.0;
  for (int col = threadIdx.x; col < a.W; col += blockDim.x) {
    double r = 0.0, d = 0.0;
    for (int b = 0; b < a.grid; b++) {
      r += __ldcg(a.part + (int64_t)b * 2 * a.W + col);
      d += __ldcg(a.part + (int64_t)b * 2 * a.W + a.W + col);
    }
    for (int64_t h = 0; h < a.nheavy; h++) {
      r += __ldcg(a.hres + h * 2 * a.W + col);
      d += __ldcg(a.hres + h * 2 * a.W + a.W + col);
    }
    a.dang[col] = d;
    mx = fmax(mx, r);
  }
  s_max[threadIdx.x] = mx;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) s_max[threadIdx.x] = fmax(s_max[threadIdx.x], s_max[threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int lvl = c->level + 1;
    c->level = lvl;
    c->dsum[0] = s_max[0];
    c->cur = cur ^ 1;
    c->blocks_done = 0;
    const bool done = s_max[0] < a.tol || lvl >= a.max_iter || c->status != 0;
    __threadfence();
    c->done = done ? 1 : 0;
    if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
  }
}

// One iteration for every column of the group. Warp items: hub chunks first (the
// longest items start first), then the non-hub rows; each warp takes the next
// item from a shared counter, so faster SMs take more.
template <int VPL, bool WEIGHTED>
__global__ void __launch_bounds__(PPR_NT) ppr_iter_kernel(PprArgs a) {
  __shared__ double s_red[2][PPR_NT / 32][32 * VPL];
  __shared__ double s_max[PPR_NT];
  __shared__ int s_last;
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const float *xo = cur ? a.x1 : a.x0;
  float *xn = cur ? a.x0 : a.x1;
  const float *go = cur ? a.g1 : a.g0;
  float *gn = cur ? a.g0 : a.g1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double dj[VPL], rs[VPL], ds[VPL];
#pragma unroll
  for (int j = 0; j < VPL; j++) {
    dj[j] = __ldcg(a.dang + ppr_col<VPL>(lane, j));
    rs[j] = 0.0;
    ds[j] = 0.0;
  }
  const int64_t total = a.nchunks + a.nlight;
  auto item = [&](int64_t it) {
    Comp acc[VPL];
#pragma unroll
    for (int j = 0; j < VPL; j++) acc[j] = Comp{0.f, 0.f};
    if (it >= a.nchunks) {
      const int32_t row = a.rows[it - a.nchunks];
      ppr_gather<VPL, WEIGHTED>(a, go, __ldg(a.off + row), __ldg(a.off + row + 1), acc);
      ppr_update<VPL>(a, row, acc, xo, xn, gn, dj, rs, ds);
      return;
    }
    // Hub chunk `it`: its hub by binary search over the chunk bases.
    int64_t lo = 0, hi = a.nheavy;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (a.hbase[mid] <= it) lo = mid;
      else hi = mid;
    }
    const int32_t row = a.hrows[lo];
    const int32_t b = __ldg(a.off + row) + (int32_t)(it - a.hbase[lo]) * PRB_CHUNK;
    const int32_t e = min(b + PRB_CHUNK, __ldg(a.off + row + 1));
    ppr_gather<VPL, WEIGHTED>(a, go, b, e, acc);
    Comp *mine = a.hpart + it * (int64_t)a.W;
#pragma unroll
    for (int j = 0; j < VPL; j++) mine[ppr_col<VPL>(lane, j)] = acc[j];
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) {
      const int32_t nch = a.hbase[lo + 1] - a.hbase[lo];
      last = atomicAdd(a.hcount + lo, 1) == nch - 1;
    }
    last = __shfl_sync(FULL, last, 0);
    if (!last) return;
    __threadfence();
    Comp tot[VPL];
#pragma unroll
    for (int j = 0; j < VPL; j++) tot[j] = Comp{0.f, 0.f};
    for (int32_t ch = a.hbase[lo]; ch < a.hbase[lo + 1]; ch++) {
      const Comp *pc = a.hpart + (int64_t)ch * a.W;
#pragma unroll
      for (int j = 0; j < VPL; j++) {
        const float2 v = __ldcg(reinterpret_cast<const float2 *>(pc + ppr_col<VPL>(lane, j)));
        comp_add(tot[j], Comp{v.x, v.y});
      }
    }
    if (lane == 0) a.hcount[lo] = 0;
    double hr[VPL], hd[VPL];
#pragma unroll
    for (int j = 0; j < VPL; j++) {
      hr[j] = 0.0;
      hd[j] = 0.0;
    }
    ppr_update<VPL>(a, row, tot, xo, xn, gn, dj, hr, hd);
    double *hc = a.hres + lo * 2 * (int64_t)a.W;
#pragma unroll
    for (int j = 0; j < VPL; j++) {
      hc[ppr_col<VPL>(lane, j)] = hr[j];
      hc[a.W + ppr_col<VPL>(lane, j)] = hd[j];
    }
    __threadfence();
  };
  for (;;) {
    int64_t it = 0;
    if (lane == 0) it = atomicAdd(a.grab, 1);
    it = __shfl_sync(FULL, it, 0);
    if (it >= total) break;
    item(it);
  }
  // Per-CTA partials, fixed order over the warps.
#pragma unroll
  for (int j = 0; j < VPL; j++) {
    s_red[0][warp][ppr_col<VPL>(lane, j)] = rs[j];
    s_red[1][warp][ppr_col<VPL>(lane, j)] = ds[j];
  }
  __syncthreads();
  for (int col = threadIdx.x; col < a.W; col += PPR_NT) {
    double r = 0.0, d = 0.0;
    for (int w = 0; w < PPR_NT / 32; w++) {
      r += s_red[0][w][col];
      d += s_red[1][w][col];
    }
    a.part[(int64_t)blockIdx.x * 2 * a.W + col] = r;
    a.part[(int64_t)blockIdx.x * 2 * a.W + a.W + col] = d;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&c->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (s_last) {
    __threadfence();
    if (threadIdx.x == 0) *a.grab = 0;
    ppr_iteration_end(a, cur, s_max);
  }
}

// x0 = t, g0 = t / s (0 dangling), per-CTA partial dangling masses.
template <int VPL>
__global__ void __launch_bounds__(PPR_NT) ppr_init_kernel(PprArgs a) {
  __shared__ double s_red[PPR_NT / 32][32 * VPL];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t W = a.W;
  double ds[VPL];
#pragma unroll
  for (int j = 0; j < VPL; j++) ds[j] = 0.0;
  const int64_t nwarps = ((int64_t)gridDim.x * PPR_NT) >> 5;
  for (int64_t v = ((int64_t)blockIdx.x * PPR_NT + threadIdx.x) >> 5; v < a.n; v += nwarps) {
    float t[VPL], gv[VPL];
    ppr_load<VPL>(a.tele + v * W, lane, t);
    const float s = a.srow[v];
#pragma unroll
    for (int j = 0; j < VPL; j++) {
      if (s > 0.f) {
        gv[j] = (float)((double)t[j] / (double)s);
      } else {
        gv[j] = 0.f;
        ds[j] += (double)t[j];
      }
    }
    ppr_store<VPL>(a.x0 + v * W, lane, t);
    ppr_store<VPL>(a.g0 + v * W, lane, gv);
  }
#pragma unroll
  for (int j = 0; j < VPL; j++) s_red[warp][ppr_col<VPL>(lane, j)] = ds[j];
  __syncthreads();
  for (int col = threadIdx.x; col < a.W; col += PPR_NT) {
    double d = 0.0;
    for (int w = 0; w < PPR_NT / 32; w++) d += s_red[w][col];
    a.part[(int64_t)blockIdx.x * 2 * a.W + col] = d;
  }
}

// dang[col] = sum of the init partials (fixed order); control block reset.
__global__ void ppr_init_reduce_kernel(PprArgs a, int32_t nparts) {
  for (int col = threadIdx.x; col < a.W; col += blockDim.x) {
    double d = 0.0;
    for (int b = 0; b < nparts; b++) d += a.part[(int64_t)b * 2 * a.W + col];
    a.dang[col] = d;
  }
  if (threadIdx.x == 0) {
    DevCtl *c = a.ctl;
    c->level = 0;
    c->cur = 0;
    c->blocks_done = 0;
    c->iter_cap = a.max_iter;
    c->done = a.max_iter <= 0 ? 1 : 0;
  }
}

// Teleport rows (k x n, row i for column c0 + i; nullptr: uniform 1/n) into the
// vertex-major n x W block; columns past k are 0.
__global__ void ppr_pack_kernel(const float *__restrict__ src, int32_t k, int64_t n, int32_t W, float *__restrict__ dst) {
  __shared__ float tile[32][33];
  const int64_t v0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int col = c0 + r;
    const int64_t v = v0 + threadIdx.x;
    float x = 0.f;
    if (col < k && v < n) x = src ? src[(int64_t)col * n + v] : (float)(1.0 / (double)n);
    tile[r][threadIdx.x] = x;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t v = v0 + r;
    if (v < n) dst[v * W + c0 + threadIdx.x] = tile[threadIdx.x][r];
  }
}

// Columns [0, k) of the vertex-major block back into k rows of n.
__global__ void ppr_unpack_kernel(const float *__restrict__ src, int32_t k, int64_t n, int32_t W, float *__restrict__ dst) {
  __shared__ float tile[32][33];
  const int64_t v0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t v = v0 + r;
    tile[r][threadIdx.x] = v < n ? src[v * W + c0 + threadIdx.x] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int col = c0 + r;
    const int64_t v = v0 + threadIdx.x;
    if (col < k && v < n) dst[(int64_t)col * n + v] = tile[threadIdx.x][r];
  }
}

}  // namespace mg
