// pr_binned.cuh -- degree-binned gather over a CSR-shaped adjacency, the default
// PageRank / adjoint gather.
//
// Rows are binned once per adjacency by degree and each bin gets the lane count
// that covers its rows in one pass:
//   bin 0..4  degree <= 1, 2, 4, 8, 16: groups of 1, 2, 4, 8, 16 lanes per row
//             (32 / G rows per warp), each group reads its row's edges with
//             consecutive lanes and reduces with a shuffle tree of log2 G steps;
//   bin 5     degree < PRB_HEAVY: one warp per row, 32 consecutive edges per step;
//   bin 6     degree >= PRB_HEAVY (hubs): split into chunks of PRB_CHUNK edges; a
//             warp reduces one chunk into a partial; the warp that completes a
//             hub's last chunk (per-row arrival counter) adds the partials in
//             chunk order and finishes the row.
// Warps are independent (no CTA barriers while gathering) and every edge load is
// a coalesced stream. The per-row sums are compensated (TwoSum per addend,
// FMA-based TwoProduct for weights) and every row's sum has a fixed order, so the
// result does not depend on scheduling. A persistent grid walks the assignments
// with a fixed stride, so each CTA's FP64 partials (residual, dangling mass) are
// deterministic too; hub rows keep their contributions in a per-hub array.
#pragma once

#include "common.cuh"
#include "pr_gather.cuh"

namespace mg {

constexpr int PRB_NT = 256;
constexpr int PRB_BINS = 7;
constexpr int32_t PRB_HEAVY = 2048;
constexpr int32_t PRB_CHUNK = 2048;

// Plan of one adjacency.
struct BinPlan {
  int32_t *rows = nullptr;      // rows grouped by bin (bins 0..5), bin b at rows[boff[b]..]
  int32_t *hrows = nullptr;     // hub rows (bin 6)
  int32_t *hbase = nullptr;     // first chunk task of each hub, nheavy + 1 entries
  int32_t *hcount = nullptr;    // arrival counters of the hubs (reset by the finishing warp)
  Comp *hpart = nullptr;        // partial sums of the hub chunks
  double *hcontrib = nullptr;   // per-hub FP64 contributions (residual, second reduction)
  int64_t boff[PRB_BINS + 1] = {0};  // bin offsets into rows (bin 6 unused)
  int64_t nheavy = 0, ntasks = 0;
  int64_t wstart[PRB_BINS + 1] = {0};  // first warp assignment of each bin
};

__device__ __forceinline__ int prb_bin_of(int32_t deg) {
  if (deg <= 1) return 0;
  if (deg <= 2) return 1;
  if (deg <= 4) return 2;
  if (deg <= 8) return 3;
  if (deg <= 16) return 4;
  if (deg < PRB_HEAVY) return 5;
  return 6;
}

__global__ void prb_count_kernel(const int32_t *__restrict__ off, int64_t n, unsigned long long *cnt) {
  __shared__ unsigned long long s[PRB_BINS + 1];
  if (threadIdx.x <= PRB_BINS) s[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = off[r + 1] - off[r];
    const int b = prb_bin_of(d);
    atomicAdd(&s[b], 1ull);
    if (b == 6) atomicAdd(&s[PRB_BINS], (unsigned long long)((d + PRB_CHUNK - 1) / PRB_CHUNK));
  }
  __syncthreads();
  if (threadIdx.x <= PRB_BINS && s[threadIdx.x]) atomicAdd(&cnt[threadIdx.x], s[threadIdx.x]);
}

// Scatters rows into their bins (order inside a bin does not affect results).
__global__ void prb_scatter_kernel(const int32_t *__restrict__ off, int64_t n, const int64_t *__restrict__ boff,
                                   unsigned long long *cursor, int32_t *rows, int32_t *hrows) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int b = prb_bin_of(off[r + 1] - off[r]);
    const unsigned long long p = atomicAdd(&cursor[b], 1ull);
    if (b < 6) rows[boff[b] + (int64_t)p] = (int32_t)r;
    else hrows[p] = (int32_t)r;
  }
}

// Sorts the hub list (tiny) and fills the chunk bases; one CTA.
__global__ void prb_hubs_kernel(const int32_t *__restrict__ off, int32_t *hrows, int64_t nheavy, int32_t *hbase) {
  if (threadIdx.x != 0) return;
  for (int64_t i = 1; i < nheavy; i++) {  // insertion sort: hubs are few and the list is built once
    const int32_t v = hrows[i];
    int64_t j = i - 1;
    while (j >= 0 && hrows[j] > v) {
      hrows[j + 1] = hrows[j];
      j--;
    }
    hrows[j + 1] = v;
  }
  int32_t acc = 0;
  for (int64_t i = 0; i < nheavy; i++) {
    hbase[i] = acc;
    const int32_t d = off[hrows[i] + 1] - off[hrows[i]];
    acc += (d + PRB_CHUNK - 1) / PRB_CHUNK;
  }
  hbase[nheavy] = acc;
}

struct PrbArgs {
  const int32_t *off, *idx;
  const float *wts;
  const int32_t *rows, *hrows, *hbase;
  int32_t *hcount;
  Comp *hpart;
  double *hcontrib;
  int64_t boff[PRB_BINS + 1];
  int64_t wstart[PRB_BINS + 1];
  int64_t nheavy;
};

template <bool WEIGHTED>
__device__ __forceinline__ void prb_add(Comp &acc, float g, const float *__restrict__ wts, int32_t k) {
  if (WEIGHTED) {
    const float a = __ldg(wts + k);
    const float p = a * g;
    two_sum_add(acc, p);
    acc.lo += __fmaf_rn(a, g, -p);
  } else {
    two_sum_add(acc, g);
  }
}

template <int G>
__device__ __forceinline__ void group_comp_reduce(Comp &c) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    Comp d{__shfl_xor_sync(0xffffffffu, c.hi, o), __shfl_xor_sync(0xffffffffu, c.lo, o)};
    // Fixed pairing: the lower lane of each pair adds the upper one's value.
    if ((threadIdx.x & o) == 0) comp_add(c, d);
    else {
      comp_add(d, c);
      c = d;
    }
  }
}

// Rows of a light bin with G lanes per row; warp assignment `wa` within the bin.
template <int G, bool WEIGHTED, typename Gather, typename Finish>
__device__ __forceinline__ void prb_light(const PrbArgs &p, int bin, int64_t wa, Gather &gather, Finish &finish) {
  const int lane = threadIdx.x & 31;
  const int64_t i = wa * (32 / G) + lane / G;
  const int gl = lane % G;
  const int64_t nb = p.boff[bin + 1] - p.boff[bin];
  int32_t row = -1, b = 0, e = 0;
  if (i < nb) {
    row = p.rows[p.boff[bin] + i];
    b = __ldg(p.off + row);
    e = __ldg(p.off + row + 1);
  }
  Comp acc{0.f, 0.f};
  for (int32_t k = b + gl; k < e; k += G) prb_add<WEIGHTED>(acc, gather(__ldg(p.idx + k)), p.wts, k);
  group_comp_reduce<G>(acc);
  if (row >= 0 && gl == 0) finish(row, acc);
}

// One warp reduces edges [b, e) of a row: 4 independent loads in flight per lane.
template <bool WEIGHTED, typename Gather>
__device__ __forceinline__ Comp prb_warp_range(const PrbArgs &p, int32_t b, int32_t e, Gather &gather) {
  const int lane = threadIdx.x & 31;
  Comp acc{0.f, 0.f};
  int32_t k = b + lane;
  for (; k + 96 < e; k += 128) {
    const int32_t c0 = __ldg(p.idx + k), c1 = __ldg(p.idx + k + 32), c2 = __ldg(p.idx + k + 64),
                  c3 = __ldg(p.idx + k + 96);
    const float g0 = gather(c0), g1 = gather(c1), g2 = gather(c2), g3 = gather(c3);
    prb_add<WEIGHTED>(acc, g0, p.wts, k);
    prb_add<WEIGHTED>(acc, g1, p.wts, k + 32);
    prb_add<WEIGHTED>(acc, g2, p.wts, k + 64);
    prb_add<WEIGHTED>(acc, g3, p.wts, k + 96);
  }
  for (; k < e; k += 32) prb_add<WEIGHTED>(acc, gather(__ldg(p.idx + k)), p.wts, k);
  group_comp_reduce<32>(acc);
  return acc;
}

// Walks every assignment of the plan with a persistent grid (fixed stride).
// finish(row, Comp) consumes a row sum; finish_hub(h, row, Comp) consumes a hub's.
template <bool WEIGHTED, typename Gather, typename Finish, typename FinishHub>
__device__ __forceinline__ void prb_run(const PrbArgs &p, Gather &&gather, Finish &&finish, FinishHub &&finish_hub) {
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t total = p.wstart[PRB_BINS];
  const int lane = threadIdx.x & 31;
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += nwarps) {
    int bin = 0;
#pragma unroll
    for (int q = 1; q < PRB_BINS; q++)
      if (w >= p.wstart[q]) bin = q;
    const int64_t wa = w - p.wstart[bin];
    switch (bin) {
      case 0: prb_light<1, WEIGHTED>(p, 0, wa, gather, finish); break;
      case 1: prb_light<2, WEIGHTED>(p, 1, wa, gather, finish); break;
      case 2: prb_light<4, WEIGHTED>(p, 2, wa, gather, finish); break;
      case 3: prb_light<8, WEIGHTED>(p, 3, wa, gather, finish); break;
      case 4: prb_light<16, WEIGHTED>(p, 4, wa, gather, finish); break;
      case 5: {
        const int32_t row = p.rows[p.boff[5] + wa];
        const Comp acc = prb_warp_range<WEIGHTED>(p, __ldg(p.off + row), __ldg(p.off + row + 1), gather);
        if (lane == 0) finish(row, acc);
        break;
      }
      default: {
        // Hub chunk task `wa`: find its hub by binary search over the chunk bases.
        int64_t lo = 0, hi = p.nheavy;
        while (hi - lo > 1) {
          const int64_t mid = (lo + hi) >> 1;
          if (p.hbase[mid] <= wa) lo = mid;
          else hi = mid;
        }
        const int32_t row = p.hrows[lo];
        const int32_t chunk = (int32_t)(wa - p.hbase[lo]);
        const int32_t rb = __ldg(p.off + row);
        const int32_t b = rb + chunk * PRB_CHUNK;
        const int32_t e = min(b + PRB_CHUNK, __ldg(p.off + row + 1));
        const Comp acc = prb_warp_range<WEIGHTED>(p, b, e, gather);
        bool last = false;
        if (lane == 0) {
          p.hpart[wa] = acc;
          __threadfence();
          const int32_t nch = p.hbase[lo + 1] - p.hbase[lo];
          last = atomicAdd(p.hcount + lo, 1) == nch - 1;
          if (last) {
            __threadfence();
            Comp tot{0.f, 0.f};
            const float2 *parts = reinterpret_cast<const float2 *>(p.hpart) + p.hbase[lo];
            for (int32_t c = 0; c < nch; c++) {
              const float2 v = __ldcg(parts + c);  // written by other SMs: read from L2
              comp_add(tot, Comp{v.x, v.y});
            }
            p.hcount[lo] = 0;
            finish_hub(lo, row, tot);
          }
        }
        break;
      }
    }
  }
}

}  // namespace mg
