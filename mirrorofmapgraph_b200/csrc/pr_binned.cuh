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
// Resident CTAs per SM the iteration kernel is compiled for, and how many passes
// of a light bin issue their loads before the first reduction.
#ifndef PRB_MIN_BLOCKS
#define PRB_MIN_BLOCKS 6
#endif
#ifndef PRB_BATCH
#define PRB_BATCH 8
#endif
// Strides of 32 edges a warp-per-row gather loads before its first add.
#ifndef PRB_UNROLL
#define PRB_UNROLL 8
#endif
// Index (and weight) streams are read once per iteration: loads marked
// evict-first (ld.global.cs) keep them from displacing the gathered vector in
// L1 and L2. PRB_STREAM_LOADS=0 uses plain read-only loads instead.
#ifndef PRB_STREAM_LOADS
#define PRB_STREAM_LOADS 1
#endif
template <typename T>
__device__ __forceinline__ T prb_stream(const T *p) {
#if PRB_STREAM_LOADS
  return __ldcs(p);
#else
  return __ldg(p);
#endif
}
#ifndef PRB_HEAVY_EDGES
#define PRB_HEAVY_EDGES 2048
#endif
// Assignment order of a persistent warp: 1 walks the plan from the hub chunks and
// the heaviest bins down to the lightest (longest items first shortens the
// tail); 0 walks bins 0..6 in order.
// Solve kernels take their work items from a shared counter (1) or by a fixed
// grid stride (0).
#ifndef PRB_DYNAMIC
#define PRB_DYNAMIC 1
#endif
// Work items a warp takes per grab of the dynamic schedule.
#ifndef PRB_GRAB
#define PRB_GRAB 1
#endif
#ifndef PRB_HEAVY_FIRST
#define PRB_HEAVY_FIRST 1
#endif
constexpr int32_t PRB_HEAVY = PRB_HEAVY_EDGES;
constexpr int32_t PRB_CHUNK = 2048;

// Plan of one adjacency.
struct BinPlan {
  int32_t *rows = nullptr;      // rows grouped by bin (bins 0..5), bin b at rows[boff[b]..]
  int32_t *hrows = nullptr;     // hub rows (bin 6)
  int32_t *hbase = nullptr;     // first chunk task of each hub, nheavy + 1 entries
  int32_t *hcount = nullptr;    // arrival counters of the hubs (reset by the finishing warp)
  Comp *hpart = nullptr;        // partial sums of the hub chunks
  double *hcontrib = nullptr;   // per-hub FP64 contributions (residual, second reduction)
  int32_t *grab = nullptr;      // work-item counter of the dynamic schedule (zero between launches)
  int64_t boff[PRB_BINS + 1] = {0};  // bin offsets into rows (bin 6 unused)
  int64_t nheavy = 0, ntasks = 0;
  int64_t wstart[PRB_BINS + 1] = {0};  // first warp assignment of each bin
};

}  // namespace mg

// Host side (pagerank.cu): builds / releases a plan over `off` (n + 1 entries);
// rows of at least `heavy` edges become hubs.
mg_status bin_plan_build(cudaStream_t s, const int32_t *off, int64_t n, mg::BinPlan &bp,
                         int32_t heavy = mg::PRB_HEAVY);
void bin_plan_release(cudaStream_t s, mg::BinPlan &bp);

namespace mg {

// Bin of a row of `deg` edges; rows of at least `heavy` edges are hubs (bin 6).
__device__ __forceinline__ int prb_bin_of(int32_t deg, int32_t heavy = PRB_HEAVY) {
  if (deg >= heavy) return 6;
  if (deg <= 1) return 0;
  if (deg <= 2) return 1;
  if (deg <= 4) return 2;
  if (deg <= 8) return 3;
  if (deg <= 16) return 4;
  return 5;
}

// Ordered binning. Rows are cut into chunks of PRB_NT * PRB_RPT rows, one per
// CTA; pass 1 counts every bin per chunk, a single CTA turns the counts into
// output offsets (bin-major, chunk order), and pass 2 writes each chunk's rows in
// row order with an in-CTA exclusive scan per bin. Bins therefore list rows in
// ascending order and the plan is deterministic.
constexpr int PRB_RPT = 8;
constexpr int PRB_CHUNK_ROWS = PRB_NT * PRB_RPT;

#ifndef MG_PRB_NO_PLAN_KERNELS  // plan building runs in pagerank.cu only
__global__ void __launch_bounds__(PRB_NT) prb_count_kernel(const int32_t *__restrict__ off, int64_t n,
                                                           int64_t *__restrict__ counts /* [chunk][BINS+1] */,
                                                           int32_t heavy) {
  __shared__ int64_t s[PRB_BINS + 1];
  if (threadIdx.x <= PRB_BINS) s[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * PRB_CHUNK_ROWS;
  for (int k = 0; k < PRB_RPT; k++) {
    const int64_t r = base + (int64_t)threadIdx.x * PRB_RPT + k;
    if (r < n) {
      const int32_t d = off[r + 1] - off[r];
      const int b = prb_bin_of(d, heavy);
      atomicAdd((unsigned long long *)&s[b], 1ull);
      if (b == 6) atomicAdd((unsigned long long *)&s[PRB_BINS], (unsigned long long)((d + PRB_CHUNK - 1) / PRB_CHUNK));
    }
  }
  __syncthreads();
  if (threadIdx.x <= PRB_BINS) counts[(int64_t)blockIdx.x * (PRB_BINS + 1) + threadIdx.x] = s[threadIdx.x];
}

// Exclusive prefix over chunks of every bin, in place; totals[b] = bin sizes.
__global__ void prb_offsets_kernel(int64_t *counts, int64_t nchunks, int64_t *totals) {
  const int b = threadIdx.x;
  if (b > PRB_BINS) return;
  int64_t acc = 0;
  for (int64_t c = 0; c < nchunks; c++) {
    const int64_t v = counts[c * (PRB_BINS + 1) + b];
    counts[c * (PRB_BINS + 1) + b] = acc;
    acc += v;
  }
  totals[b] = acc;
}

__global__ void __launch_bounds__(PRB_NT) prb_scatter_kernel(const int32_t *__restrict__ off, int64_t n,
                                                             const int64_t *__restrict__ offsets,
                                                             const int64_t *__restrict__ boff, int32_t *rows,
                                                             int32_t *hrows, int32_t heavy) {
  __shared__ int32_t red[PRB_NT / 32 + 1];
  const int64_t base = (int64_t)blockIdx.x * PRB_CHUNK_ROWS;
  int bins[PRB_RPT];
#pragma unroll
  for (int k = 0; k < PRB_RPT; k++) {
    const int64_t r = base + (int64_t)threadIdx.x * PRB_RPT + k;
    bins[k] = r < n ? prb_bin_of(off[r + 1] - off[r], heavy) : -1;
  }
  for (int b = 0; b < PRB_BINS; b++) {
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < PRB_RPT; k++) cnt += bins[k] == b;
    int32_t tot;
    int pos = block_exclusive_scan<PRB_NT>(cnt, red, &tot);
    const int64_t o = offsets[(int64_t)blockIdx.x * (PRB_BINS + 1) + b];
#pragma unroll
    for (int k = 0; k < PRB_RPT; k++) {
      if (bins[k] == b) {
        const int32_t r = (int32_t)(base + (int64_t)threadIdx.x * PRB_RPT + k);
        if (b < 6) rows[boff[b] + o + pos] = r;
        else hrows[o + pos] = r;
        pos++;
      }
    }
  }
}

// Chunk bases of the hubs (listed in ascending order): one CTA, exclusive scan of
// their chunk counts PRB_NT at a time.
__global__ void __launch_bounds__(PRB_NT) prb_hubs_kernel(const int32_t *__restrict__ off, const int32_t *hrows,
                                                          int64_t nheavy, int32_t *hbase) {
  __shared__ int32_t red[PRB_NT / 32 + 1];
  int32_t carry = 0;
  for (int64_t b0 = 0; b0 < nheavy; b0 += PRB_NT) {
    const int64_t i = b0 + threadIdx.x;
    int32_t c = 0;
    if (i < nheavy) {
      const int32_t d = off[hrows[i] + 1] - off[hrows[i]];
      c = (d + PRB_CHUNK - 1) / PRB_CHUNK;
    }
    int32_t tot;
    const int32_t ex = block_exclusive_scan<PRB_NT>(c, red, &tot);
    if (i < nheavy) hbase[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) hbase[nheavy] = carry;
}
#endif  // MG_PRB_NO_PLAN_KERNELS

struct PrbArgs {
  const int32_t *off, *idx;
  const float *wts;
  const int32_t *rows, *hrows, *hbase;
  int32_t *hcount;
  Comp *hpart;
  double *hcontrib;
  // Dynamic schedule: warps take PRB_GRAB work items at a time from this counter
  // (heaviest first) instead of a fixed grid stride; the launch's last CTA
  // resets it. nullptr: fixed stride.
  int32_t *grab;
  int64_t boff[PRB_BINS + 1];
  int64_t wstart[PRB_BINS + 1];
  int64_t nheavy;
};

template <bool WEIGHTED>
__device__ __forceinline__ void prb_add(Comp &acc, float g, const float *__restrict__ wts, int32_t k) {
  if (WEIGHTED) {
    const float a = prb_stream(wts + k);
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

// U strides of 32 edges of a row from `base` (warp-uniform); CHECK predicates
// each slot on the row end (the last round of a row).
template <bool WEIGHTED, int U, bool CHECK, typename Gather>
__device__ __forceinline__ void prb_round(const PrbArgs &p, int32_t base, int32_t e, Gather &gather, Comp &acc) {
  const int32_t k = base + (threadIdx.x & 31);
  int32_t c[U];
  float x[U];
#pragma unroll
  for (int j = 0; j < U; j++) c[j] = (!CHECK || k + 32 * j < e) ? prb_stream(p.idx + k + 32 * j) : 0;
#pragma unroll
  for (int j = 0; j < U; j++) x[j] = (!CHECK || k + 32 * j < e) ? gather(c[j]) : 0.f;
#pragma unroll
  for (int j = 0; j < U; j++)
    if (!CHECK || k + 32 * j < e) prb_add<WEIGHTED>(acc, x[j], p.wts, k + 32 * j);
}

// One warp reduces edges [b, e) of a row in rounds of PRB_UNROLL strides of 32
// edges (all loads of a round in flight together). ADAPT: full rounds run without
// per-slot checks and the last round is sized to what is left (8, 4, 2 or 1
// strides), so short rows do not pay for idle slots; otherwise each lane walks
// its own edges in full predicated rounds (fewer code paths, which suits some
// register-tight launch shapes).
template <bool WEIGHTED, bool ADAPT, typename Gather>
__device__ __forceinline__ Comp prb_warp_range(const PrbArgs &p, int32_t b, int32_t e, Gather &gather) {
  Comp acc{0.f, 0.f};
  if (ADAPT) {
    int32_t base = b;
    for (; base + 32 * PRB_UNROLL <= e; base += 32 * PRB_UNROLL)
      prb_round<WEIGHTED, PRB_UNROLL, false>(p, base, e, gather, acc);
    const int32_t rem = e - base;
    if (rem > 128) prb_round<WEIGHTED, PRB_UNROLL, true>(p, base, e, gather, acc);
    else if (rem > 64) prb_round<WEIGHTED, 4, true>(p, base, e, gather, acc);
    else if (rem > 32) prb_round<WEIGHTED, 2, true>(p, base, e, gather, acc);
    else if (rem > 0) prb_round<WEIGHTED, 1, true>(p, base, e, gather, acc);
  } else {
    // per-lane loop: a lane stops after its last edge
    for (int32_t k = b + (threadIdx.x & 31); k < e; k += 32 * PRB_UNROLL) {
      int32_t c[PRB_UNROLL];
      float x[PRB_UNROLL];
#pragma unroll
      for (int j = 0; j < PRB_UNROLL; j++) c[j] = k + 32 * j < e ? prb_stream(p.idx + k + 32 * j) : 0;
#pragma unroll
      for (int j = 0; j < PRB_UNROLL; j++) x[j] = k + 32 * j < e ? gather(c[j]) : 0.f;
#pragma unroll
      for (int j = 0; j < PRB_UNROLL; j++)
        if (k + 32 * j < e) prb_add<WEIGHTED>(acc, x[j], p.wts, k + 32 * j);
    }
  }
  group_comp_reduce<32>(acc);
  return acc;
}

// 32 consecutive rows of bin `bin` (warp assignment `wa`), G lanes per row:
// every lane first loads its slot's row and offsets; then G passes of 32/G rows
// each. For light bins (G < 32, at most G edges per row) all G passes issue their
// index loads and then their gathers back to back before any reduction, so a warp
// waits for three memory round trips per assignment rather than three per pass.
// The sum of slot l ends up in lane l, whose row is returned in *my_row (-1 past
// the bin), so the row updates then run on all lanes at once.
// prb_ranges32 is the same for 32 edge ranges [mb, me) given per lane (at most G
// edges each for G < 32): the sum of lane l's range ends up in lane l.
template <int G, bool WEIGHTED, bool ADAPT, typename Gather>
__device__ __forceinline__ Comp prb_ranges32(const PrbArgs &p, int32_t mb, int32_t me, Gather &gather) {
  constexpr int RPP = 32 / G;  // rows per pass
  const int lane = threadIdx.x & 31;
  const int gl = lane % G, grp = lane / G;
  Comp mine{0.f, 0.f};
  if (G == 32) {
#pragma unroll 1
    for (int q = 0; q < 32; q++) {
      const int32_t b = __shfl_sync(0xffffffffu, mb, q), e = __shfl_sync(0xffffffffu, me, q);
      const Comp acc = prb_warp_range<WEIGHTED, ADAPT>(p, b, e, gather);
      if (lane == q) mine = acc;
    }
  } else {
    // Passes run in batches of up to 8 so the in-flight loads fit the register budget.
    constexpr int BATCH = G < PRB_BATCH ? G : PRB_BATCH;
#pragma unroll
    for (int q0 = 0; q0 < G; q0 += BATCH) {
      int32_t k_of[BATCH];
      int32_t c_of[BATCH];
      float v_of[BATCH];
#pragma unroll
      for (int j = 0; j < BATCH; j++) {
        const int src = (q0 + j) * RPP + grp;
        const int32_t b = __shfl_sync(0xffffffffu, mb, src), e = __shfl_sync(0xffffffffu, me, src);
        k_of[j] = b + gl < e ? b + gl : -1;
      }
#pragma unroll
      for (int j = 0; j < BATCH; j++) c_of[j] = k_of[j] >= 0 ? prb_stream(p.idx + k_of[j]) : 0;
#pragma unroll
      for (int j = 0; j < BATCH; j++) v_of[j] = k_of[j] >= 0 ? gather(c_of[j]) : 0.f;
#pragma unroll
      for (int j = 0; j < BATCH; j++) {
        Comp acc{0.f, 0.f};
        if (k_of[j] >= 0) prb_add<WEIGHTED>(acc, v_of[j], p.wts, k_of[j]);
        group_comp_reduce<G>(acc);
        const int src = (lane % RPP) * G;
        const float h = __shfl_sync(0xffffffffu, acc.hi, src), l = __shfl_sync(0xffffffffu, acc.lo, src);
        if (lane / RPP == q0 + j) mine = Comp{h, l};
      }
    }
  }
  return mine;
}

template <int G, bool WEIGHTED, bool ADAPT, typename Gather>
__device__ __forceinline__ Comp prb_rows32(const PrbArgs &p, int bin, int64_t wa, Gather &gather, int32_t *my_row) {
  const int lane = threadIdx.x & 31;
  const int64_t slot = p.boff[bin] + wa * 32 + lane;
  const int32_t mine_row = slot < p.boff[bin + 1] ? p.rows[slot] : -1;
  const int32_t mb = mine_row >= 0 ? __ldg(p.off + mine_row) : 0;
  const int32_t me = mine_row >= 0 ? __ldg(p.off + mine_row + 1) : 0;
  *my_row = mine_row;
  return prb_ranges32<G, WEIGHTED, ADAPT>(p, mb, me, gather);
}

// Walks every assignment of the plan with a persistent grid (fixed stride).
// finish(row, Comp) consumes a row sum; finish_hub(h, row, Comp) consumes a hub's.
template <bool WEIGHTED, bool ADAPT = true, typename Gather, typename Finish, typename FinishHub>
__device__ __forceinline__ void prb_run(const PrbArgs &p, Gather &&gather, Finish &&finish, FinishHub &&finish_hub) {
  const int64_t total = p.wstart[PRB_BINS];
  const int lane = threadIdx.x & 31;
  auto item = [&](int64_t wi) {
    const int64_t w = PRB_HEAVY_FIRST ? total - 1 - wi : wi;
    int bin = 0;
#pragma unroll
    for (int q = 1; q < PRB_BINS; q++)
      if (w >= p.wstart[q]) bin = q;
    const int64_t wa = w - p.wstart[bin];
    if (bin < 6) {
      int32_t row = -1;
      Comp acc;
      switch (bin) {
        case 0: acc = prb_rows32<1, WEIGHTED, ADAPT>(p, 0, wa, gather, &row); break;
        case 1: acc = prb_rows32<2, WEIGHTED, ADAPT>(p, 1, wa, gather, &row); break;
        case 2: acc = prb_rows32<4, WEIGHTED, ADAPT>(p, 2, wa, gather, &row); break;
        case 3: acc = prb_rows32<8, WEIGHTED, ADAPT>(p, 3, wa, gather, &row); break;
        case 4: acc = prb_rows32<16, WEIGHTED, ADAPT>(p, 4, wa, gather, &row); break;
        default: acc = prb_rows32<32, WEIGHTED, ADAPT>(p, 5, wa, gather, &row); break;
      }
      if (row >= 0) finish(row, acc);
      return;
    }
    switch (bin) {
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
        const Comp acc = prb_warp_range<WEIGHTED, ADAPT>(p, b, e, gather);
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
  };
  if (p.grab) {
    for (;;) {
      int64_t base = 0;
      if (lane == 0) base = atomicAdd(p.grab, PRB_GRAB);
      base = __shfl_sync(FULL, base, 0);
      if (base >= total) break;
      const int64_t end = min(base + (int64_t)PRB_GRAB, total);
      for (int64_t wi = base; wi < end; wi++) item(wi);
    }
  } else {
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t wi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < total; wi += nwarps) item(wi);
  }
}

}  // namespace mg
