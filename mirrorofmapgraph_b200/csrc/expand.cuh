// expand.cuh -- degree-binned expansion of a tile of vertices (thread / warp /
// CTA bins), shared by the traversal programs.
//
// Each thread of an NT-thread CTA brings one vertex (or -1). Vertices with at
// least CTA_TH edges are expanded by the whole CTA, those with at least 32 by
// one warp, and the rest through a block-wide exclusive scan of their degrees:
// the CTA then walks the concatenated edge slots and each slot finds its owner by
// binary search in shared memory. Every edge load is coalesced within a warp.
// This is the role of the reference's TWC expansion
// (GASengine/vertex_centric/expand_atomic/cta.cuh:268-421 ExpandByCta /
// ExpandByWarp, :705-758 scan-based gather).
//
// visit(v, k) is called once per edge k of vertex v (k indexes the edge arrays
// behind `off`).
#pragma once

#include "common.cuh"

namespace mg {

// P: the type of a per-vertex payload handed to visit() beside the vertex (for
// example the vertex's distance or frontier mask, read once per vertex instead of
// once per edge).
template <int NT, typename P = int32_t>
struct ExpandSmem {
  int32_t scan[NT];
  int32_t beg[NT];
  int32_t vtx[NT];
  P pay[NT];
  int32_t red[NT / 32 + 1];
  int32_t cta[4];
  P cpay;
};

struct BigList;
__device__ __forceinline__ bool defer_big(const BigList &big, int32_t v, int32_t deg);

// visit(v, payload, k) for every edge k of the tile's vertices; each thread brings
// its vertex v (or -1) and that vertex's payload.
//
// `vmask` maps a frontier item to the vertex whose offsets it uses (item & vmask);
// -1 (every bit) is the identity. Batched runs pack an instance number into the
// item's high bits and pass the low-bit mask.
//
// `cta_th` (default CTA_TH) is the out-degree from which the whole CTA expands a
// vertex; callers with a tuned threshold pass it at run time.
template <int NT, int CTA_TH, typename P, typename Visit>
__device__ __forceinline__ void expand_tile_p(ExpandSmem<NT, P> &sm, const int32_t *__restrict__ off, int32_t v,
                                              P pay, int64_t &insp, Visit &&visit, const BigList *big = nullptr,
                                              int32_t vmask = -1, int32_t cta_th = CTA_TH) {
  const int tid = threadIdx.x, lane = lane_id();
  int32_t beg = 0, deg = 0;
  if (v >= 0) {
    beg = off[v & vmask];
    deg = off[(v & vmask) + 1] - beg;
    insp += deg;
  }
  // Vertices for the grid-strided bin are expanded by a later kernel.
  if (big && defer_big(*big, v, deg)) deg = 0;
  // CTA bin.
  while (__syncthreads_or(deg >= cta_th)) {
    if (deg >= cta_th) sm.cta[0] = tid;
    __syncthreads();
    if (sm.cta[0] == tid) {
      sm.cta[1] = beg;
      sm.cta[2] = beg + deg;
      sm.cta[3] = v;
      sm.cpay = pay;
      deg = 0;
    }
    __syncthreads();
    const int32_t b = sm.cta[1], e = sm.cta[2], cv = sm.cta[3];
    const P cp = sm.cpay;
    for (int32_t k = b + tid; k < e; k += NT) visit(cv, cp, k);
  }
  // Warp bin.
  for (;;) {
    const unsigned wm = __ballot_sync(FULL, deg >= 32);
    if (!wm) break;
    const int l = __ffs(wm) - 1;
    const int32_t b = __shfl_sync(FULL, beg, l), e = __shfl_sync(FULL, beg + deg, l);
    const int32_t wv = __shfl_sync(FULL, v, l);
    const P wp = __shfl_sync(FULL, pay, l);
    if (lane == l) deg = 0;
    for (int32_t k = b + lane; k < e; k += 32) visit(wv, wp, k);
  }
  // Thread bin.
  int32_t total;
  const int32_t ex = block_exclusive_scan<NT>(deg, sm.red, &total);
  sm.scan[tid] = ex;
  sm.beg[tid] = beg;
  sm.vtx[tid] = v;
  sm.pay[tid] = pay;
  __syncthreads();
  for (int32_t k = tid; k < total; k += NT) {
    int lo = 0, hi = NT;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (sm.scan[mid] <= k) lo = mid;
      else hi = mid;
    }
    visit(sm.vtx[lo], sm.pay[lo], sm.beg[lo] + (k - sm.scan[lo]));
  }
  __syncthreads();
}

// expand_tile_p without a payload: visit(v, k).
template <int NT, int CTA_TH, typename Visit>
__device__ __forceinline__ void expand_tile(ExpandSmem<NT> &sm, const int32_t *__restrict__ off, int32_t v,
                                            int64_t &insp, Visit &&visit, const BigList *big = nullptr,
                                            int32_t vmask = -1, int32_t cta_th = CTA_TH) {
  expand_tile_p<NT, CTA_TH>(sm, off, v, (int32_t)0, insp, [&](int32_t sv, int32_t, int32_t k) { visit(sv, k); },
                            big, vmask, cta_th);
}

template <typename T>
__device__ __forceinline__ T vload(const T *p) {
  return *(const volatile T *)p;
}

// ---- grid-strided bin ------------------------------------------------------
// Vertices with at least GRID_TH edges are too big for one CTA: the tile pass
// defers them to a list, and a second kernel spreads their concatenated edges
// evenly over every CTA of the grid.
constexpr int GRID_TH = 4096;
#ifndef MG_DEFER_WARP
#define MG_DEFER_WARP 1
#endif
constexpr int BIG_CAP = 4096;  // deferred vertices per level (more fall back to the CTA bin)

struct BigList {
  int32_t *v;            // deferred vertices
  int32_t *len;          // their count (reset at the end of every level)
  int32_t th = GRID_TH;  // out-degree at or above which a vertex is deferred
};

// Deferral threshold for a frontier of nin vertices expanded by this grid. When
// the frontier fills fewer tiles than there are CTAs, the CTA bin would leave
// most CTAs idle while a few walk heavy rows alone (a few hundred hubs of
// thousands of edges each), so every vertex the CTA bin would take goes to the
// grid-wide pass instead; when it fills under an eighth of them, so does every
// vertex the warp bin would take (32 edges or more). R-MAT s22 BFS, mean of 13
// sources: 0.54 ms with the CTA-bin rule alone, 0.42 ms with both.
//
// grid_th and defer_warp (the warp-bin rule on or off) default to GRID_TH and
// MG_DEFER_WARP; callers with tuned values pass them at run time.
template <int NT>
__device__ __forceinline__ int32_t defer_threshold(int64_t nin, int32_t cta_th, int32_t grid_th = GRID_TH,
                                                   int32_t defer_warp = MG_DEFER_WARP) {
  if (defer_warp && nin * 8 < (int64_t)gridDim.x * NT) return 32;
  return nin < (int64_t)gridDim.x * NT ? cta_th : grid_th;
}

// Returns true (and records v) when v goes to the grid bin.
__device__ __forceinline__ bool defer_big(const BigList &big, int32_t v, int32_t deg) {
  if (v < 0 || deg < big.th) return false;
  const int32_t pos = atomicAdd(big.len, 1);
  if (pos >= BIG_CAP) return false;
  big.v[pos] = v;
  return true;
}

template <int NT>
struct BigSmem {
  int32_t v[BIG_CAP];
  int32_t pre[BIG_CAP + 1];
  int32_t red[NT / 32 + 1];
};

// Every CTA takes an equal slice of the concatenated edges of the deferred
// vertices; an edge slot finds its vertex by binary search over their prefix sums.
template <int NT, typename Visit>
__device__ __forceinline__ void expand_big(BigSmem<NT> &sm, const int32_t *__restrict__ off, const BigList &big,
                                           Visit &&visit, int32_t vmask = -1) {
  const int32_t nb = min(*(const volatile int32_t *)big.len, BIG_CAP);
  if (nb == 0) return;
  // Degrees and their exclusive prefix, NT * ceil(nb / NT) at a time.
  int32_t carry = 0;
  for (int32_t b0 = 0; b0 < nb; b0 += NT) {
    const int32_t i = b0 + threadIdx.x;
    int32_t d = 0;
    if (i < nb) {
      const int32_t v = big.v[i];
      sm.v[i] = v;
      d = off[(v & vmask) + 1] - off[v & vmask];
    }
    int32_t tot;
    const int32_t ex = block_exclusive_scan<NT>(d, sm.red, &tot);
    if (i < nb) sm.pre[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sm.pre[nb] = carry;
  __syncthreads();
  const int64_t total = carry;
  const int64_t lo = total * blockIdx.x / gridDim.x, hi = total * (blockIdx.x + 1) / gridDim.x;
  for (int64_t k = lo + threadIdx.x; k < hi; k += NT) {
    int a = 0, b = nb;
    while (b - a > 1) {
      const int mid = (a + b) >> 1;
      if (sm.pre[mid] <= k) a = mid;
      else b = mid;
    }
    const int32_t v = sm.v[a];
    visit(v, off[v & vmask] + (int32_t)(k - sm.pre[a]));
  }
  __syncthreads();
}

}  // namespace mg
