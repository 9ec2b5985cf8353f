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

template <int NT>
struct ExpandSmem {
  int32_t scan[NT];
  int32_t beg[NT];
  int32_t vtx[NT];
  int32_t red[NT / 32 + 1];
  int32_t cta[4];
};

template <int NT, int CTA_TH, typename Visit>
__device__ __forceinline__ void expand_tile(ExpandSmem<NT> &sm, const int32_t *__restrict__ off, int32_t v,
                                            int64_t &insp, Visit &&visit) {
  const int tid = threadIdx.x, lane = lane_id();
  int32_t beg = 0, deg = 0;
  if (v >= 0) {
    beg = off[v];
    deg = off[v + 1] - beg;
    insp += deg;
  }
  // CTA bin.
  while (__syncthreads_or(deg >= CTA_TH)) {
    if (deg >= CTA_TH) sm.cta[0] = tid;
    __syncthreads();
    if (sm.cta[0] == tid) {
      sm.cta[1] = beg;
      sm.cta[2] = beg + deg;
      sm.cta[3] = v;
      deg = 0;
    }
    __syncthreads();
    const int32_t b = sm.cta[1], e = sm.cta[2], cv = sm.cta[3];
    for (int32_t k = b + tid; k < e; k += NT) visit(cv, k);
  }
  // Warp bin.
  for (;;) {
    const unsigned wm = __ballot_sync(FULL, deg >= 32);
    if (!wm) break;
    const int l = __ffs(wm) - 1;
    const int32_t b = __shfl_sync(FULL, beg, l), e = __shfl_sync(FULL, beg + deg, l);
    const int32_t wv = __shfl_sync(FULL, v, l);
    if (lane == l) deg = 0;
    for (int32_t k = b + lane; k < e; k += 32) visit(wv, k);
  }
  // Thread bin.
  int32_t total;
  const int32_t ex = block_exclusive_scan<NT>(deg, sm.red, &total);
  sm.scan[tid] = ex;
  sm.beg[tid] = beg;
  sm.vtx[tid] = v;
  __syncthreads();
  for (int32_t k = tid; k < total; k += NT) {
    int lo = 0, hi = NT;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (sm.scan[mid] <= k) lo = mid;
      else hi = mid;
    }
    visit(sm.vtx[lo], sm.beg[lo] + (k - sm.scan[lo]));
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ T vload(const T *p) {
  return *(const volatile T *)p;
}

}  // namespace mg
