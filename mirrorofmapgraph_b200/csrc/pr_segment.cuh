// pr_segment.cuh -- column-segmented gather of the high-degree rows (PageRank's
// "segmented" gather, mg_pr_opts.gather_kernel = 3). The reference's gather this
// replaces is gather_mgpu / kernel_gather_mgpu
// (GASengine/enactor_vertex_centric.cuh:1285-1879, mgpukernel/kernel.cuh:215-339).
//
// Why: a random 4-byte gather from global memory costs one L1 wavefront per
// distinct 32-byte sector and an SM retires about one such wavefront per clock, so
// the binned gather is held near one gathered edge per clock per SM however many
// loads are in flight (measured on B200: 0.98 random global gathers per clock per
// SM against 7.6 from shared memory, where only bank conflicts serialise). This
// gather moves most random gathers into shared memory:
//
//  - Rows of at least T edges (the plan's hubs) are cut by column block: block j
//    holds columns [j*S, (j+1)*S), S chosen so x/s[block] fits in one CTA's
//    shared memory. A hub row's edges are stored grouped by block (a stable
//    reorder of the row), so its edges in block j form one contiguous fragment,
//    split further at SEG_FMAX edges. Phase 1 of an iteration walks fragments
//    block by block: the CTA copies x/s[block] into shared memory with TMA bulk
//    copies (cp.async.bulk, completion on an mbarrier, bounded waits) and each
//    lane of its warps reduces one fragment from there. A fragment's compensated
//    sum goes to a fixed slot.
//  - Phase 2, the next kernel: one warp per hub row adds the row's fragment sums
//    in a fixed order (lanes strided, then a fixed pairing tree) and applies the
//    row update. Every row below T (zero-degree rows included) is laid out as
//    sliced ELL too: rows sorted by degree, longest first, 32 to a group, a lane
//    per row, index loads one round ahead of the gathers, so no warp walks rows
//    one after another behind dependent loads. Its gathers take the most-gathered
//    columns from a shared-memory cache and the rest from global memory. Groups go
//    to warps from a counter; the last CTA ends the iteration. During a segmented
//    solve the iterate x, the row sums and the teleport entries are kept in phase
//    2's lane order, so the row updates read and write them with coalesced
//    accesses. Results do not depend on scheduling.
//
// Bank spreading: a block load copies x/s[block] into shared memory as it lies
// in global memory, so a column's bank is its position mod 32. R-MAT-like graphs
// favour ids with zero low bits (about a quarter of the edges of an R-MAT graph
// land on columns that are multiples of 32), which would pile the gathers of a
// warp onto a few banks. The segmented solver therefore stores the gathered vector
// x/s with vertex c at position seg_swz(c): the low five bits XORed with a
// multiplicative hash of the 32-vertex chunk index. The map permutes every 32-entry
// chunk, so blocks (multiples of 32 wide) keep their vertices; the plan stores
// permuted positions in its index arrays, and the rows' updates write x/s there.
//
// Phase 1 stores the hub fragments as sliced ELL: the fragments of a block, sorted
// by length (longest first), form groups of 32; a group's indices are laid out
// column-major (entry i of lane l at 32*i + l, -1 past a fragment's end), so lane l
// walks fragment l with one coalesced 128-byte load per step and no per-fragment
// reduction. Sorting by length keeps the padding small. Phase 1's groups are cut
// into one contiguous range per CTA by estimated cost, so a CTA loads only the few
// blocks its range spans.
#pragma once

#include "common.cuh"
#include "pr_binned.cuh"
#include "pr_gather.cuh"

namespace mg {

constexpr int32_t SEG_FMAX = 256;       // longest fragment (longer runs are split)
constexpr int32_t SEG_MAXB = 8192;      // most column blocks a plan supports
constexpr uint32_t SEG_COPY = 32768;    // bytes per bulk copy of a block load
// Scheduling costs of phase 1, in sliced-ELL entries: a group's fixed cost (its
// entry loads, partial stores, fence and arrival atomics), a block load, and the
// factor of a global gather over a shared-memory one. A block is staged in shared
// memory when it holds at least SEG_DENSE entries; the groups of sparser blocks
// gather straight from global memory (a block load would cost more than it saves).
// With 16-bit indices a shared-memory step costs less next to a global gather:
// factor 6 balanced the CTAs best (R-MAT s22: 300.5 us per iteration against
// 305.0-305.5 with 4, 300.9-301.3 with 8; group costs 256 and 1024 were slower).
constexpr int64_t SEG_GROUP_COST = 512;
constexpr int64_t SEG_LOAD_COST = 65536;
constexpr int64_t SEG_GLOBAL_FACTOR = 6;
constexpr int64_t SEG_DENSE = 131072;
#ifndef SEG_U
#define SEG_U 8                         // ELL steps a lane loads before its first add
#endif

__host__ __device__ __forceinline__ int32_t seg_swz(int32_t c) {
  const uint32_t k = (uint32_t)c >> 5;
  return (int32_t)(((uint32_t)c & ~31u) | (((uint32_t)c ^ ((k * 0x9E3779B1u) >> 27)) & 31u));
}

// Plan of the forward (CSC) gather, built once per graph and (T, S).
struct SegPlan {
  int32_t T = 0, S = 0, nblocks = 0, grid = 0;
  BinPlan bins;              // rows below T in bins 0..5; rows of >= T edges are its hubs;
                             // hbase / hpart count fragments instead of fixed chunks
  int32_t *sidx = nullptr;   // m + 8 indices: rows below T with cached columns as
                             // (slot | 0x80000000); hub rows block-grouped (plan scratch)
  float *swts = nullptr;     // edge weights in sidx's order (weighted graphs)
  int2 *ent = nullptr;       // {fragment id, hub} of every group lane ({-1, -1}: empty lane)
  int64_t *gofs = nullptr;   // first sliced-ELL entry of each group, ngroups + 1 entries
  uint16_t *pidx = nullptr;  // sliced-ELL column offsets of the hub fragments within their block, two
                             // steps of a lane per 32-bit word (seg_pk; 0xFFFF: padding)
  float *pwts = nullptr;     // their edge weights (weighted graphs)
  int32_t *bgrp = nullptr;   // first group of each block, nblocks + 1 entries
  uint8_t *bdense = nullptr; // 1: the block is staged in shared memory; 0: gathered from global
  int32_t *cta = nullptr;    // first group of each CTA, grid + 1 entries
  int64_t ngroups = 0, nfrag = 0, nell = 0;
  // phase 2: the rows below T as sliced ELL (entries from sidx, -1 past a row's end)
  int32_t *rrow = nullptr;   // row of every group lane (-1: empty lane), nrgroups * 32
  int64_t *rgofs = nullptr;  // first entry of each group, nrgroups + 1
  int32_t *ridx = nullptr;   // column entries
  float *rwts = nullptr;     // their weights (weighted graphs)
  int32_t *rgrab = nullptr;  // group counter of phase 2 (zero between launches)
  int64_t nrgroups = 0, nrell = 0;
  int64_t nrgroups_e = 0;    // groups holding an edge (the rest, last in the order, hold rows without edges)
  int64_t nrgroups_l = 0;    // groups deeper than SEG_SHORT (the first ones in the order)
  // Positions of the iterate during a segmented solve: g * 32 + l for phase 2's
  // group g, lane l, then nrgroups * 32 + h for hub h. Per position: its row (-1
  // for empty lanes) and the row's cached-column slot.
  int32_t *ppos = nullptr;   // position of every row, n entries
  int32_t *prow = nullptr;   // row of every position, npos entries
  int32_t *pslot = nullptr;  // column-cache slot of every position (-1: not cached)
  int64_t npos = 0;
  bool weighted = false;
  bool ok = false;
};

struct SegArgs {
  const int2 *ent;
  const int64_t *gofs;
  const uint16_t *pidx;
  const float *pwts;
  const int32_t *bgrp, *cta;
  const uint8_t *bdense;
  int64_t n32;  // vertices rounded up to whole 32-entry chunks (the permuted x/s extent)
  int32_t S, nblocks;
  const int32_t *rrow;
  const int64_t *rgofs;
  const int32_t *ridx;
  const float *rwts;
  int32_t *rgrab;
  int64_t nrgroups;
  int64_t nrgroups_e;    // groups with an edge; positions from nrgroups_e * 32 on are rows without one
  int64_t nrgroups_l;    // groups deeper than SEG_SHORT; [nrgroups_l, nrgroups_e) are short
  const int32_t *pslot;  // per position: cached-column slot
  const float *ps;       // per position: row sum s (0: dangling), filled per solve
  const float *pt;       // per position: teleport entry (nullptr: uniform), filled per solve
};

#ifndef MG_PRB_NO_PLAN_KERNELS  // plan building runs in pagerank.cu only
// Per hub row: edges per column block (shared-memory histogram), the row's
// fragment count, and per block the number of fragments of every length
// (lencnt[block * SEG_FMAX + SEG_FMAX - len], so ascending keys list longer first).
__global__ void __launch_bounds__(256) seg_hist_kernel(const int32_t *__restrict__ off, const int32_t *__restrict__ idx,
                                                       const int32_t *__restrict__ hrows, int32_t S, int32_t B,
                                                       int32_t *__restrict__ nfr, int32_t *__restrict__ lencnt) {
  extern __shared__ int32_t sh[];
  __shared__ int32_t red[256 / 32 + 1];
  const int32_t r = hrows[blockIdx.x];
  const int32_t b0 = off[r], b1 = off[r + 1];
  for (int i = threadIdx.x; i < B; i += 256) sh[i] = 0;
  __syncthreads();
  for (int32_t k = b0 + threadIdx.x; k < b1; k += 256) atomicAdd(sh + idx[k] / S, 1);
  __syncthreads();
  int32_t nf = 0;
  for (int i = threadIdx.x; i < B; i += 256) {
    const int32_t c = sh[i];
    if (c == 0) continue;
    const int32_t full = (c - 1) / SEG_FMAX;  // fragments of SEG_FMAX edges before the last
    nf += full + 1;
    if (full) atomicAdd(lencnt + (int64_t)i * SEG_FMAX, full);
    atomicAdd(lencnt + (int64_t)i * SEG_FMAX + SEG_FMAX - (c - full * SEG_FMAX), 1);
  }
  int32_t tot;
  block_exclusive_scan<256>(nf, red, &tot);
  if (threadIdx.x == 0) nfr[blockIdx.x] = tot;
}

// Exclusive scan of `in` (n entries) into out[0..n], one CTA.
__global__ void __launch_bounds__(256) seg_scan_kernel(const int32_t *__restrict__ in, int64_t n, int32_t *out) {
  __shared__ int32_t red[256 / 32 + 1];
  int32_t carry = 0;
  for (int64_t b0 = 0; b0 < n; b0 += 256) {
    const int64_t i = b0 + threadIdx.x;
    const int32_t v = i < n ? in[i] : 0;
    int32_t tot;
    const int32_t ex = block_exclusive_scan<256>(v, red, &tot);
    if (i < n) out[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// One warp per hub row: reorders the row's edges by block (stable: the edges of
// one block keep their order) into sidx / swts, numbers the row's fragments in
// block order, and gives each fragment its slot in its block's length-sorted list
// (slot cursors per (block, length) key): {fragment id, hub} in ent, and the
// fragment's first reordered edge and length in fsrc / flen.
__global__ void __launch_bounds__(32) seg_fill_kernel(const int32_t *__restrict__ off, const int32_t *__restrict__ idx,
                                                      const float *__restrict__ wts, const int32_t *__restrict__ hrows,
                                                      const int32_t *__restrict__ hbase, int32_t S, int32_t B,
                                                      int32_t *__restrict__ cursor, int32_t *__restrict__ sidx,
                                                      float *__restrict__ swts, int2 *__restrict__ ent,
                                                      int32_t *__restrict__ fsrc, int32_t *__restrict__ flen) {
  extern __shared__ int32_t cur[];
  const int lane = threadIdx.x;
  const int32_t h = blockIdx.x;
  const int32_t r = hrows[h];
  const int32_t o0 = off[r], o1 = off[r + 1];
  for (int i = lane; i < B; i += 32) cur[i] = 0;
  __syncwarp();
  for (int32_t k = o0 + lane; k < o1; k += 32) atomicAdd(cur + idx[k] / S, 1);
  __syncwarp();
  // lane l owns blocks [lo, hi): its edge and fragment totals, then warp prefixes
  const int32_t per = (B + 31) / 32;
  const int32_t lo = min(B, lane * per), hi = min(B, lo + per);
  int32_t esum = 0, fsum = 0;
  for (int32_t i = lo; i < hi; i++) {
    const int32_t c = cur[i];
    esum += c;
    fsum += c ? (c + SEG_FMAX - 1) / SEG_FMAX : 0;
  }
  int32_t e = warp_inclusive_scan(esum) - esum;
  int32_t f = hbase[h] + warp_inclusive_scan(fsum) - fsum;
  __syncwarp();
  for (int32_t i = lo; i < hi; i++) {
    const int32_t c = cur[i];
    cur[i] = e;  // first position of block i in the reordered row
    for (int32_t q = 0; q < c; q += SEG_FMAX) {
      const int32_t len = min(SEG_FMAX, c - q);
      const int32_t slot = atomicAdd(cursor + (int64_t)i * SEG_FMAX + SEG_FMAX - len, 1);
      ent[slot] = make_int2(f, h);
      fsrc[slot] = o0 + e + q;
      flen[slot] = len;
      f++;
    }
    e += c;
  }
  __syncwarp();
  for (int32_t base = o0; base < o1; base += 32) {
    const int32_t k = base + lane;
    const bool valid = k < o1;
    const int32_t c = valid ? idx[k] : 0;
    const int32_t b = valid ? c / S : -1 - lane;
    const unsigned peers = __match_any_sync(FULL, b);
    const int32_t rank = __popc(peers & lanemask_lt());
    if (valid) {
      const int32_t pos = cur[b] + rank;
      sidx[o0 + pos] = c;
      if (swts) swts[o0 + pos] = wts[k];
    }
    __syncwarp();
    if (valid && rank == 0) cur[b] += __popc(peers);
    __syncwarp();
  }
}

// Sliced-ELL layout: one warp per group copies lane l's fragment (fsrc, flen) into
// entries gofs[g] + 32 i + l, as permuted x/s positions (seg_swz). Padding entries
// keep the -1 they were cleared to.
// Entry of step i of lane `lane` in a group whose entries start at g0 (even): the
// 16-bit column offsets of a lane's steps 2p and 2p + 1 share one 32-bit word, the
// 32 lanes' words of a step pair are consecutive.
__host__ __device__ __forceinline__ int64_t seg_pk(int64_t g0, int lane, int64_t i) {
  return g0 + 64 * (i >> 1) + 2 * lane + (i & 1);
}

__global__ void __launch_bounds__(256) seg_sell_kernel(const int2 *__restrict__ ent, const int32_t *__restrict__ fsrc,
                                                       const int32_t *__restrict__ flen,
                                                       const int64_t *__restrict__ gofs, int64_t ngroups,
                                                       const int32_t *__restrict__ sidx, const float *__restrict__ swts,
                                                       int32_t S, uint16_t *__restrict__ pidx,
                                                       float *__restrict__ pwts) {
  const int lane = threadIdx.x & 31;
  for (int64_t gi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < ngroups;
       gi += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t slot = gi * 32 + lane;
    if (ent[slot].x < 0) continue;
    const int32_t src = fsrc[slot], len = flen[slot];
    const int64_t g0 = gofs[gi], o = g0 + lane;
    for (int32_t i = 0; i < len; i++) {
      pidx[seg_pk(g0, lane, i)] = (uint16_t)(seg_swz(sidx[src + i]) % S);  // a fragment lies in one block
      if (pwts) pwts[o + 32 * (int64_t)i] = swts[src + i];
    }
  }
}
// Phase 2's sliced ELL: one warp per group copies lane l's row (sidx / swts over
// the row's edges, in edge order) into entries rgofs[g] + 32 i + l.
__global__ void __launch_bounds__(256) seg_rows_fill_kernel(const int32_t *__restrict__ rrow,
                                                            const int64_t *__restrict__ rgofs, int64_t ngroups,
                                                            const int32_t *__restrict__ off,
                                                            const int32_t *__restrict__ sidx,
                                                            const float *__restrict__ swts, int32_t *__restrict__ ridx,
                                                            float *__restrict__ rwts) {
  const int lane = threadIdx.x & 31;
  for (int64_t gi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < ngroups;
       gi += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int32_t r = rrow[gi * 32 + lane];
    if (r < 0) continue;
    const int32_t b = off[r], d = off[r + 1] - b;
    const int64_t o = rgofs[gi] + lane;
    for (int32_t i = 0; i < d; i++) {
      ridx[o + 32 * (int64_t)i] = sidx[b + i];
      if (rwts) rwts[o + 32 * (int64_t)i] = swts[b + i];
    }
  }
}

// Cached-column slot of every iterate position, and the position of every row
// (ppos, the inverse of prow; rows without a position keep the -1 it was set to).
__global__ void seg_pos_slot_kernel(const int32_t *__restrict__ prow, int64_t npos, const int32_t *__restrict__ slot,
                                    int32_t *__restrict__ pslot, int32_t *__restrict__ ppos) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npos; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = prow[i];
    pslot[i] = r >= 0 ? slot[r] : -1;
    if (r >= 0) ppos[r] = (int32_t)i;
  }
}
#endif  // MG_PRB_NO_PLAN_KERNELS

// One lane's row of a sliced-ELL group (a phase-1 fragment or a phase-2 row):
// `depth` steps from q (qw), index loads one round of U steps ahead of the
// gathers; -1 entries are padding.
template <bool WEIGHTED, int U, typename Gather>
__device__ __forceinline__ Comp sell_walk(const int32_t *q, const float *qw, int32_t depth, Gather &gather) {
  Comp acc{0.f, 0.f};
  int32_t c[U];
  float w[U];
#pragma unroll
  for (int j = 0; j < U; j++) {
    c[j] = j < depth ? prb_stream(q + 32 * j) : -1;
    w[j] = (WEIGHTED && j < depth) ? prb_stream(qw + 32 * j) : 0.f;
  }
  for (int32_t i = 0; i < depth; i += U) {
    int32_t cn[U];
    float wn[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      const int32_t k = i + U + j;
      cn[j] = k < depth ? prb_stream(q + 32 * k) : -1;
      wn[j] = (WEIGHTED && k < depth) ? prb_stream(qw + 32 * k) : 0.f;
    }
    float v[U];
#pragma unroll
    for (int j = 0; j < U; j++) v[j] = c[j] != -1 ? gather(c[j]) : 0.f;
#pragma unroll
    for (int j = 0; j < U; j++) {
      if (c[j] == -1) continue;
      if (WEIGHTED) {
        const float p = w[j] * v[j];
        two_sum_add(acc, p);
        acc.lo += __fmaf_rn(w[j], v[j], -p);
      } else {
        two_sum_add(acc, v[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      c[j] = cn[j];
      w[j] = wn[j];
    }
  }
  return acc;
}

// One lane's hub fragment (phase 1): `depth` (even) steps of 16-bit block offsets,
// two per 32-bit word at q + 32 p (seg_pk), weights (weighted graphs) one per step
// at qw + 32 i; index words loaded one round of U steps ahead of the gathers, the
// sum taken in step order like sell_walk's. 0xFFFF entries are padding.
template <bool WEIGHTED, int U, typename Gather>
__device__ __forceinline__ Comp sell_walk16(const uint32_t *q, const float *qw, int32_t depth, Gather &gather) {
  static_assert(U % 2 == 0, "two steps per index word");
  Comp acc{0.f, 0.f};
  uint32_t c[U / 2];
  float w[U];
#pragma unroll
  for (int p = 0; p < U / 2; p++) c[p] = 2 * p < depth ? prb_stream(q + 32 * p) : 0xffffffffu;
#pragma unroll
  for (int j = 0; j < U; j++) w[j] = (WEIGHTED && j < depth) ? prb_stream(qw + 32 * j) : 0.f;
  for (int32_t i = 0; i < depth; i += U) {
    uint32_t cn[U / 2];
    float wn[U];
#pragma unroll
    for (int p = 0; p < U / 2; p++) {
      const int32_t k = i + U + 2 * p;
      cn[p] = k < depth ? prb_stream(q + 32 * (k >> 1)) : 0xffffffffu;
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      const int32_t k = i + U + j;
      wn[j] = (WEIGHTED && k < depth) ? prb_stream(qw + 32 * k) : 0.f;
    }
    float v[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      const uint32_t off = (c[j >> 1] >> (16 * (j & 1))) & 0xffffu;
      v[j] = off != 0xffffu ? gather((int32_t)off) : 0.f;
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      if (((c[j >> 1] >> (16 * (j & 1))) & 0xffffu) == 0xffffu) continue;
      if (WEIGHTED) {
        const float pr = w[j] * v[j];
        two_sum_add(acc, pr);
        acc.lo += __fmaf_rn(w[j], v[j], -pr);
      } else {
        two_sum_add(acc, v[j]);
      }
    }
#pragma unroll
    for (int p = 0; p < U / 2; p++) c[p] = cn[p];
#pragma unroll
    for (int j = 0; j < U; j++) w[j] = wn[j];
  }
  return acc;
}

// Two short rows (depth <= SEG_SHORT each, sliced-ELL layout as in sell_walk) of
// two groups walked together: both rows' index loads, then both rows' gathers,
// then the sums, each row's in the order sell_walk adds them (so the results are
// the same bits).
constexpr int SEG_SHORT = 4;
template <bool WEIGHTED, typename Gather>
__device__ __forceinline__ void sell_short2(const int32_t *qa, const float *qwa, int32_t da, const int32_t *qb,
                                            const float *qwb, int32_t db, Gather &gather, Comp &acc_a, Comp &acc_b) {
  int32_t ca[SEG_SHORT], cb[SEG_SHORT];
  float wa[SEG_SHORT], wb[SEG_SHORT], va[SEG_SHORT], vb[SEG_SHORT];
#pragma unroll
  for (int j = 0; j < SEG_SHORT; j++) {
    ca[j] = j < da ? prb_stream(qa + 32 * j) : -1;
    cb[j] = j < db ? prb_stream(qb + 32 * j) : -1;
    wa[j] = (WEIGHTED && j < da) ? prb_stream(qwa + 32 * j) : 0.f;
    wb[j] = (WEIGHTED && j < db) ? prb_stream(qwb + 32 * j) : 0.f;
  }
#pragma unroll
  for (int j = 0; j < SEG_SHORT; j++) {
    va[j] = ca[j] != -1 ? gather(ca[j]) : 0.f;
    vb[j] = cb[j] != -1 ? gather(cb[j]) : 0.f;
  }
  acc_a = Comp{0.f, 0.f};
  acc_b = Comp{0.f, 0.f};
#pragma unroll
  for (int j = 0; j < SEG_SHORT; j++) {
    if (ca[j] != -1) {
      if (WEIGHTED) {
        const float p = wa[j] * va[j];
        two_sum_add(acc_a, p);
        acc_a.lo += __fmaf_rn(wa[j], va[j], -p);
      } else {
        two_sum_add(acc_a, va[j]);
      }
    }
    if (cb[j] != -1) {
      if (WEIGHTED) {
        const float p = wb[j] * vb[j];
        two_sum_add(acc_b, p);
        acc_b.lo += __fmaf_rn(wb[j], vb[j], -p);
      } else {
        two_sum_add(acc_b, vb[j]);
      }
    }
  }
}

// Phase 1 of a segmented iteration on one CTA: walks the CTA's groups block by
// block, staging x/s[block] (gathered values `gold`) in `sbuf` with bulk copies;
// lane l of a group reduces fragment l and hands its sum to fin(entry, sum)
// (empty lanes pass entry.x < 0). Every thread of
// the CTA calls it. Warps take a segment's groups from a shared counter; each
// segment uses the other of two counters (s_next[2]) and ends with a CTA barrier,
// so no warp can still draw from a counter that is being reset for the next
// segment. `phase` is the mbarrier's next parity; `ok` turns false if a bounded
// wait ran out.
template <bool WEIGHTED, typename Finish>
__device__ __forceinline__ void seg_phase(const SegArgs &sg, const float *gold, float *sbuf, uint64_t *bar,
                                          int32_t *s_next, uint32_t &phase, bool &ok, Finish &fin) {
  const int lane = threadIdx.x & 31;
  const int64_t g0 = sg.cta[blockIdx.x], g1 = sg.cta[blockIdx.x + 1];
  if (g0 >= g1) return;
  int32_t lo = 0, hi = sg.nblocks;  // block j of group g0: bgrp[j] <= g0 < bgrp[j + 1]
  while (hi - lo > 1) {
    const int32_t mid = (lo + hi) >> 1;
    if (sg.bgrp[mid] <= g0) lo = mid;
    else hi = mid;
  }
  int32_t j = lo;
  int seg = 0;
  for (int64_t gs = g0; gs < g1 && j < sg.nblocks; j++) {
    const int64_t ge = min(g1, (int64_t)sg.bgrp[j + 1]);
    if (ge <= gs) continue;
    const int64_t c_lo = (int64_t)j * sg.S;
    const bool dense = sg.bdense[j] != 0;
    int32_t *next = s_next + (seg & 1);
    __syncthreads();  // every warp is done with the previous block
    if (threadIdx.x == 0) {
      *next = (int32_t)gs;
      if (dense) {
        const int64_t cnt = min((int64_t)sg.S, sg.n32 - c_lo);
        const uint32_t bytes = (uint32_t)((cnt * 4 + 15) & ~(int64_t)15);  // gathered arrays are padded
        fence_proxy_async();
        mbar_arrive_expect_tx(bar, bytes);
        for (uint32_t o = 0; o < bytes; o += SEG_COPY)
          bulk_g2s(reinterpret_cast<char *>(sbuf) + o, reinterpret_cast<const char *>(gold + c_lo) + o,
                   min(SEG_COPY, bytes - o), bar);
      }
    }
    __syncthreads();
    if (dense) {
      if (!mbar_wait_bounded(bar, phase)) {
        ok = false;
        mbar_wait_bounded(bar, phase);  // once more, for the copy still in flight
      }
      phase ^= 1;
    }
    const float *gblk = gold + c_lo;
    auto from_smem = [&](int32_t off) { return sbuf[off]; };
    auto from_global = [&](int32_t off) { return __ldg(gblk + off); };
    for (;;) {
      int32_t gi = 0;
      if (lane == 0) gi = atomicAdd(next, 1);
      gi = __shfl_sync(FULL, gi, 0);
      if (gi >= ge) break;
      const int2 e = sg.ent[(int64_t)gi * 32 + lane];
      const int64_t s0 = sg.gofs[gi];
      const int32_t steps = (int32_t)((sg.gofs[gi + 1] - s0) >> 5);
      const uint32_t *q = reinterpret_cast<const uint32_t *>(sg.pidx + s0) + lane;
      const float *qw = WEIGHTED ? sg.pwts + s0 + lane : nullptr;
      constexpr int U = WEIGHTED ? 4 : SEG_U;
      const Comp acc = dense ? sell_walk16<WEIGHTED, U>(q, qw, steps, from_smem)
                             : sell_walk16<WEIGHTED, U>(q, qw, steps, from_global);
      fin(e, acc);
    }
    __syncthreads();  // the segment ends for every warp at once
    seg++;
    gs = ge;
  }
}

}  // namespace mg
