// common.cuh -- device helpers shared by the engine's kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "mg_internal.h"

namespace mg {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(FULL, v, o);
    if (l >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan for blockDim.x == NT (multiple of 32, <= 1024).
// `smem` must hold NT/32 + 1 elements. Returns the exclusive prefix; *total gets the sum.
template <int NT, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *smem, T *total) {
  const int l = lane_id(), w = warp_id();
  T inc = warp_inclusive_scan(v);
  if (l == 31) smem[w] = inc;
  __syncthreads();
  if (w == 0) {
    T s = l < NT / 32 ? smem[l] : T(0);
    T si = warp_inclusive_scan(s);
    if (l < NT / 32) smem[l] = si - s;
    if (l == NT / 32 - 1) smem[NT / 32] = si;
  }
  __syncthreads();
  T r = smem[w] + inc - v;
  *total = smem[NT / 32];
  __syncthreads();
  return r;
}

template <int NT, typename T>
__device__ __forceinline__ T block_sum(T v, T *smem) {
  const int l = lane_id(), w = warp_id();
  v = warp_sum(v);
  if (l == 0) smem[w] = v;
  __syncthreads();
  T r = T(0);
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; i++) r += smem[i];
  }
  __syncthreads();
  return r;  // valid in thread 0 only
}

// Last-block-done election: every CTA calls this once after finishing its work
// (all threads). Returns true in every thread of the last CTA to arrive. Writes
// made by any CTA before its call are visible to the last CTA afterwards.
__device__ __forceinline__ bool last_block(unsigned *counter) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// Grid-wide barrier for kernels whose blocks are all resident (cooperative
// launch): arrivals are counted in *count and the last block bumps *gen. The
// wait is bounded: after `limit` polls the block gives up and the function
// returns false (the caller reports MG_ERR_TIMEOUT and stops), so a missing
// block cannot hang the GPU. Every thread of every block must call it.
// `extra` raises the number of arrivals the barrier waits for (a test hook: a
// barrier that cannot complete, to check that the bounded wait reports
// MG_ERR_TIMEOUT); 0 in normal runs.
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *gen, unsigned long long limit,
                                             unsigned extra = 0) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = *(volatile unsigned *)gen;  // read before arriving: gen moves only after every arrival
    __threadfence();
    int ok = 1;
    if (atomicAdd(count, 1u) + 1 == gridDim.x + extra) {
      *count = 0;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      unsigned long long it = 0;
      while (*(volatile unsigned *)gen == g) {
        if (++it > limit) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Warp-aggregated append of `item` to `queue` (capacity `cap`) for every active
// lane with `pred` set; the queue length lives at *len. Lanes whose slot lands
// past the capacity set *overflow instead of writing.
__device__ __forceinline__ void warp_append(bool pred, int32_t item, int32_t *queue, int32_t *len,
                                            int32_t cap, int32_t *overflow) {
  const unsigned active = __activemask();
  const unsigned pm = __ballot_sync(active, pred);
  if (pm == 0) return;
  const int leader = __ffs(active) - 1;
  int base = 0;
  if (lane_id() == leader) base = atomicAdd(len, __popc(pm));
  base = __shfl_sync(active, base, leader);
  if (pred) {
    int pos = base + __popc(pm & lanemask_lt());
    if (pos < cap) queue[pos] = item;
    else *overflow = 1;
  }
}

// Block-local staging of the vertices a level adds to a frontier queue: threads
// take slots with a shared-memory atomic and the block appends its whole batch to
// the queue with one global atomic when it flushes. With one global atomic per
// warp instead, a level that adds ~10^6 vertices serialises on the queue's length
// word (R-MAT s22 BFS: a 6.1 M-edge push level took 510 us).
constexpr int BQ_CAP = 2048;
struct BlockQueue {
  int32_t n;
  int32_t base;
  int32_t v[BQ_CAP];
};

__device__ __forceinline__ void bq_init(BlockQueue &bq) {
  if (threadIdx.x == 0) bq.n = 0;
  __syncthreads();
}

// Every thread of the block calls it (it synchronises the block).
__device__ __forceinline__ void bq_flush(BlockQueue &bq, int32_t *qout, int32_t *qlen, int32_t cap,
                                         int32_t *overflow) {
  __syncthreads();
  const int32_t n = min(bq.n, BQ_CAP);
  if (threadIdx.x == 0) bq.base = n ? atomicAdd(qlen, n) : 0;
  __syncthreads();
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int32_t pos = bq.base + i;
    if (pos < cap) qout[pos] = bq.v[i];
    else *overflow = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) bq.n = 0;
  __syncthreads();
}

// Appends item (where pred) through the staging area, or straight to the queue
// when there is none or it is full. One shared-memory atomic per warp, like
// warp_append's one global atomic per warp.
__device__ __forceinline__ void staged_append(BlockQueue *bq, bool pred, int32_t item, int32_t *queue, int32_t *len,
                                              int32_t cap, int32_t *overflow) {
  if (!bq) {
    warp_append(pred, item, queue, len, cap, overflow);
    return;
  }
  const unsigned active = __activemask();
  const unsigned pm = __ballot_sync(active, pred);
  if (pm == 0) return;
  const int leader = __ffs(active) - 1;
  int32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(&bq->n, __popc(pm));
  base = __shfl_sync(active, base, leader);
  bool spill = false;
  if (pred) {
    const int32_t pos = base + __popc(pm & lanemask_lt());
    if (pos < BQ_CAP) bq->v[pos] = item;
    else spill = true;
  }
  warp_append(spill, item, queue, len, cap, overflow);
}

__device__ __forceinline__ int32_t ld_nc(const int32_t *p) { return __ldg(p); }

// Reductions whose old value nobody waits for (PTX red): the issuing warp does
// not stall on them, unlike atomics whose result is used.
__device__ __forceinline__ void red_min(int32_t *p, int32_t v) {
  asm volatile("red.relaxed.gpu.global.min.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_or(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace mg
