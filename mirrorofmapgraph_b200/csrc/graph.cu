// graph.cu -- device graph storage: upload, validation and the CSC build.
//
// Replaces CsrProblem::FromHostProblem (GASengine/csr_problem.cuh:401-621) and
// its thrust CSC build (util.cuh:55-126). Layout in HBM, all int32:
//   CSR  row_offsets[n+1], col_idx[m], values[m] (int32 or float)
//   CSC  col_offsets[n+1], row_idx[m], perm[m] (CSC slot -> CSR edge id),
//        cvals[m] (values already permuted, so in-edge kernels read them
//        sequentially instead of through perm)
// The CSC is built on the device by counting sort: per-column counts, an
// exclusive scan, an atomic scatter, then a segmented sort of every column by
// CSR edge id, which makes it identical to the reference's stable sort by column
// (within a column, edges in CSR order) and therefore deterministic.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "mg_internal.h"

namespace {
thread_local char g_err[1024] = "";
}

void mg_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// Test hooks: host-side fault injection (no device fault is ever caused).
// g_fail_alloc: 0 off; k > 0: the k-th allocation from now and every later one
// fail (until the hook is disarmed), so no retry can mask the failure.
static std::atomic<int64_t> g_fail_alloc{0};
static std::atomic<int32_t> g_bar_extra{0};
static std::atomic<unsigned long long> g_bar_limit{1ull << 12};

cudaError_t mg_malloc_async(void **p, size_t bytes, cudaStream_t s) {
  int64_t k = g_fail_alloc.load();
  while (k > 1 && !g_fail_alloc.compare_exchange_weak(k, k - 1)) {
  }
  if (k == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocAsync(p, bytes, s);
}

int32_t debug_barrier_extra() { return g_bar_extra.load(); }
unsigned long long debug_barrier_limit() { return g_bar_limit.load(); }

extern "C" mg_status mg_graph_sync(mg_graph *g) {
  if (!g) {
    mg_set_error("mg_graph_sync: null graph");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return MG_OK;
}

extern "C" void mg_tuning_defaults(mg_tuning *t) {
  if (t) *t = tuning_defaults();
}

extern "C" mg_status mg_graph_get_tuning(mg_graph *g, mg_tuning *t) {
  if (!g || !t) {
    mg_set_error("mg_graph_get_tuning: null argument");
    return MG_ERR_ARG;
  }
  *t = g->tune;
  return MG_OK;
}

extern "C" mg_status mg_graph_set_tuning(mg_graph *g, const mg_tuning *t) {
  if (!g || !t) {
    mg_set_error("mg_graph_set_tuning: null argument");
    return MG_ERR_ARG;
  }
  struct Range {
    const char *name;
    int32_t v, lo, hi;
  } const r[] = {{"sssp_heavy", t->sssp_heavy, 1, 1 << 30},
                 {"sssp_heavy_small", t->sssp_heavy_small, 1, t->sssp_heavy},
                 {"sssp_ctas_per_sm", t->sssp_ctas_per_sm, 1, 8},
                 {"sssp_chunk_cap", t->sssp_chunk_cap, 0, 1 << 30},
                 {"sssp_batch_heavy", t->sssp_batch_heavy, 1, 1 << 30},
                 {"bfs_cta_th", t->bfs_cta_th, 32, 1 << 30},
                 {"bfs_grid_th", t->bfs_grid_th, 32, 1 << 30},
                 {"bfs_defer_warp", t->bfs_defer_warp, 0, 1},
                 {"bfs_persist_max", t->bfs_persist_max, 0, 1 << 30},
                 {"bfs_persist_edges", t->bfs_persist_edges, 0, 1 << 30},
                 {"bfs_alpha", t->bfs_alpha, 1, 1 << 20},
                 {"bfs_beta", t->bfs_beta, 1, 1 << 20},
                 {"bfs_sparse_degree", t->bfs_sparse_degree, 0, 1 << 20},
                 {"bfs_ctas_per_sm", t->bfs_ctas_per_sm, 1, 8},
                 {"bfs_tail_max", t->bfs_tail_max, 0, 1 << 30},
                 {"bfs_tail_edges", t->bfs_tail_edges, 0, 1 << 30},
                 {"cc_rounds", t->cc_rounds, 0, 8}};
  for (const Range &x : r) {
    if (x.v < x.lo || x.v > x.hi) {
      mg_set_error("mg_graph_set_tuning: %s = %d outside [%d, %d]", x.name, x.v, x.lo, x.hi);
      return MG_ERR_ARG;
    }
  }
  g->tune = *t;
  return MG_OK;
}

extern "C" mg_status mg_graph_trace(mg_graph *g, mg_level_record *out, int32_t cap, int32_t *count) {
  if (!g || !count || (cap > 0 && !out)) {
    mg_set_error("mg_graph_trace: null argument");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  int32_t len = 0;
  MG_CUDA_TRY(cudaMemcpyAsync(&len, &g->ctl->trace_len, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  len = std::max(0, std::min(std::min(len, (int32_t)MG_TRACE_LEVELS), std::max(cap, 0)));
  if (len > 0)
    MG_CUDA_TRY(cudaMemcpyAsync(out, trace_of(g->ctl), sizeof(mg_level_record) * (size_t)len, cudaMemcpyDeviceToHost,
                                g->stream));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  *count = len;
  return MG_OK;
}

extern "C" mg_status mg_debug_fail_alloc(int64_t k) {
  if (k < 0) {
    mg_set_error("mg_debug_fail_alloc: k must be >= 0");
    return MG_ERR_ARG;
  }
  g_fail_alloc.store(k);
  return MG_OK;
}

extern "C" mg_status mg_debug_barrier_skew(int32_t extra, int64_t poll_limit) {
  if (extra < 0 || poll_limit <= 0) {
    mg_set_error("mg_debug_barrier_skew: extra must be >= 0 and poll_limit > 0");
    return MG_ERR_ARG;
  }
  g_bar_extra.store(extra);
  g_bar_limit.store((unsigned long long)poll_limit);
  return MG_OK;
}

mg_status dev_alloc(mg_graph *g, void **p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = mg_malloc_async(p, std::max<size_t>(bytes, 1), g->stream);
  if (e == cudaErrorMemoryAllocation) {
    // Return the pool's idle blocks to the driver and try once more.
    cudaGetLastError();
    cudaMemPool_t pool;
    if (cudaStreamSynchronize(g->stream) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, g->device) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
    e = mg_malloc_async(p, std::max<size_t>(bytes, 1), g->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    mg_set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MG_ERR_OOM : MG_ERR_CUDA;
  }
  return MG_OK;
}

void dev_free(mg_graph *g, void *p) {
  if (p) cudaFreeAsync(p, g->stream);
}

mg_status ws_reserve(mg_graph *g, Workspace &w, size_t bytes) {
  if (w.bytes >= bytes) return MG_OK;
  dev_free(g, w.ptr);
  w.ptr = nullptr;
  const size_t grown = std::max(bytes, w.bytes + w.bytes / 4);
  w.bytes = 0;
  if (dev_alloc(g, &w.ptr, grown) != MG_OK) {
    mg_status st = dev_alloc(g, &w.ptr, bytes);
    if (st != MG_OK) {
      mg_set_error("workspace allocation of %zu bytes failed", bytes);
      return st;
    }
    w.bytes = bytes;
    return MG_OK;
  }
  w.bytes = grown;
  return MG_OK;
}

mg_status graph_enter(mg_graph *g) {
  MG_CUDA_TRY(cudaSetDevice(g->device));
  if (g->pending_validation) {
    // an asynchronous upload: wait for it and read the validation flags before any
    // kernel touches the arrays
    int hbad = 0;
    const int *bad = reinterpret_cast<const int *>(reinterpret_cast<const char *>(g->ctl) + sizeof(DevCtl));
    MG_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (hbad) {
      mg_set_error("mg_graph_create (asynchronous upload): %s",
                   (hbad & 1) ? "row offsets are not a valid CSR (0..m, non-decreasing)"
                              : "column index out of range [0, n)");
      return MG_ERR_ARG;
    }
    g->pending_validation = false;
  }
  return MG_OK;
}

mg_status check_device_ptr(const mg_graph *g, const void *p, const char *fn, const char *what) {
  if (!p) return MG_OK;
  cudaPointerAttributes at;
  const cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    mg_set_error("%s: cannot query %s (%s): it must be device memory", fn, what, cudaGetErrorString(e));
    return MG_ERR_ARG;
  }
  if (at.type == cudaMemoryTypeManaged) return MG_OK;
  if (at.type != cudaMemoryTypeDevice) {
    mg_set_error("%s: %s is %s memory; it must be device memory of device %d", fn, what,
                 at.type == cudaMemoryTypeHost ? "pinned host" : "pageable host", g->device);
    return MG_ERR_ARG;
  }
  if (at.device != g->device) {
    mg_set_error("%s: %s is memory of device %d, the graph lives on device %d", fn, what, at.device, g->device);
    return MG_ERR_ARG;
  }
  return MG_OK;
}

mg_status copy_out(mg_graph *g, void *dst, const void *src, size_t bytes, int device_output) {
  if (bytes == 0) return MG_OK;
  MG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, device_output ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                              g->stream));
  return MG_OK;
}

namespace mg {

// ---------------------------------------------------------------------------
// Validation: row offsets non-decreasing from 0 to m, column indices in [0, n).
// Column indices are read with 16-byte vector loads.
__global__ void validate_kernel(const int32_t *__restrict__ ro, const int32_t *__restrict__ ci, int64_t n,
                                int64_t m, int *__restrict__ bad) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int b = 0;
  for (int64_t i = tid; i <= n; i += stride) {
    int32_t r = ro[i];
    if (i == 0 && r != 0) b |= 1;
    if (i == n && r != (int32_t)m) b |= 1;
    if (i < n && ro[i + 1] < r) b |= 1;
  }
  const int64_t m4 = m / 4;
  const int4 *ci4 = reinterpret_cast<const int4 *>(ci);
  const uint32_t un = (uint32_t)n;
  for (int64_t i = tid; i < m4; i += stride) {
    int4 c = __ldg(ci4 + i);
    if ((uint32_t)c.x >= un || (uint32_t)c.y >= un || (uint32_t)c.z >= un || (uint32_t)c.w >= un) b |= 2;
  }
  for (int64_t i = m4 * 4 + tid; i < m; i += stride)
    if ((uint32_t)ci[i] >= un) b |= 2;
  if (b) atomicOr(bad, b);
}

// ---------------------------------------------------------------------------
// Exclusive scan of int32 counts (n items) into int32 offsets (n + 1 items),
// three passes over tiles of 2048.
constexpr int SCAN_NT = 256, SCAN_VT = 8, SCAN_TILE = SCAN_NT * SCAN_VT;

__global__ void __launch_bounds__(SCAN_NT) scan_tile_sums(const int32_t *__restrict__ in, int64_t n,
                                                          int64_t *__restrict__ sums) {
  __shared__ int64_t sm[SCAN_NT / 32 + 1];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_VT; k++) {
    int64_t i = base + k * SCAN_NT + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = block_sum<SCAN_NT>(s, sm);
  if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) scan_sums_single(int64_t *__restrict__ sums, int64_t nt) {
  __shared__ int64_t sm[1024 / 32 + 1];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b = 0; b < nt; b += 1024) {
    int64_t i = b + threadIdx.x;
    int64_t v = i < nt ? sums[i] : 0;
    int64_t tot;
    int64_t ex = block_exclusive_scan<1024>(v, sm, &tot);
    if (i < nt) sums[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SCAN_NT) scan_tiles(const int32_t *__restrict__ in, int64_t n,
                                                      const int64_t *__restrict__ sums, int32_t *__restrict__ out) {
  __shared__ int64_t sm[SCAN_NT / 32 + 1];
  __shared__ int32_t tile[SCAN_TILE];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int k = 0; k < SCAN_VT; k++) {
    int64_t i = base + k * SCAN_NT + threadIdx.x;
    tile[k * SCAN_NT + threadIdx.x] = i < n ? in[i] : 0;
  }
  __syncthreads();
  int64_t loc[SCAN_VT];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_VT; k++) {
    loc[k] = s;
    s += tile[threadIdx.x * SCAN_VT + k];
  }
  int64_t tot;
  int64_t ex = block_exclusive_scan<SCAN_NT>(s, sm, &tot);
  int64_t off = sums[blockIdx.x] + ex;
#pragma unroll
  for (int k = 0; k < SCAN_VT; k++) {
    int64_t i = base + threadIdx.x * SCAN_VT + k;
    if (i < n) out[i] = (int32_t)(off + loc[k]);
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_NT - 1) out[n] = (int32_t)(off + s);
}

}  // namespace mg

// Exclusive scan of n int32 counts into n+1 offsets; tmp must hold
// ceil(n / 2048) int64 values.
mg_status device_exclusive_scan(const int32_t *in, int32_t *out, int64_t n, int64_t *tmp, cudaStream_t s) {
  using namespace mg;
  int64_t nt = std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
  scan_tile_sums<<<(unsigned)nt, SCAN_NT, 0, s>>>(in, n, tmp);
  scan_sums_single<<<1, 1024, 0, s>>>(tmp, nt);
  scan_tiles<<<(unsigned)nt, SCAN_NT, 0, s>>>(in, n, tmp, out);
  MG_CUDA_TRY(cudaGetLastError());
  return MG_OK;
}

namespace mg {

// Pads of an offsets array (INT_MAX after entry n) and of its edge arrays (0).
__global__ void fill_pad_kernel(int32_t *off, int64_t n, int32_t *edges, void *vals, int64_t m) {
  const int t = threadIdx.x;
  if (t < MG_OFF_PAD) off[n + 1 + t] = INT_MAX;
  if (t < MG_EDGE_PAD) {
    edges[m + t] = 0;
    if (vals) reinterpret_cast<int32_t *>(vals)[m + t] = 0;
  }
}

// ---------------------------------------------------------------------------
// CSC build kernels.
__global__ void count_cols_kernel(const int32_t *__restrict__ ci, int64_t m, int32_t *__restrict__ cnt) {
  const int64_t m4 = m / 4;
  const int4 *ci4 = reinterpret_cast<const int4 *>(ci);
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < m4; i += stride) {
    int4 c = __ldg(ci4 + i);
    atomicAdd(&cnt[c.x], 1);
    atomicAdd(&cnt[c.y], 1);
    atomicAdd(&cnt[c.z], 1);
    atomicAdd(&cnt[c.w], 1);
  }
  for (int64_t i = m4 * 4 + tid; i < m; i += stride) atomicAdd(&cnt[ci[i]], 1);
}

// One warp per row: the warp walks the row's edges with coalesced loads and
// drops (row, edge id) into the column buckets.
__global__ void scatter_csc_kernel(const int32_t *__restrict__ ro, const int32_t *__restrict__ ci, int64_t n,
                                   const int32_t *__restrict__ co, int32_t *__restrict__ cursor,
                                   int32_t *__restrict__ ri, int32_t *__restrict__ perm) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int l = lane_id();
  for (int64_t v = warp; v < n; v += nwarps) {
    const int32_t b = ro[v], e = ro[v + 1];
    for (int32_t k = b + l; k < e; k += 32) {
      int32_t c = ci[k];
      int32_t pos = co[c] + atomicAdd(&cursor[c], 1);
      ri[pos] = (int32_t)v;
      perm[pos] = k;
    }
  }
}

// Sorting classes of column segments.
constexpr int SEG_SMALL = 32;    // insertion sort by one thread
constexpr int SEG_MEDIUM = 2048; // bitonic sort of the whole segment in shared memory
constexpr int SORT_NT = 256;

__global__ void classify_segments_kernel(const int32_t *__restrict__ co, int64_t n, int32_t *__restrict__ lists,
                                         int32_t *__restrict__ lens, int32_t cap) {
  int32_t dummy_overflow = 0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t len = co[c + 1] - co[c];
    int cls = len <= 1 ? -1 : (len <= SEG_SMALL ? 0 : (len <= SEG_MEDIUM ? 1 : 2));
    for (int k = 0; k < 3; k++) warp_append(cls == k, (int32_t)c, lists + (size_t)k * cap, &lens[k], cap, &dummy_overflow);
  }
}

__global__ void sort_small_kernel(const int32_t *__restrict__ co, const int32_t *__restrict__ list,
                                  const int32_t *__restrict__ len, int32_t *__restrict__ key,
                                  int32_t *__restrict__ val) {
  const int32_t cnt = *len;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int32_t c = list[i];
    const int32_t b = co[c], e = co[c + 1];
    for (int32_t x = b + 1; x < e; x++) {
      int32_t k = key[x], v = val[x];
      int32_t y = x - 1;
      while (y >= b && key[y] > k) {
        key[y + 1] = key[y];
        val[y + 1] = val[y];
        y--;
      }
      key[y + 1] = k;
      val[y + 1] = v;
    }
  }
}

// Bitonic sort of `cnt` (<= SEG_MEDIUM) key/value pairs held in shared memory,
// padded to the next power of two with INT_MAX keys.
__device__ void smem_bitonic(int32_t *sk, int32_t *sv, int p2) {
  for (int size = 2; size <= p2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < p2 / 2; t += blockDim.x) {
        int lo = 2 * t - (t & (stride - 1));
        int hi = lo + stride;
        bool up = ((lo & size) == 0);
        int32_t a = sk[lo], b = sk[hi];
        if ((a > b) == up) {
          sk[lo] = b;
          sk[hi] = a;
          int32_t tv = sv[lo];
          sv[lo] = sv[hi];
          sv[hi] = tv;
        }
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(SORT_NT) sort_medium_kernel(const int32_t *__restrict__ co,
                                                               const int32_t *__restrict__ list,
                                                               const int32_t *__restrict__ len,
                                                               int32_t *__restrict__ key, int32_t *__restrict__ val) {
  __shared__ int32_t sk[SEG_MEDIUM], sv[SEG_MEDIUM];
  const int32_t cnt = *len;
  for (int32_t i = blockIdx.x; i < cnt; i += gridDim.x) {
    const int32_t c = list[i];
    const int32_t b = co[c], L = co[c + 1] - b;
    int p2 = 1;
    while (p2 < L) p2 <<= 1;
    for (int t = threadIdx.x; t < p2; t += SORT_NT) {
      sk[t] = t < L ? key[b + t] : INT_MAX;
      sv[t] = t < L ? val[b + t] : 0;
    }
    __syncthreads();
    smem_bitonic(sk, sv, p2);
    for (int t = threadIdx.x; t < L; t += SORT_NT) {
      key[b + t] = sk[t];
      val[b + t] = sv[t];
    }
    __syncthreads();
  }
}

// Large segments: one CTA per segment sorts SEG_MEDIUM-sized runs in shared
// memory, then merges runs pairwise through a scratch buffer (tk/tv, same
// offsets as key/val). Each thread merges a fixed slice of the output found by
// a merge-path search.
__device__ int merge_path(const int32_t *a, int la, const int32_t *b, int lb, int diag) {
  int lo = max(0, diag - lb), hi = min(diag, la);
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(SORT_NT) sort_large_kernel(const int32_t *__restrict__ co,
                                                              const int32_t *__restrict__ list,
                                                              const int32_t *__restrict__ len, int32_t *key,
                                                              int32_t *val, int32_t *tk, int32_t *tv) {
  __shared__ int32_t sk[SEG_MEDIUM], sv[SEG_MEDIUM];
  const int32_t cnt = *len;
  for (int32_t i = blockIdx.x; i < cnt; i += gridDim.x) {
    const int32_t c = list[i];
    const int32_t b = co[c], L = co[c + 1] - b;
    for (int32_t r0 = 0; r0 < L; r0 += SEG_MEDIUM) {
      int rl = min(SEG_MEDIUM, L - r0);
      for (int t = threadIdx.x; t < SEG_MEDIUM; t += SORT_NT) {
        sk[t] = t < rl ? key[b + r0 + t] : INT_MAX;
        sv[t] = t < rl ? val[b + r0 + t] : 0;
      }
      __syncthreads();
      smem_bitonic(sk, sv, SEG_MEDIUM);
      for (int t = threadIdx.x; t < rl; t += SORT_NT) {
        key[b + r0 + t] = sk[t];
        val[b + r0 + t] = sv[t];
      }
      __syncthreads();
    }
    int32_t *srck = key + b, *srcv = val + b, *dstk = tk + b, *dstv = tv + b;
    for (int32_t w = SEG_MEDIUM; w < L; w <<= 1) {
      for (int32_t p0 = 0; p0 < L; p0 += 2 * w) {
        const int32_t la = min(w, L - p0), lb = max(0, min(w, L - p0 - w));
        const int32_t *ak = srck + p0, *bk = srck + p0 + la;
        const int32_t *av = srcv + p0, *bv = srcv + p0 + la;
        const int32_t tot = la + lb;
        const int32_t per = (tot + SORT_NT - 1) / SORT_NT;
        int32_t d0 = min(tot, (int32_t)threadIdx.x * per), d1 = min(tot, d0 + per);
        int ia = merge_path(ak, la, bk, lb, d0);
        int ib = d0 - ia;
        for (int32_t d = d0; d < d1; d++) {
          bool takea = ib >= lb || (ia < la && ak[ia] <= bk[ib]);
          if (takea) {
            dstk[p0 + d] = ak[ia];
            dstv[p0 + d] = av[ia];
            ia++;
          } else {
            dstk[p0 + d] = bk[ib];
            dstv[p0 + d] = bv[ib];
            ib++;
          }
        }
      }
      __syncthreads();
      int32_t *t1 = srck, *t2 = srcv;
      srck = dstk;
      srcv = dstv;
      dstk = t1;
      dstv = t2;
    }
    if (srck != key + b) {
      for (int32_t t = threadIdx.x; t < L; t += SORT_NT) {
        key[b + t] = srck[t];
        val[b + t] = srcv[t];
      }
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void permute_values_kernel(const int32_t *__restrict__ perm, const T *__restrict__ src, int64_t m,
                                      T *__restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

}  // namespace mg

static int grid_for(const mg_graph *g, int per_sm = 8) { return g->num_sms * per_sm; }

// Builds the CSC of g (co, ri, perm, cvals). Scratch is taken from ws_aux.
static mg_status build_csc(mg_graph *g) {
  using namespace mg;
  const int64_t n = g->n, m = g->m;
  cudaStream_t s = g->stream;
  const size_t vbytes = g->vtype == MG_DTYPE_NONE ? 0 : 4;
  g->csc_owned = true;  // set first: a failure below frees what was allocated
  MG_CUDA_TRY(mg_malloc_async((void **)&g->co, sizeof(int32_t) * (n + 1 + MG_OFF_PAD), s));
  MG_CUDA_TRY(mg_malloc_async((void **)&g->ri, sizeof(int32_t) * (m + MG_EDGE_PAD), s));
  MG_CUDA_TRY(mg_malloc_async((void **)&g->perm, sizeof(int32_t) * (m + MG_EDGE_PAD), s));
  if (vbytes) MG_CUDA_TRY(mg_malloc_async(&g->cvals, vbytes * (m + MG_EDGE_PAD), s));
  mg::fill_pad_kernel<<<1, 32, 0, s>>>(g->co, n, g->ri, g->cvals, m);
  g->has_csc = true;
  const int64_t ntiles = std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
  const size_t need = Carve::need({sizeof(int32_t) * (size_t)(n + 1), sizeof(int32_t) * (size_t)(n + 1),
                                   sizeof(int64_t) * (size_t)ntiles, sizeof(int32_t) * 3 * (size_t)(n + 1),
                                   sizeof(int32_t) * 4, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1),
                                   sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1)});
  MG_TRY(ws_reserve(g, g->ws_aux, need));
  Carve cv(g->ws_aux.ptr);
  int32_t *cnt = cv.take<int32_t>(n + 1);
  int32_t *cursor = cv.take<int32_t>(n + 1);
  int64_t *tmp = cv.take<int64_t>(ntiles);
  int32_t *lists = cv.take<int32_t>(3 * (size_t)(n + 1));
  int32_t *lens = cv.take<int32_t>(4);
  int32_t *tk = cv.take<int32_t>(std::max<int64_t>(m, 1));
  int32_t *tv = cv.take<int32_t>(std::max<int64_t>(m, 1));
  MG_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), s));
  MG_CUDA_TRY(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (n + 1), s));
  MG_CUDA_TRY(cudaMemsetAsync(lens, 0, sizeof(int32_t) * 4, s));
  const int grid = grid_for(g);
  if (m > 0) count_cols_kernel<<<grid, 256, 0, s>>>(g->ci, m, cnt);
  MG_TRY(device_exclusive_scan(cnt, g->co, n, tmp, s));
  if (m > 0) {
    scatter_csc_kernel<<<grid, 256, 0, s>>>(g->ro, g->ci, n, g->co, cursor, g->ri, g->perm);
    classify_segments_kernel<<<grid, 256, 0, s>>>(g->co, n, lists, lens, (int32_t)(n + 1));
    sort_small_kernel<<<grid, 256, 0, s>>>(g->co, lists, lens + 0, g->perm, g->ri);
    sort_medium_kernel<<<grid, SORT_NT, 0, s>>>(g->co, lists + (n + 1), lens + 1, g->perm, g->ri);
    sort_large_kernel<<<grid, SORT_NT, 0, s>>>(g->co, lists + 2 * (n + 1), lens + 2, g->perm, g->ri, tk, tv);
    if (g->vtype == MG_DTYPE_I32)
      permute_values_kernel<int32_t><<<grid, 256, 0, s>>>(g->perm, (const int32_t *)g->vals, m, (int32_t *)g->cvals);
    else if (g->vtype == MG_DTYPE_F32)
      permute_values_kernel<float><<<grid, 256, 0, s>>>(g->perm, (const float *)g->vals, m, (float *)g->cvals);
  }
  MG_CUDA_TRY(cudaGetLastError());
  return MG_OK;
}

// Pinned host mirrors of the control blocks, recycled across graphs: pinning
// and unpinning host memory costs a driver round trip each time.
static std::mutex g_pinned_mu;
static std::vector<void *> g_pinned_free;

static DevCtl *pinned_ctl_get() {
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    if (!g_pinned_free.empty()) {
      void *p = g_pinned_free.back();
      g_pinned_free.pop_back();
      return static_cast<DevCtl *>(p);
    }
  }
  void *p = nullptr;
  if (cudaHostAlloc(&p, sizeof(DevCtl) + 64, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return static_cast<DevCtl *>(p);
}

static void pinned_ctl_put(DevCtl *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  g_pinned_free.push_back(p);
}

static void graph_free_device(mg_graph *g) {
  cudaStream_t s = g->stream;
  auto fr = [&](void *p) {
    if (p) cudaFreeAsync(p, s);
  };
  fr(g->ro);
  fr(g->ci);
  fr(g->vals);
  if (g->csc_owned) {
    fr(g->co);
    fr(g->ri);
    fr(g->perm);
    fr(g->cvals);
  }
  fr(g->ws_main.ptr);
  fr(g->ws_aux.ptr);
  fr(g->ws_out.ptr);
  fr(g->ctl);
  if (s) cudaStreamSynchronize(s);
  pinned_ctl_put(g->ctl_host);
  g->ctl_host = nullptr;
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (s) cudaStreamDestroy(s);
  cudaGetLastError();
}

void engine_release_cached(mg_graph *g);  // defined with the iteration drivers
void pr_release_plans(mg_graph *g);       // defined with PageRank

extern "C" {

const char *mg_status_string(mg_status s) {
  switch (s) {
    case MG_OK: return "MG_OK";
    case MG_ERR_ARG: return "MG_ERR_ARG: invalid argument";
    case MG_ERR_OOM: return "MG_ERR_OOM: out of memory";
    case MG_ERR_QUEUE_OVERFLOW: return "MG_ERR_QUEUE_OVERFLOW: frontier queue overflow, increase queue_sizing";
    case MG_ERR_TIMEOUT: return "MG_ERR_TIMEOUT: a bounded device wait ran out";
    case MG_ERR_CUDA: return "MG_ERR_CUDA: CUDA runtime error";
    case MG_ERR_NO_DEVICE: return "MG_ERR_NO_DEVICE: no usable CUDA device";
    case MG_ERR_UNSUPPORTED: return "MG_ERR_UNSUPPORTED: unsupported option combination";
  }
  return "unknown mg_status";
}

const char *mg_last_error(void) { return g_err; }

const char *mg_version(void) { return "mapgraph_b200 0.1.0 (sm_100a)"; }

int32_t mg_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

static mg_status create_impl(const int32_t *row_offsets, const int32_t *col_idx, const void *edge_vals,
                             mg_dtype vals_t, int64_t n, int64_t m, uint32_t flags, mg_graph **out) {
  if (!out) {
    mg_set_error("mg_graph_create: out is NULL");
    return MG_ERR_ARG;
  }
  *out = nullptr;
  if (n < 0 || m < 0 || n > INT32_MAX - 1 || m > INT32_MAX || !row_offsets || (m > 0 && !col_idx) ||
      (vals_t != MG_DTYPE_NONE && m > 0 && !edge_vals) || vals_t < MG_DTYPE_NONE || vals_t > MG_DTYPE_F32) {
    mg_set_error("mg_graph_create: invalid sizes or null arrays (n=%lld m=%lld)", (long long)n, (long long)m);
    return MG_ERR_ARG;
  }
  if (mg_device_count() <= 0) {
    mg_set_error("mg_graph_create: no CUDA device");
    return MG_ERR_NO_DEVICE;
  }
  mg_graph *g = new mg_graph();
  g->n = n;
  g->m = m;
  g->flags = flags;
  g->vtype = vals_t;
  auto fail = [&](mg_status st) {
    graph_free_device(g);
    delete g;
    return st;
  };
  if (cudaGetDevice(&g->device) != cudaSuccess) return fail(MG_ERR_CUDA);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
  g->num_sms = sms > 0 ? sms : 148;
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
    mg_set_error("mg_graph_create: stream creation failed");
    return fail(MG_ERR_CUDA);
  }
  {
    // Keep freed graph memory in the stream-ordered pool so that repeated
    // create/destroy cycles reuse it instead of returning it to the driver.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g->device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
  }
  cudaStream_t s = g->stream;
  const size_t vb = vals_t == MG_DTYPE_NONE ? 0 : 4;
  const cudaMemcpyKind kind = (flags & MG_GRAPH_DEVICE_INPUT) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
#define CREATE_TRY(expr)                                                                        \
  do {                                                                                          \
    cudaError_t _e = (expr);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      mg_set_error("mg_graph_create: %s failed: %s", #expr, cudaGetErrorString(_e));           \
      cudaGetLastError();                                                                       \
      return fail(_e == cudaErrorMemoryAllocation ? MG_ERR_OOM : MG_ERR_CUDA);                  \
    }                                                                                           \
  } while (0)
  CREATE_TRY(mg_malloc_async((void **)&g->ro, sizeof(int32_t) * (n + 1 + MG_OFF_PAD), s));
  CREATE_TRY(mg_malloc_async((void **)&g->ci, sizeof(int32_t) * (m + MG_EDGE_PAD), s));
  if (vb) CREATE_TRY(mg_malloc_async(&g->vals, vb * (m + MG_EDGE_PAD), s));
  mg::fill_pad_kernel<<<1, 32, 0, s>>>(g->ro, n, g->ci, g->vals, m);
  CREATE_TRY(cudaMemcpyAsync(g->ro, row_offsets, sizeof(int32_t) * (n + 1), kind, s));
  if (m > 0) CREATE_TRY(cudaMemcpyAsync(g->ci, col_idx, sizeof(int32_t) * m, kind, s));
  if (vb && m > 0) CREATE_TRY(cudaMemcpyAsync(g->vals, edge_vals, vb * m, kind, s));
  if (dev_alloc(g, (void **)&g->ctl, MG_TRACE_OFF + sizeof(mg_level_record) * MG_TRACE_LEVELS) != MG_OK)
    return fail(MG_ERR_OOM);
  g->ctl_host = pinned_ctl_get();
  if (!g->ctl_host) {
    mg_set_error("mg_graph_create: pinned host allocation failed");
    return fail(MG_ERR_OOM);
  }
  CREATE_TRY(cudaEventCreate(&g->ev0));
  CREATE_TRY(cudaEventCreate(&g->ev1));
  // Validate on the device.
  int *bad = reinterpret_cast<int *>(reinterpret_cast<char *>(g->ctl) + sizeof(DevCtl));
  CREATE_TRY(cudaMemsetAsync(bad, 0, sizeof(int) * 2, s));
  mg::validate_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ro, g->ci, n, m, bad);
  CREATE_TRY(cudaGetLastError());
  if ((flags & MG_GRAPH_ASYNC_UPLOAD) && (flags & (MG_GRAPH_SYMMETRIC | MG_GRAPH_NO_CSC))) {
    // no CSC to build from unvalidated arrays: return now, check on first use
    g->pending_validation = true;
    if (flags & MG_GRAPH_SYMMETRIC) {
      g->co = g->ro;
      g->ri = g->ci;
      g->perm = nullptr;
      g->cvals = g->vals;
      g->has_csc = true;
      g->csc_owned = false;
    }
    *out = g;
    return MG_OK;
  }
  int hbad[2] = {0, 0};
  CREATE_TRY(cudaMemcpyAsync(hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  CREATE_TRY(cudaStreamSynchronize(s));
  if (hbad[0]) {
    mg_set_error("mg_graph_create: %s", (hbad[0] & 1) ? "row offsets are not a valid CSR (0..m, non-decreasing)"
                                                      : "column index out of range [0, n)");
    return fail(MG_ERR_ARG);
  }
  if (flags & MG_GRAPH_SYMMETRIC) {
    g->co = g->ro;
    g->ri = g->ci;
    g->perm = nullptr;
    g->cvals = g->vals;
    g->has_csc = true;
    g->csc_owned = false;
  } else if (!(flags & MG_GRAPH_NO_CSC)) {
    mg_status st = build_csc(g);
    if (st != MG_OK) return fail(st);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    mg_set_error("mg_graph_create: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(MG_ERR_CUDA);
  }
#undef CREATE_TRY
  *out = g;
  return MG_OK;
}

mg_status mg_graph_create(const int32_t *row_offsets, const int32_t *col_idx, const void *edge_vals,
                          mg_dtype vals_t, int64_t n, int64_t m, uint32_t flags, mg_graph **out) {
  return create_impl(row_offsets, col_idx, edge_vals, vals_t, n, m, flags, out);
}

mg_status mg_graph_destroy(mg_graph *g) {
  if (!g) return MG_OK;
  cudaSetDevice(g->device);
  engine_release_cached(g);
  pr_release_plans(g);
  graph_free_device(g);
  delete g;
  return MG_OK;
}

mg_status mg_graph_stream(const mg_graph *g, void **stream) {
  if (!g || !stream) {
    mg_set_error("mg_graph_stream: null argument");
    return MG_ERR_ARG;
  }
  *stream = (void *)g->stream;
  return MG_OK;
}

mg_status mg_graph_info(const mg_graph *g, int64_t *n, int64_t *m, uint32_t *flags, int32_t *device) {
  if (!g) {
    mg_set_error("mg_graph_info: graph is NULL");
    return MG_ERR_ARG;
  }
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (flags) *flags = g->flags;
  if (device) *device = g->device;
  return MG_OK;
}

namespace {
// out[0] = max out-degree, out[1] = vertices without out-edges.
__global__ void degree_stats_kernel(const int32_t *__restrict__ ro, int64_t n, unsigned long long *out) {
  int32_t mx = 0;
  unsigned long long zero = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = ro[i + 1] - ro[i];
    mx = max(mx, d);
    zero += d == 0;
  }
  mx = __reduce_max_sync(0xffffffffu, mx);
  for (int o = 16; o > 0; o >>= 1) zero += __shfl_xor_sync(0xffffffffu, zero, o);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)mx);
    if (zero) atomicAdd(out + 1, zero);
  }
}
}  // namespace

mg_status mg_graph_degree_stats(mg_graph *g, int64_t *max_out_degree, int64_t *no_out_edges) {
  if (!g) {
    mg_set_error("mg_graph_degree_stats: graph is NULL");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  // two counters in the control block's spare bytes behind the DevCtl
  unsigned long long *d = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(g->ctl) + sizeof(DevCtl));
  unsigned long long h[2] = {0, 0};
  MG_CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
  if (g->n > 0) degree_stats_kernel<<<g->num_sms * 4, 256, 0, g->stream>>>(g->ro, g->n, d);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (max_out_degree) *max_out_degree = (int64_t)h[0];
  if (no_out_edges) *no_out_edges = (int64_t)h[1];
  return MG_OK;
}

mg_status mg_graph_device_arrays(const mg_graph *g, const int32_t **row_offsets, const int32_t **col_idx,
                                 const void **edge_vals, const int32_t **col_offsets, const int32_t **row_idx,
                                 const int32_t **csc_perm) {
  if (!g) {
    mg_set_error("mg_graph_device_arrays: graph is NULL");
    return MG_ERR_ARG;
  }
  if (row_offsets) *row_offsets = g->ro;
  if (col_idx) *col_idx = g->ci;
  if (edge_vals) *edge_vals = g->vals;
  if (col_offsets) *col_offsets = g->has_csc ? g->co : nullptr;
  if (row_idx) *row_idx = g->has_csc ? g->ri : nullptr;
  if (csc_perm) *csc_perm = g->perm;
  return MG_OK;
}

mg_status mg_graph_create_ragged(int32_t ngraphs, const int32_t *const *row_offsets, const int32_t *const *col_idx,
                                 const int64_t *n, const int64_t *m, uint32_t flags, mg_graph **out) {
  if (!out || ngraphs <= 0 || !row_offsets || !col_idx || !n || !m || (flags & MG_GRAPH_DEVICE_INPUT)) {
    mg_set_error("mg_graph_create_ragged: invalid arguments");
    return MG_ERR_ARG;
  }
  int64_t N = 0, M = 0;
  std::vector<int64_t> vbase(ngraphs + 1, 0);
  for (int32_t i = 0; i < ngraphs; i++) {
    if (n[i] < 0 || m[i] < 0 || !row_offsets[i] || (m[i] > 0 && !col_idx[i])) {
      mg_set_error("mg_graph_create_ragged: member %d invalid", i);
      return MG_ERR_ARG;
    }
    vbase[i] = N;
    N += n[i];
    M += m[i];
  }
  vbase[ngraphs] = N;
  if (N > INT32_MAX - 1 || M > INT32_MAX) {
    mg_set_error("mg_graph_create_ragged: union exceeds int32");
    return MG_ERR_ARG;
  }
  std::vector<int32_t> ro(N + 1), ci(std::max<int64_t>(M, 1));
  int64_t eo = 0;
  for (int32_t i = 0; i < ngraphs; i++) {
    const int32_t *r = row_offsets[i];
    if (r[0] != 0 || r[n[i]] != m[i]) {
      mg_set_error("mg_graph_create_ragged: member %d row offsets do not span 0..m", i);
      return MG_ERR_ARG;
    }
    for (int64_t v = 0; v < n[i]; v++) ro[vbase[i] + v] = (int32_t)(eo + r[v]);
    for (int64_t e = 0; e < m[i]; e++) {
      int32_t c = col_idx[i][e];
      if (c < 0 || c >= n[i]) {
        mg_set_error("mg_graph_create_ragged: member %d column index out of range", i);
        return MG_ERR_ARG;
      }
      ci[eo + e] = (int32_t)(vbase[i] + c);
    }
    eo += m[i];
  }
  ro[N] = (int32_t)M;
  mg_status st = create_impl(ro.data(), ci.data(), nullptr, MG_DTYPE_NONE, N, M, flags, out);
  if (st == MG_OK) (*out)->vbase = vbase;
  return st;
}

mg_status mg_graph_ragged_bases(const mg_graph *g, int64_t *vertex_base) {
  if (!g || !vertex_base || g->vbase.empty()) {
    mg_set_error("mg_graph_ragged_bases: not a ragged graph");
    return MG_ERR_ARG;
  }
  std::memcpy(vertex_base, g->vbase.data(), sizeof(int64_t) * g->vbase.size());
  return MG_OK;
}

}  // extern "C"
