// pagerank.cu -- PageRank (struct pagerank, Algorithms/PageRank/PageRank.h:33-409)
// and its adjoint.
//
// Two modes:
//  NORMALIZED  x' = alpha * (P^T x + d t) + (1 - alpha) t over all vertices each
//              iteration; P_uv = a_uv / s_u (a = 1 unweighted), d = rank mass on
//              dangling vertices, t = teleport. One iteration is two kernels: the
//              merge-path gather over the CSC (pr_gather.cuh) with the update fused
//              into its epilogue (new x, new x/s for the next gather, |dx| and
//              dangling-mass partials), then the fix-up of rows split across tiles,
//              whose last CTA sums the FP64 partials in a fixed order and decides
//              convergence on the device (L1 change < tol or max_iter).
//  REFCOMPAT   the reference's program: x' = 0.15 + 0.85 * sum x_u / deg_u over the
//              in-edges of the frontier, a vertex stays active while |dx| >= 0.01,
//              the next frontier is the out-neighbourhood of the changed vertices
//              (gather_edge/apply/expand_edge, PageRank.h:233-363); deg = outdeg,
//              or outdeg + indeg with directed == 0 (PageRank.h:141-161).
//
// The adjoint of the NORMALIZED fixed point reuses the same gather on the CSR
// (the reversed graph) and one edge kernel for the weight gradients.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "expand.cuh"
#include "pr_binned.cuh"
#include "pr_gather.cuh"
#include "pr_segment.cuh"
#include "ppr.cuh"

namespace mg {

// ---------------------------------------------------------------------------
// Plans: merge-path tile coordinates of one adjacency, cached per graph.
struct GatherPlan {
  int32_t ntiles = 0;
  int32_t *tx = nullptr, *ty = nullptr;
};

// Shared-memory cache of the most gathered columns (forward gather over the
// CSC): the K vertices of largest out-degree get slots 0..K-1; cidx is the CSC
// index array with each cached column replaced by (slot | 0x80000000), so the
// gather reads those values from shared memory.
struct HubCache {
  int32_t *cidx = nullptr;  // m + 8 entries
  int32_t *slot = nullptr;  // n: slot of a vertex, -1 if not cached
  int32_t *hv = nullptr;    // K: vertex of a slot
  int32_t K = 0;
  int32_t cap = 0;          // capacity it was built for
  bool ok = false;
};

struct PlanSet {
  GatherPlan csc, csr;
  BinPlan bcsc, bcsr;
  bool bcsc_ok = false, bcsr_ok = false;
  HubCache hubs;
  SegPlan seg;  // column-segmented gather of the hub rows (forward gather)
  // Autotuned forward gather (-1: not tuned): its gather_kernel variant, column-cache
  // capacity (0 none), and for the segmented gather its hub threshold and block width.
  int32_t tuned_variant = -1;
  int32_t tuned_cap = 0;
  int32_t tuned_seg_T = 0;
  int32_t tuned_seg_S = 0;
  int32_t tuned_ppr_w = -1;  // autotuned personalised-PageRank group width (-1 not tuned)
};

}  // namespace mg

static void seg_plan_release(mg_graph *g, mg::SegPlan &sp);

static mg::PlanSet *plans_of(mg_graph *g) {
  if (!g->plan_csc) g->plan_csc = new mg::PlanSet();
  return static_cast<mg::PlanSet *>(g->plan_csc);
}

void pr_release_plans(mg_graph *g) {
  if (!g->plan_csc) return;
  mg::PlanSet *ps = static_cast<mg::PlanSet *>(g->plan_csc);
  for (mg::GatherPlan *p : {&ps->csc, &ps->csr}) {
    dev_free(g, p->tx);
    dev_free(g, p->ty);
  }
  for (mg::BinPlan *b : {&ps->bcsc, &ps->bcsr}) bin_plan_release(g->stream, *b);
  for (void *q : {(void *)ps->hubs.cidx, (void *)ps->hubs.slot, (void *)ps->hubs.hv}) dev_free(g, q);
  seg_plan_release(g, ps->seg);
  delete ps;
  g->plan_csc = nullptr;
}

static mg_status get_plan(mg_graph *g, bool csr, mg::GatherPlan **out) {
  using namespace mg;
  PlanSet *ps = plans_of(g);
  GatherPlan &p = csr ? ps->csr : ps->csc;
  if (!p.tx) {
    const int64_t items = g->n + g->m;
    const int64_t nt = (items + PRG_IPC - 1) / PRG_IPC;
    p.ntiles = (int32_t)std::max<int64_t>(nt, 1);
    mg_status st = dev_alloc(g, (void **)&p.tx, sizeof(int32_t) * (p.ntiles + 1));
    if (st == MG_OK) st = dev_alloc(g, (void **)&p.ty, sizeof(int32_t) * (p.ntiles + 1));
    if (st != MG_OK) {  // no half-built plan survives a failure
      dev_free(g, p.tx);
      dev_free(g, p.ty);
      p.tx = p.ty = nullptr;
      return st;
    }
    prg_plan_kernel<<<(p.ntiles + 256) / 256, 256, 0, g->stream>>>(csr ? g->ro : g->co, g->n, g->m, p.ntiles, p.tx,
                                                                    p.ty);
    MG_CUDA_TRY(cudaGetLastError());
  }
  *out = &p;
  return MG_OK;
}

// Degree-binned plan of any row-offset array (n + 1 entries) on stream s: the
// CSC of a graph (forward gather), its CSR (adjoint, row sums) or the owned rows
// of a partition slice.
static mg_status bin_plan_build_impl(cudaStream_t s, const int32_t *off, int64_t n, mg::BinPlan &bp,
                                     int32_t heavy) {
  using namespace mg;
  auto alloc = [&](void **p, size_t bytes) -> mg_status {
    if (mg_malloc_async(p, std::max<size_t>(bytes, 4), s) != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      mg_set_error("PageRank plan: device allocation of %zu bytes failed", bytes);
      return MG_ERR_OOM;
    }
    return MG_OK;
  };
  const int64_t nchunks = std::max<int64_t>(1, (n + PRB_CHUNK_ROWS - 1) / PRB_CHUNK_ROWS);
  int64_t *counts = nullptr;
  MG_CUDA_TRY(mg_malloc_async((void **)&counts, sizeof(int64_t) * ((nchunks + 2) * (PRB_BINS + 1)), s));
  int64_t *totals = counts + nchunks * (PRB_BINS + 1);
  int64_t *dboff = totals + (PRB_BINS + 1);
  prb_count_kernel<<<(unsigned)nchunks, PRB_NT, 0, s>>>(off, n, counts, heavy);
  prb_offsets_kernel<<<1, 32, 0, s>>>(counts, nchunks, totals);
  int64_t cnt[PRB_BINS + 1];
  MG_CUDA_TRY(cudaMemcpyAsync(cnt, totals, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  int64_t acc = 0;
  for (int b = 0; b < PRB_BINS; b++) {
    bp.boff[b] = acc;
    if (b < 6) acc += cnt[b];
  }
  bp.boff[PRB_BINS] = acc;
  bp.boff[6] = acc;
  bp.nheavy = cnt[6];
  bp.ntasks = cnt[PRB_BINS];
  // One warp assignment per 32 rows of bins 0..5, one per hub chunk.
  int64_t w = 0;
  for (int b = 0; b < PRB_BINS; b++) {
    bp.wstart[b] = w;
    if (b < 6) w += (cnt[b] + 31) / 32;
    else w += bp.ntasks;
  }
  bp.wstart[PRB_BINS] = w;
  MG_TRY(alloc((void **)&bp.rows, sizeof(int32_t) * std::max<int64_t>(acc, 1)));
  MG_TRY(alloc((void **)&bp.hrows, sizeof(int32_t) * std::max<int64_t>(bp.nheavy, 1)));
  MG_TRY(alloc((void **)&bp.hbase, sizeof(int32_t) * (bp.nheavy + 1)));
  MG_TRY(alloc((void **)&bp.hcount, sizeof(int32_t) * std::max<int64_t>(bp.nheavy, 1)));
  MG_TRY(alloc((void **)&bp.hpart, sizeof(Comp) * std::max<int64_t>(bp.ntasks, 1)));
  MG_TRY(alloc((void **)&bp.hcontrib, sizeof(double) * 2 * std::max<int64_t>(bp.nheavy, 1)));
  MG_TRY(alloc((void **)&bp.grab, sizeof(int32_t)));
  MG_CUDA_TRY(cudaMemsetAsync(bp.grab, 0, sizeof(int32_t), s));
  MG_CUDA_TRY(cudaMemsetAsync(bp.hcount, 0, sizeof(int32_t) * std::max<int64_t>(bp.nheavy, 1), s));
  MG_CUDA_TRY(cudaMemcpyAsync(dboff, bp.boff, sizeof(int64_t) * (PRB_BINS + 1), cudaMemcpyHostToDevice, s));
  prb_scatter_kernel<<<(unsigned)nchunks, PRB_NT, 0, s>>>(off, n, counts, dboff, bp.rows, bp.hrows, heavy);
  prb_hubs_kernel<<<1, PRB_NT, 0, s>>>(off, bp.hrows, bp.nheavy, bp.hbase);
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaFreeAsync(counts, s));
  return MG_OK;
}

// A failed build releases what it had allocated.
mg_status bin_plan_build(cudaStream_t s, const int32_t *off, int64_t n, mg::BinPlan &bp, int32_t heavy) {
  bp = mg::BinPlan();
  const mg_status st = bin_plan_build_impl(s, off, n, bp, heavy);
  if (st != MG_OK) bin_plan_release(s, bp);
  return st;
}

void bin_plan_release(cudaStream_t s, mg::BinPlan &bp) {
  for (void *q : {(void *)bp.rows, (void *)bp.hrows, (void *)bp.hbase, (void *)bp.hcount, (void *)bp.hpart,
                  (void *)bp.hcontrib, (void *)bp.grab})
    if (q) cudaFreeAsync(q, s);
  bp = mg::BinPlan();
}

// Degree-binned plan of the CSC (forward gather) or the CSR (adjoint, row sums).
static mg_status get_bin_plan(mg_graph *g, bool csr, mg::BinPlan **out) {
  using namespace mg;
  PlanSet *ps = plans_of(g);
  BinPlan &bp = csr ? ps->bcsr : ps->bcsc;
  bool &ok = csr ? ps->bcsr_ok : ps->bcsc_ok;
  if (!ok) {
    MG_TRY(bin_plan_build(g->stream, csr ? g->ro : g->co, g->n, bp));
    ok = true;
  }
  *out = &bp;
  return MG_OK;
}

// Column cache of the forward gather (built once per graph): the vertices of
// largest out-degree, at most `cap` of them, with every vertex of degree >= T
// for the smallest T that fits.
static mg_status get_hub_cache(mg_graph *g, int32_t cap, mg::HubCache **out);

static mg::PrbArgs prb_args_of(const mg_graph *g, const mg::BinPlan &bp, bool csr, const float *wts) {
  mg::PrbArgs p;
  p.off = csr ? g->ro : g->co;
  p.idx = csr ? g->ci : g->ri;
  p.wts = wts;
  p.rows = bp.rows;
  p.hrows = bp.hrows;
  p.hbase = bp.hbase;
  p.hcount = bp.hcount;
  p.hpart = bp.hpart;
  p.hcontrib = bp.hcontrib;
  for (int b = 0; b <= mg::PRB_BINS; b++) {
    p.boff[b] = bp.boff[b];
    p.wstart[b] = bp.wstart[b];
  }
  p.nheavy = bp.nheavy;
  p.grab = nullptr;
  return p;
}

namespace mg {

// Per-row inputs of the row update.
struct RowIn {
  float vold;  // previous iterate
  float s;     // row sum s_r (0: dangling)
  double t;    // teleport entry
  float w;     // adjoint right-hand side
};

// Shared arguments of the gather-based solvers (forward and adjoint).
struct SolveArgs {
  const int32_t *off, *idx;   // adjacency gathered over (CSC forward, CSR adjoint)
  const float *wts;           // its edge weights (nullptr unweighted)
  const int32_t *tx, *ty;
  int32_t ntiles;
  int64_t n;
  int32_t *carry_row, *head_row;
  Comp *carry_val, *head_val;
  float *v0, *v1;             // iterate ping-pong (x forward, lambda adjoint)
  float *g0, *g1;             // gathered values ping-pong (x/s forward; unused adjoint)
  const float *srow;          // s_u, 0 for dangling
  const float *tele;          // teleport (nullptr: uniform tn)
  const float *wvec;          // adjoint right-hand side dL/dx (nullptr forward)
  int32_t soff;               // row sums are the gathered adjacency's degrees (read from its offsets)
  int32_t ri_srow, ri_tele, ri_wvec;  // stage slots of the per-row arrays (-1: not staged; slot 0: iterate)
  double tn, alpha, tol;
  int32_t max_iter;
  int32_t adjoint;
  double *part1, *part2;      // per-CTA FP64 partials of the two kernels
  int32_t grid1, grid2;
  const int32_t *hslot;       // shared-memory column cache: slot of each vertex (nullptr: no cache)
  int32_t gswz;               // 1: x/s of vertex v lives at g[seg_swz(v)] (segmented gather)
  const int32_t *vpos;        // position of each row's x in v0 / v1 (nullptr: the row itself)
  float *gh0, *gh1;           // cached columns' gathered values, ping-pong with g0/g1
  int32_t nhub;               // cached columns
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

__device__ __forceinline__ double tele_of(const SolveArgs &a, int64_t r) {
  return a.tele ? (double)a.tele[r] : a.tn;
}

// Per-row update. Forward: x' = alpha (acc + d t) + (1 - alpha) t, g' = x'/s.
// Adjoint: lambda' = w + alpha * (s > 0 ? acc / s : t.lambda). Partials: |change|
// and (forward) dangling mass of x' / (adjoint) t . lambda'.
struct RowUpdate {
  const SolveArgs *a;
  const float *vold;
  float *vnew, *gnew;
  double scal;  // forward: dangling mass d of the current iterate; adjoint: t.lambda
  double resid = 0.0, red2 = 0.0;
  float *ghnew = nullptr;  // forward with the column cache: its copy of gnew

  __device__ __forceinline__ void apply(int32_t r, Comp v, const RowIn &in) {
    const double acc = (double)v.hi + (double)v.lo;
    const double s = (double)in.s;
    double nv;
    if (!a->adjoint) {
      nv = a->alpha * (acc + scal * in.t) + (1.0 - a->alpha) * in.t;
      float gv = 0.f;
      if (s > 0.0) gv = (float)(nv / s);
      else red2 += nv;
      gnew[a->gswz ? seg_swz(r) : r] = gv;
      if (ghnew) {
        const int32_t sl = __ldg(a->hslot + r);
        if (sl >= 0) ghnew[sl] = gv;
      }
    } else {
      nv = (double)in.w + a->alpha * (s > 0.0 ? acc / s : scal);
      red2 += in.t * nv;
    }
    const float nf = (float)nv;
    resid += fabs((double)nf - (double)in.vold);
    vnew[r] = nf;
  }
  // Row inputs from global memory (rows finished by the fix-up kernel).
  __device__ __forceinline__ void operator()(int32_t r, Comp v) {
    RowIn in;
    in.vold = vold[r];
    in.s = a->soff ? (float)(a->off[r + 1] - a->off[r]) : a->srow[r];
    in.t = tele_of(*a, r);
    in.w = a->wvec ? a->wvec[r] : 0.f;
    apply(r, v, in);
  }
  // Row inputs from the staged tile.
  template <typename Stage>
  __device__ __forceinline__ void operator()(int32_t r, Comp v, const Stage &st) {
    const int j = r - st.coord[4];
    RowIn in;
    in.vold = st.rows[0][j];
    in.s = a->soff ? (float)(st.raw[j + 1] - st.raw[j]) : st.rows[a->ri_srow][j];
    in.t = a->ri_tele >= 0 ? (double)st.rows[a->ri_tele][j] : a->tn;
    in.w = a->ri_wvec >= 0 ? st.rows[a->ri_wvec][j] : 0.f;
    apply(r, v, in);
  }
};

__device__ __forceinline__ bool solve_skip(const SolveArgs &a) {
  if (vload(&a.ctl->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return true;
  }
  return false;
}

__device__ __forceinline__ PrgGraph prg_graph_of(const SolveArgs &a) {
  PrgGraph g{a.off, a.idx, a.wts, a.tx, a.ty, a.ntiles, a.n, a.carry_row, a.head_row, a.carry_val, a.head_val,
             {nullptr, nullptr, nullptr, nullptr}};
  return g;
}

template <bool WEIGHTED, int NR>
__global__ void __launch_bounds__(PRG_NT) solve_gather_kernel(SolveArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PrgSmem<WEIGHTED, NR> &sm = *reinterpret_cast<PrgSmem<WEIGHTED, NR> *>(smem_raw);
  __shared__ double s_red[PRG_NT / 32 + 1];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *vold = cur ? a.v1 : a.v0;
  const float *__restrict__ gold = a.adjoint ? vold : (cur ? a.g1 : a.g0);
  RowUpdate up{&a, vold, cur ? a.v0 : a.v1, cur ? a.g0 : a.g1, vload(&c->dprev[1])};
  PrgGraph pg = prg_graph_of(a);
  pg.rowsrc[0] = vold;
  if (a.ri_srow >= 0) pg.rowsrc[a.ri_srow] = a.srow;
  if (a.ri_tele >= 0) pg.rowsrc[a.ri_tele] = a.tele;
  if (a.ri_wvec >= 0) pg.rowsrc[a.ri_wvec] = a.wvec;
  const bool ok = prg_run<WEIGHTED, NR>(sm, pg, [&](int32_t col) { return __ldg(gold + col); }, up);
  if (!ok && threadIdx.x == 0) {
    c->status = MG_ERR_TIMEOUT;
    c->done = 1;
  }
  const double r = block_sum<PRG_NT>(up.resid, s_red);
  const double d = block_sum<PRG_NT>(up.red2, s_red);
  if (threadIdx.x == 0) {
    a.part1[2 * blockIdx.x] = r;
    a.part1[2 * blockIdx.x + 1] = d;
  }
}

// Last CTA of an iteration: fixed-order FP64 reduction of the per-CTA partials
// (and of the hub contributions), then the convergence decision.
template <int NT = PRG_NT>
__device__ void solve_iteration_end(const SolveArgs &a, int cur, const double *hcontrib, int64_t nheavy,
                                    double *s_red) {
  DevCtl *c = a.ctl;
  double r = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < a.grid1; i += blockDim.x) {
    r += a.part1[2 * i];
    d += a.part1[2 * i + 1];
  }
  for (int i = threadIdx.x; i < a.grid2; i += blockDim.x) {
    r += a.part2[2 * i];
    d += a.part2[2 * i + 1];
  }
  for (int64_t i = threadIdx.x; i < nheavy; i += blockDim.x) {
    r += __ldcg(hcontrib + 2 * i);
    d += __ldcg(hcontrib + 2 * i + 1);
  }
  r = block_sum<NT>(r, s_red);
  d = block_sum<NT>(d, s_red);
  if (threadIdx.x == 0) {
    const int lvl = c->level + 1;
    trace_level(c, lvl - 1, MG_DIR_PUSH, a.n, 0, r);
    c->level = lvl;
    c->dsum[0] = r;
    c->dprev[1] = d;
    c->cur = cur ^ 1;
    c->blocks_done = 0;
    const double thr = a.adjoint ? a.tol * c->dprev[2] : a.tol;  // adjoint: relative to ||w||_1
    const bool done = r < thr || lvl >= a.max_iter || c->status != 0;
    __threadfence();
    c->done = done ? 1 : 0;
    if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
  }
}

// One whole iteration of the degree-binned solver.
template <bool WEIGHTED>
__global__ void __launch_bounds__(PRB_NT, PRB_MIN_BLOCKS) solve_binned_kernel(SolveArgs a, PrbArgs p) {
  __shared__ double s_red[PRB_NT / 32 + 1];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *vold = cur ? a.v1 : a.v0;
  const float *__restrict__ gold = a.adjoint ? vold : (cur ? a.g1 : a.g0);
  float *vnew = cur ? a.v0 : a.v1, *gnew = cur ? a.g0 : a.g1;
  const double scal = vload(&c->dprev[1]);
  RowUpdate up{&a, vold, vnew, gnew, scal};
  auto hub = [&](int64_t h, int32_t row, Comp v) {
    RowUpdate hu{&a, vold, vnew, gnew, scal};
    hu(row, v);
    p.hcontrib[2 * h] = hu.resid;
    p.hcontrib[2 * h + 1] = hu.red2;
    __threadfence();
  };
  prb_run<WEIGHTED>(p, [&](int32_t col) { return __ldg(gold + col); }, up, hub);
  const double r = block_sum<PRB_NT>(up.resid, s_red);
  const double d = block_sum<PRB_NT>(up.red2, s_red);
  if (threadIdx.x == 0) {
    a.part1[2 * blockIdx.x] = r;
    a.part1[2 * blockIdx.x + 1] = d;
  }
  if (last_block(&c->blocks_done)) {
    if (threadIdx.x == 0 && p.grab) *p.grab = 0;
    solve_iteration_end(a, cur, p.hcontrib, p.nheavy, s_red);
  }
}

// One whole iteration of the degree-binned solver with the column cache: every
// CTA first copies the cached columns' gathered values into shared memory. One
// CTA of 1024 threads per SM, so the SM's cache is one copy. Measured on R-MAT
// s22 with the dynamic schedule (us per iteration): 1024 threads x 1 CTA with
// 24K / 32K / 40K / 50K columns 514 / 500 / 495 / 665 (L1 starves), 768 x 1 with
// 40K 545, 640 x 2 with 20K 513.
#ifndef PRB_HUB_THREADS
#define PRB_HUB_THREADS 1024
#endif
#ifndef PRB_HUB_MINB
#define PRB_HUB_MINB 1
#endif
// Columns cached per CTA: the rest of the SM's shared memory stays L1 for the
// uncached gathers.
#ifndef PRB_HUB_CAP
#define PRB_HUB_CAP 40960
#endif
// Rounds of the warp-per-row gather sized to the row's tail (prb_warp_range's
// ADAPT) in the column-cache kernel. Measured on R-MAT s22 (us per iteration,
// static schedule): 640 threads with ADAPT 591, 768 with ADAPT 628, 768 without
// 599, 640 without 774.
#ifndef PRB_HUB_ADAPT
#define PRB_HUB_ADAPT true
#endif
constexpr int PRB_HUB_NT = PRB_HUB_THREADS;

template <bool WEIGHTED>
__global__ void __launch_bounds__(PRB_HUB_NT, PRB_HUB_MINB) solve_binned_hub_kernel(SolveArgs a, PrbArgs p) {
  extern __shared__ __align__(16) float s_hub[];
  __shared__ double s_red[PRB_HUB_NT / 32 + 1];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *vold = cur ? a.v1 : a.v0;
  const float *__restrict__ gold = cur ? a.g1 : a.g0;
  const float *ghold = cur ? a.gh1 : a.gh0;
  float *vnew = cur ? a.v0 : a.v1, *gnew = cur ? a.g0 : a.g1, *ghnew = cur ? a.gh0 : a.gh1;
  const int32_t nh4 = a.nhub >> 2;
  for (int32_t i = threadIdx.x; i < nh4; i += PRB_HUB_NT)
    reinterpret_cast<float4 *>(s_hub)[i] = __ldcg(reinterpret_cast<const float4 *>(ghold) + i);
  for (int32_t i = 4 * nh4 + threadIdx.x; i < a.nhub; i += PRB_HUB_NT) s_hub[i] = __ldcg(ghold + i);
  __syncthreads();
  const double scal = vload(&c->dprev[1]);
  RowUpdate up{&a, vold, vnew, gnew, scal};
  up.ghnew = ghnew;
  auto hub = [&](int64_t h, int32_t row, Comp v) {
    RowUpdate hu{&a, vold, vnew, gnew, scal};
    hu.ghnew = ghnew;
    hu(row, v);
    p.hcontrib[2 * h] = hu.resid;
    p.hcontrib[2 * h + 1] = hu.red2;
    __threadfence();
  };
  prb_run<WEIGHTED, PRB_HUB_ADAPT>(p, [&](int32_t col) { return col < 0 ? s_hub[col & 0x7fffffff] : __ldg(gold + col); }, up,
                    hub);
  const double r = block_sum<PRB_HUB_NT>(up.resid, s_red);
  const double d = block_sum<PRB_HUB_NT>(up.red2, s_red);
  if (threadIdx.x == 0) {
    a.part1[2 * blockIdx.x] = r;
    a.part1[2 * blockIdx.x + 1] = d;
  }
  if (last_block(&c->blocks_done)) {
    if (threadIdx.x == 0 && p.grab) *p.grab = 0;
    solve_iteration_end<PRB_HUB_NT>(a, cur, p.hcontrib, p.nheavy, s_red);
  }
}

// Phase 1 of a segmented iteration (pr_segment.cuh): the hub rows' fragments,
// block by block, out of shared-memory copies of x/s; each fragment's sum goes to
// its slot in hpart. Phase 2, solve_rows_kernel launched after this kernel,
// finishes the hub rows from those sums, runs the other rows and ends the
// iteration. One CTA of SEG_NT threads per SM (the plan's ranges are cut for that
// grid).
constexpr int SEG_NT = 1024;

template <bool WEIGHTED>
__global__ void __launch_bounds__(SEG_NT, 1) solve_segment_kernel(SolveArgs a, PrbArgs p, SegArgs sg) {
  extern __shared__ __align__(128) float s_buf[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int32_t s_next[2];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *__restrict__ gold = cur ? a.g1 : a.g0;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  auto fin = [&](const int2 &e, const Comp &acc) {
    if (e.x >= 0) p.hpart[e.x] = acc;
  };
  uint32_t phase = 0;
  bool ok = true;
  seg_phase<WEIGHTED>(sg, gold, s_buf, &s_bar, s_next, phase, ok, fin);
  if (!ok) {
    c->status = MG_ERR_TIMEOUT;
    c->done = 1;
  }
}

// Phase 2 of a segmented iteration: the hub rows from phase 1's fragment sums (a
// warp per hub: lanes strided over the sums, then a fixed pairing tree), then the
// other rows from their sliced ELL (a lane per row, groups from a counter), with
// the most-gathered columns in shared memory. The iterate and the per-row data
// are in the solve's position order (SegPlan::ppos); the last CTA ends the
// iteration.
template <bool WEIGHTED>
__global__ void __launch_bounds__(SEG_NT, 1) solve_rows_kernel(SolveArgs a, PrbArgs p, SegArgs sg) {
  extern __shared__ __align__(16) float s_hub[];
  __shared__ double s_red[SEG_NT / 32 + 1];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *vold = cur ? a.v1 : a.v0;
  const float *__restrict__ gold = cur ? a.g1 : a.g0;
  const float *ghold = cur ? a.gh1 : a.gh0;
  float *vnew = cur ? a.v0 : a.v1, *gnew = cur ? a.g0 : a.g1, *ghnew = cur ? a.gh0 : a.gh1;
  const int32_t nh4 = a.nhub >> 2;
  for (int32_t i = threadIdx.x; i < nh4; i += SEG_NT)
    reinterpret_cast<float4 *>(s_hub)[i] = __ldcg(reinterpret_cast<const float4 *>(ghold) + i);
  for (int32_t i = 4 * nh4 + threadIdx.x; i < a.nhub; i += SEG_NT) s_hub[i] = __ldcg(ghold + i);
  __syncthreads();
  const double scal = vload(&c->dprev[1]);
  double resid = 0.0, red2 = 0.0;
  // Row update at position `pos` (row r): x' = alpha (acc + d t) + (1 - alpha) t,
  // x'/s into the gathered vector (not for dangling rows: never gathered), |dx|
  // and dangling mass into this thread's partials.
  auto update = [&](int64_t pos, int32_t r, Comp v) {
    const double acc = (double)v.hi + (double)v.lo;
    const double t = sg.pt ? (double)sg.pt[pos] : a.tn;
    const double s = (double)sg.ps[pos];
    const double nv = a.alpha * (acc + scal * t) + (1.0 - a.alpha) * t;
    if (s > 0.0) {
      const float gv = (float)(nv / s);
      gnew[seg_swz(r)] = gv;
      const int32_t sl = sg.pslot[pos];
      if (sl >= 0) ghnew[sl] = gv;
    } else {
      red2 += nv;
    }
    const float nf = (float)nv;
    resid += fabs((double)nf - (double)vold[pos]);
    vnew[pos] = nf;
  };
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (SEG_NT / 32);
  const int64_t hub0 = sg.nrgroups * 32;
  for (int64_t h = (int64_t)blockIdx.x * (SEG_NT / 32) + (threadIdx.x >> 5); h < p.nheavy; h += nw) {
    const int32_t fb = p.hbase[h], nfr = p.hbase[h + 1] - fb;
    const float2 *parts = reinterpret_cast<const float2 *>(p.hpart) + fb;
    Comp t{0.f, 0.f};
    for (int32_t k = lane; k < nfr; k += 32) {
      const float2 v = parts[k];  // written by the previous kernel
      comp_add(t, Comp{v.x, v.y});
    }
    group_comp_reduce<32>(t);
    if (lane == 0) update(hub0 + h, p.hrows[h], t);
  }
  // Rows without in-edges (the last groups of the degree order) take only the
  // teleport and dangling terms: one coalesced pass over their positions, outside
  // the group counter.
  for (int64_t pos = sg.nrgroups_e * 32 + (int64_t)blockIdx.x * SEG_NT + threadIdx.x; pos < sg.nrgroups * 32;
       pos += (int64_t)gridDim.x * SEG_NT) {
    const int32_t r = sg.rrow[pos];
    if (r >= 0) update(pos, r, Comp{0.f, 0.f});
  }
  auto gather = [&](int32_t col) { return col < 0 ? s_hub[col & 0x7fffffff] : __ldg(gold + col); };
  // Short groups (depth <= SEG_SHORT; rows of a few edges, most of the groups that
  // hold an edge): a fixed share per warp, two groups at a time with their loads
  // issued together, no counter and no header round trip in between.
  {
    const int64_t wg = (int64_t)blockIdx.x * (SEG_NT / 32) + (threadIdx.x >> 5);
    for (int64_t ga = sg.nrgroups_l + 2 * wg; ga < sg.nrgroups_e; ga += 2 * nw) {
      const int64_t gb = ga + 1 < sg.nrgroups_e ? ga + 1 : -1;
      const int64_t pa = ga * 32 + lane, pb = gb * 32 + lane;
      const int32_t ra = sg.rrow[pa], rb = gb >= 0 ? sg.rrow[pb] : -1;
      const int64_t a0 = sg.rgofs[ga], a1 = sg.rgofs[ga + 1];
      const int64_t b0 = gb >= 0 ? sg.rgofs[gb] : 0, b1 = gb >= 0 ? sg.rgofs[gb + 1] : 0;
      Comp va, vb;
      sell_short2<WEIGHTED>(sg.ridx + a0 + lane, WEIGHTED ? sg.rwts + a0 + lane : nullptr, (int32_t)((a1 - a0) >> 5),
                            sg.ridx + b0 + lane, WEIGHTED ? sg.rwts + b0 + lane : nullptr, (int32_t)((b1 - b0) >> 5),
                            gather, va, vb);
      if (ra >= 0) update(pa, ra, va);
      if (rb >= 0) update(pb, rb, vb);
    }
  }
  for (;;) {
    int32_t gi = 0;
    if (lane == 0) gi = atomicAdd(sg.rgrab, 1);
    gi = __shfl_sync(FULL, gi, 0);
    if (gi >= sg.nrgroups_l) break;
    const int32_t r = sg.rrow[(int64_t)gi * 32 + lane];
    const int64_t s0 = sg.rgofs[gi];
    const int32_t depth = (int32_t)((sg.rgofs[gi + 1] - s0) >> 5);
    const Comp acc = sell_walk<WEIGHTED, WEIGHTED ? 4 : SEG_U>(sg.ridx + s0 + lane,
                                                              WEIGHTED ? sg.rwts + s0 + lane : nullptr, depth, gather);
    if (r >= 0) update((int64_t)gi * 32 + lane, r, acc);
  }
  const double rr = block_sum<SEG_NT>(resid, s_red);
  const double d = block_sum<SEG_NT>(red2, s_red);
  if (threadIdx.x == 0) {
    a.part1[2 * blockIdx.x] = rr;
    a.part1[2 * blockIdx.x + 1] = d;
  }
  if (last_block(&c->blocks_done)) {
    if (threadIdx.x == 0) *sg.rgrab = 0;
    solve_iteration_end<SEG_NT>(a, cur, nullptr, 0, s_red);
  }
}

// Column-cache set-up kernels.
// Out-degree histogram (bins 0..65535, the last one collecting every larger
// degree): small degrees are counted in shared memory first, since most vertices
// share a handful of small-degree bins.
constexpr int HUB_SMEM_BINS = 4096;

__global__ void __launch_bounds__(256) hub_hist_kernel(const int32_t *__restrict__ ro, int64_t n, unsigned *hist) {
  __shared__ unsigned sh[HUB_SMEM_BINS];
  for (int i = threadIdx.x; i < HUB_SMEM_BINS; i += 256) sh[i] = 0;
  __syncthreads();
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = min(ro[v + 1] - ro[v], 65535);
    if (d < HUB_SMEM_BINS) atomicAdd(sh + d, 1u);
    else atomicAdd(hist + d, 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < HUB_SMEM_BINS; i += 256)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

__global__ void hub_slot_kernel(const int32_t *__restrict__ ro, int64_t n, int32_t thr, int32_t cap, int32_t *slot,
                                int32_t *hv, unsigned *count) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    int32_t sl = -1;
    if (ro[v + 1] - ro[v] >= thr) {
      const unsigned t = atomicAdd(count, 1u);
      if ((int32_t)t < cap) {
        sl = (int32_t)t;
        hv[sl] = (int32_t)v;
      }
    }
    slot[v] = sl;
  }
}

__global__ void hub_remap_kernel(const int32_t *__restrict__ ri, int64_t m, const int32_t *__restrict__ slot,
                                 int32_t *cidx, int32_t swz = 0) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m + 8; k += (int64_t)gridDim.x * blockDim.x) {
    if (k >= m) {
      cidx[k] = 0;
      continue;
    }
    const int32_t c = ri[k];
    const int32_t sl = slot[c];
    cidx[k] = sl >= 0 ? (int32_t)((uint32_t)sl | 0x80000000u) : (swz ? seg_swz(c) : c);
  }
}

__global__ void hub_fill_kernel(const int32_t *__restrict__ hv, int32_t K, const float *__restrict__ g, float *gh,
                                int32_t swz) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < K; i += gridDim.x * blockDim.x)
    gh[i] = g[swz ? seg_swz(hv[i]) : hv[i]];
}

struct RowSumStore {
  float *s;
  __device__ __forceinline__ void operator()(int32_t r, Comp v) { s[r] = v.hi + v.lo; }
};

// Row sums s_u of the weighted CSR through the binned gather (unit gathered values).
__global__ void __launch_bounds__(PRB_NT) rowsum_binned_kernel(PrbArgs p, float *s) {
  RowSumStore st{s};
  prb_run<true>(p, [](int32_t) { return 1.0f; }, st, [&](int64_t, int32_t row, Comp v) { s[row] = v.hi + v.lo; });
}

__global__ void __launch_bounds__(PRG_NT) solve_fixup_kernel(SolveArgs a) {
  __shared__ double s_red[PRG_NT / 32 + 1];
  if (solve_skip(a)) return;
  DevCtl *c = a.ctl;
  const int cur = vload(&c->cur);
  const float *vold = cur ? a.v1 : a.v0;
  RowUpdate up{&a, vold, cur ? a.v0 : a.v1, cur ? a.g0 : a.g1, vload(&c->dprev[1])};
  for (int64_t t = (int64_t)blockIdx.x * PRG_NT + threadIdx.x; t < a.ntiles; t += (int64_t)gridDim.x * PRG_NT)
    prg_fixup_tile((int32_t)t, a.carry_row, a.carry_val, a.head_row, a.head_val, up);
  {
    const double r = block_sum<PRG_NT>(up.resid, s_red);
    const double d = block_sum<PRG_NT>(up.red2, s_red);
    if (threadIdx.x == 0) {
      a.part2[2 * blockIdx.x] = r;
      a.part2[2 * blockIdx.x + 1] = d;
    }
  }
  if (last_block(&c->blocks_done)) solve_iteration_end(a, cur, nullptr, 0, s_red);
}

// Initial iterate. Forward: x0 = t, g0 = t/s; partial sums of the dangling mass.
// Adjoint: lambda0 = w; partial sums of t . w.
__global__ void __launch_bounds__(256) solve_init_kernel(SolveArgs a) {
  __shared__ double s_red[256 / 32 + 1];
  double acc = 0.0, wabs = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double t = tele_of(a, i);
    if (!a.adjoint) {
      const double s = (double)a.srow[i];
      a.v0[a.vpos ? a.vpos[i] : i] = (float)t;
      const int64_t gi = a.gswz ? seg_swz((int32_t)i) : i;
      if (s > 0.0) a.g0[gi] = (float)(t / s);
      else {
        a.g0[gi] = 0.f;
        acc += (double)(float)t;
      }
    } else {
      a.v0[i] = a.wvec[i];
      acc += t * (double)a.wvec[i];
      wabs += fabs((double)a.wvec[i]);
    }
  }
  acc = block_sum<256>(acc, s_red);
  wabs = block_sum<256>(wabs, s_red);
  if (threadIdx.x == 0) {
    a.part1[2 * blockIdx.x] = wabs;
    a.part1[2 * blockIdx.x + 1] = acc;
  }
}

__global__ void __launch_bounds__(256) solve_init_reduce_kernel(SolveArgs a, int32_t ginit) {
  __shared__ double s_red[256 / 32 + 1];
  double d = 0.0, wabs = 0.0;
  for (int i = threadIdx.x; i < ginit; i += 256) {
    wabs += a.part1[2 * i];
    d += a.part1[2 * i + 1];
  }
  d = block_sum<256>(d, s_red);
  wabs = block_sum<256>(wabs, s_red);
  if (threadIdx.x == 0) {
    DevCtl *c = a.ctl;
    c->dprev[1] = d;
    c->dprev[2] = wabs;  // adjoint: ||w||_1, the scale of the relative stopping rule
    c->level = 0;
    c->cur = 0;
    c->iter_cap = a.max_iter;
    c->done = a.max_iter <= 0 ? 1 : 0;
  }
}

// Row sums and teleport entries of a segmented solve in its position order.
__global__ void seg_pos_rows_kernel(SolveArgs a, const int32_t *__restrict__ prow, int64_t npos, float *ps,
                                    float *pt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npos; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = prow[i];
    float sv = 0.f, tv = 0.f;
    if (r >= 0) {
      sv = a.soff ? (float)(a.off[r + 1] - a.off[r]) : a.srow[r];
      if (pt) tv = a.tele[r];
    }
    ps[i] = sv;
    if (pt) pt[i] = tv;
  }
}

// x in row order from a segmented solve's position order.
__global__ void seg_unpermute_kernel(const float *__restrict__ v, const int32_t *__restrict__ ppos, int64_t n,
                                     float *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = v[ppos[i]];
}

// Row sums s_u of the CSR (outdeg unweighted; sum of weights otherwise, through
// the same compensated merge-path gather with unit gathered values).
__global__ void outdeg_kernel(const int32_t *__restrict__ ro, int64_t n, float *__restrict__ s) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s[i] = (float)(ro[i + 1] - ro[i]);
}

__global__ void fill_i32_kernel(int32_t *p, int64_t n, int32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace mg

// ---------------------------------------------------------------------------
// Host side of the gather-based solvers.

// Kernel variants of the pipelined gather: edge weights or not, and how many
// per-row arrays the tiles stage (1..4).
using GatherLaunch = void (*)(int grid, cudaStream_t st, const mg::SolveArgs &b);

template <bool W, int NR>
static void launch_gather(int grid, cudaStream_t st, const mg::SolveArgs &b) {
  mg::solve_gather_kernel<W, NR><<<grid, mg::PRG_NT, mg::prg_smem_bytes<W, NR>(), st>>>(b);
}

// Opts a variant into its dynamic shared memory; returns resident CTAs per SM.
template <bool W, int NR>
static int prepare_gather() {
  const int bytes = (int)mg::prg_smem_bytes<W, NR>();
  cudaFuncSetAttribute(mg::solve_gather_kernel<W, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::solve_gather_kernel<W, NR>, mg::PRG_NT, bytes);
  cudaGetLastError();
  return occ;
}

static GatherLaunch gather_variant(bool w, int nr, int *occ) {
  switch (nr + (w ? 8 : 0)) {
    case 1: *occ = prepare_gather<false, 1>(); return launch_gather<false, 1>;
    case 2: *occ = prepare_gather<false, 2>(); return launch_gather<false, 2>;
    case 3: *occ = prepare_gather<false, 3>(); return launch_gather<false, 3>;
    case 4: *occ = prepare_gather<false, 4>(); return launch_gather<false, 4>;
    case 9: *occ = prepare_gather<true, 1>(); return launch_gather<true, 1>;
    case 10: *occ = prepare_gather<true, 2>(); return launch_gather<true, 2>;
    case 11: *occ = prepare_gather<true, 3>(); return launch_gather<true, 3>;
    default: *occ = prepare_gather<true, 4>(); return launch_gather<true, 4>;
  }
}

struct SolvePlan {
  mg::SolveArgs a;
  GatherLaunch gather;  // merge-path variant (use_tma)
  mg::PrbArgs p;        // degree-binned variant (default)
  mg::SegArgs sg;       // segmented variant: phase 1's fragments
  bool weighted;
  bool use_tma;
  bool use_hub;         // degree-binned with the shared-memory column cache
  bool use_seg;         // segmented hub rows + column cache for the rest
  int32_t hub_bytes;    // dynamic shared memory of the column-cache kernel
  int32_t seg_bytes;    // dynamic shared memory of the segmented gather's phase 1 (a column block)
  const int32_t *ppos = nullptr;  // segmented: position of each row's x in v0 / v1
};

template <bool W>
static int hub_occupancy(int32_t bytes) {
  int occ = 0;
  cudaFuncSetAttribute(mg::solve_binned_hub_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::solve_binned_hub_kernel<W>, mg::PRB_HUB_NT, bytes);
  cudaGetLastError();
  return std::max(1, std::min(occ, PRB_HUB_MINB));
}

template <bool W>
static int seg_occupancy(int32_t bytes) {
  int occ = 0;
  cudaFuncSetAttribute(mg::solve_segment_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::solve_segment_kernel<W>, mg::SEG_NT, bytes);
  cudaGetLastError();
  return occ;
}

template <bool W>
static int binned_occupancy() {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::solve_binned_kernel<W>, mg::PRB_NT, 0);
  cudaGetLastError();
  return std::max(1, std::min(occ, 8));
}

static mg_status get_hub_cache(mg_graph *g, int32_t cap, mg::HubCache **out) {
  using namespace mg;
  HubCache &hc = plans_of(g)->hubs;
  if (hc.ok && hc.cap != cap) {  // rebuilt for another capacity
    for (void *q : {(void *)hc.cidx, (void *)hc.slot, (void *)hc.hv}) dev_free(g, q);
    hc = HubCache();
  }
  if (!hc.ok) {
    // leftovers of a build that failed part-way
    for (void *q : {(void *)hc.cidx, (void *)hc.slot, (void *)hc.hv}) dev_free(g, q);
    hc = HubCache();
    const int64_t n = g->n, m = g->m;
    cudaStream_t s = g->stream;
    unsigned *hist = nullptr;
    MG_CUDA_TRY(mg_malloc_async((void **)&hist, sizeof(unsigned) * (65536 + 1), s));
    auto alloc = [&](void **q, size_t bytes) -> mg_status {
      const mg_status st = dev_alloc(g, q, bytes);
      if (st != MG_OK) dev_free(g, hist);
      return st;
    };
    MG_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(unsigned) * (65536 + 1), s));
    hub_hist_kernel<<<g->num_sms * 4, 256, 0, s>>>(g->ro, n, hist);
    std::vector<unsigned> h(65536);
    MG_CUDA_TRY(cudaMemcpyAsync(h.data(), hist, sizeof(unsigned) * 65536, cudaMemcpyDeviceToHost, s));
    MG_CUDA_TRY(cudaStreamSynchronize(s));
    int64_t cum = 0;
    int32_t thr = 65536;
    for (int32_t d = 65535; d >= 1; d--) {
      if (cum + h[d] > cap) break;
      cum += h[d];
      thr = d;
    }
    MG_TRY(alloc((void **)&hc.slot, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    MG_TRY(alloc((void **)&hc.hv, sizeof(int32_t) * std::max<int64_t>(cap, 1)));
    MG_TRY(alloc((void **)&hc.cidx, sizeof(int32_t) * (m + 8)));
    unsigned *count = hist + 65536;
    hub_slot_kernel<<<g->num_sms * 4, 256, 0, s>>>(g->ro, n, thr, cap, hc.slot, hc.hv, count);
    hub_remap_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ri, m, hc.slot, hc.cidx);
    unsigned k = 0;
    MG_CUDA_TRY(cudaMemcpyAsync(&k, count, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    MG_CUDA_TRY(cudaStreamSynchronize(s));
    MG_CUDA_TRY(cudaFreeAsync(hist, s));
    hc.K = (int32_t)std::min<unsigned>(k, (unsigned)cap);
    hc.cap = cap;
    hc.ok = true;
  }
  *out = &hc;
  return MG_OK;
}

// ---- segmented gather plan (pr_segment.cuh) ----
static void seg_plan_release(mg_graph *g, mg::SegPlan &sp) {
  bin_plan_release(g->stream, sp.bins);
  for (void *q : {(void *)sp.sidx, (void *)sp.swts, (void *)sp.ent, (void *)sp.gofs, (void *)sp.pidx,
                  (void *)sp.pwts, (void *)sp.bgrp, (void *)sp.bdense, (void *)sp.cta, (void *)sp.rrow,
                  (void *)sp.rgofs, (void *)sp.ridx, (void *)sp.rwts, (void *)sp.rgrab, (void *)sp.ppos,
                  (void *)sp.prow, (void *)sp.pslot})
    dev_free(g, q);
  sp = mg::SegPlan();
}

static mg_status seg_plan_build(mg_graph *g, int32_t T, int32_t S, bool weighted, const mg::HubCache &hc,
                                mg::SegPlan &sp) {
  using namespace mg;
  const int64_t n = g->n, m = g->m;
  cudaStream_t s = g->stream;
  const int64_t B = (n + S - 1) / S;
  if (B > SEG_MAXB || S % 32 != 0) {
    mg_set_error("segmented gather: %lld column blocks of %d exceed the plan's limit of %d", (long long)B, S,
                 SEG_MAXB);
    return MG_ERR_UNSUPPORTED;
  }
  sp.T = T;
  sp.S = S;
  sp.nblocks = (int32_t)B;
  sp.grid = g->num_sms;
  sp.weighted = weighted;
  MG_TRY(bin_plan_build(s, g->co, n, sp.bins, T));
  const int64_t nh = sp.bins.nheavy;
  auto scratch = [&](void **q, size_t bytes) -> mg_status {
    if (mg_malloc_async(q, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      cudaGetLastError();
      *q = nullptr;
      mg_set_error("segmented gather plan: device allocation of %zu bytes failed", bytes);
      return MG_ERR_OOM;
    }
    return MG_OK;
  };
  struct Tmp {  // plan-build scratch, released on every return
    cudaStream_t s;
    std::vector<void *> p;
    ~Tmp() {
      for (void *q : p)
        if (q) cudaFreeAsync(q, s);
    }
  } tmp{s, {}};
  int32_t *nfr = nullptr, *lencnt = nullptr;
  const size_t nkeys = (size_t)B * SEG_FMAX;
  MG_TRY(scratch((void **)&nfr, sizeof(int32_t) * (size_t)std::max<int64_t>(nh, 1)));
  tmp.p.push_back(nfr);
  MG_TRY(scratch((void **)&lencnt, sizeof(int32_t) * nkeys));
  tmp.p.push_back(lencnt);
  MG_CUDA_TRY(cudaMemsetAsync(lencnt, 0, sizeof(int32_t) * nkeys, s));
  const size_t hsm = sizeof(int32_t) * (size_t)B;
  if (nh > 0) seg_hist_kernel<<<(unsigned)nh, 256, hsm, s>>>(g->co, g->ri, sp.bins.hrows, S, (int32_t)B, nfr, lencnt);
  seg_scan_kernel<<<1, 256, 0, s>>>(nfr, nh, sp.bins.hbase);
  MG_CUDA_TRY(cudaGetLastError());
  std::vector<int32_t> lc(nkeys);
  int32_t nfrag = 0;
  MG_CUDA_TRY(cudaMemcpyAsync(lc.data(), lencnt, sizeof(int32_t) * nkeys, cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaMemcpyAsync(&nfrag, sp.bins.hbase + nh, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  sp.nfrag = nfrag;
  // Slots: per block, fragments longest first, the block's list padded to whole
  // groups of 32. A group's longest fragment (its first slot) sets its ELL depth.
  std::vector<int32_t> cursor(nkeys), bgrp((size_t)B + 1);
  std::vector<int32_t> gdepth;
  int64_t grp = 0;
  for (int64_t b = 0; b < B; b++) {
    bgrp[b] = (int32_t)grp;
    const int64_t s0 = grp * 32;
    int64_t k = 0;
    for (int32_t key = 0; key < SEG_FMAX; key++) {
      const int32_t len = SEG_FMAX - key, cnt = lc[(size_t)b * SEG_FMAX + key];
      cursor[(size_t)b * SEG_FMAX + key] = (int32_t)(s0 + k);
      // depths even: a lane's index words hold two steps (seg_pk)
      for (int64_t kk = (k + 31) / 32 * 32; kk < k + cnt; kk += 32) gdepth.push_back((len + 1) & ~1);
      k += cnt;
    }
    grp += (k + 31) / 32;
  }
  if (grp * 32 > INT32_MAX) {
    mg_set_error("segmented gather plan: %lld fragment slots exceed 2^31", (long long)(grp * 32));
    return MG_ERR_UNSUPPORTED;
  }
  sp.ngroups = grp;
  bgrp[B] = (int32_t)grp;
  std::vector<int64_t> gofs((size_t)grp + 1);
  gofs[0] = 0;
  for (int64_t gi = 0; gi < grp; gi++) gofs[gi + 1] = gofs[gi] + 32 * (int64_t)gdepth[gi];
  sp.nell = gofs[grp];
  const size_t slots = (size_t)std::max<int64_t>(grp * 32, 1);
  // hub partials count fragments
  cudaFreeAsync(sp.bins.hpart, s);
  sp.bins.hpart = nullptr;
  MG_TRY(scratch((void **)&sp.bins.hpart, sizeof(Comp) * (size_t)std::max<int32_t>(nfrag, 1)));
  MG_TRY(dev_alloc(g, (void **)&sp.ent, sizeof(int2) * slots));
  MG_TRY(dev_alloc(g, (void **)&sp.gofs, sizeof(int64_t) * gofs.size()));
  MG_TRY(dev_alloc(g, (void **)&sp.pidx, sizeof(uint16_t) * (size_t)std::max<int64_t>(sp.nell, 2)));
  if (weighted) MG_TRY(dev_alloc(g, (void **)&sp.pwts, sizeof(float) * (size_t)std::max<int64_t>(sp.nell, 1)));
  MG_TRY(dev_alloc(g, (void **)&sp.bgrp, sizeof(int32_t) * bgrp.size()));
  MG_TRY(dev_alloc(g, (void **)&sp.bdense, (size_t)std::max<int64_t>(B, 1)));
  MG_TRY(dev_alloc(g, (void **)&sp.cta, sizeof(int32_t) * (size_t)(sp.grid + 1)));
  MG_TRY(dev_alloc(g, (void **)&sp.sidx, sizeof(int32_t) * (size_t)(m + 8)));
  if (weighted) MG_TRY(dev_alloc(g, (void **)&sp.swts, sizeof(float) * (size_t)(m + 8)));
  int32_t *fsrc = nullptr, *flen = nullptr;
  MG_TRY(scratch((void **)&fsrc, sizeof(int32_t) * slots));
  tmp.p.push_back(fsrc);
  MG_TRY(scratch((void **)&flen, sizeof(int32_t) * slots));
  tmp.p.push_back(flen);
  MG_CUDA_TRY(cudaMemsetAsync(sp.ent, 0xff, sizeof(int2) * slots, s));
  MG_CUDA_TRY(cudaMemsetAsync(sp.pidx, 0xff, sizeof(uint16_t) * (size_t)std::max<int64_t>(sp.nell, 2), s));
  if (weighted) MG_CUDA_TRY(cudaMemsetAsync(sp.pwts, 0, sizeof(float) * (size_t)std::max<int64_t>(sp.nell, 1), s));
  MG_CUDA_TRY(cudaMemcpyAsync(sp.gofs, gofs.data(), sizeof(int64_t) * gofs.size(), cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaMemcpyAsync(sp.bgrp, bgrp.data(), sizeof(int32_t) * bgrp.size(), cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaMemcpyAsync(lencnt, cursor.data(), sizeof(int32_t) * nkeys, cudaMemcpyHostToDevice, s));
  // sidx: every row's indices with the cached columns flagged, then the hub rows
  // regrouped by block (plain indices); swts follows sidx's order
  hub_remap_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ri, m, hc.slot, sp.sidx, 1);
  if (weighted) {
    MG_CUDA_TRY(cudaMemcpyAsync(sp.swts, g->cvals, sizeof(float) * (size_t)m, cudaMemcpyDeviceToDevice, s));
    MG_CUDA_TRY(cudaMemsetAsync(sp.swts + m, 0, sizeof(float) * 8, s));
  }
  if (nh > 0)
    seg_fill_kernel<<<(unsigned)nh, 32, hsm, s>>>(g->co, g->ri, weighted ? (const float *)g->cvals : nullptr,
                                                  sp.bins.hrows, sp.bins.hbase, S, (int32_t)B, lencnt, sp.sidx,
                                                  sp.swts, sp.ent, fsrc, flen);
  if (grp > 0)
    seg_sell_kernel<<<g->num_sms * 8, 256, 0, s>>>(sp.ent, fsrc, flen, sp.gofs, grp, sp.sidx, sp.swts, S, sp.pidx,
                                                   sp.pwts);
  MG_CUDA_TRY(cudaGetLastError());
  // Phase 2's rows (in-degree below T) as sliced ELL, longest first: a counting
  // sort by degree on the host (rows of one degree in id order). Then the iterate
  // positions: phase 2's lanes, then the hubs.
  {
    std::vector<int32_t> co((size_t)n + 1);
    MG_CUDA_TRY(cudaMemcpyAsync(co.data(), g->co, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, s));
    MG_CUDA_TRY(cudaStreamSynchronize(s));
    int32_t dmax = 0;
    for (int64_t r = 0; r < n; r++) {
      const int32_t d = co[r + 1] - co[r];
      if (d < T) dmax = std::max(dmax, d);
    }
    std::vector<int64_t> start((size_t)dmax + 2, 0);
    for (int64_t r = 0; r < n; r++) {
      const int32_t d = co[r + 1] - co[r];
      if (d < T) start[dmax - d + 1]++;
    }
    for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
    const int64_t nrows = start.back();
    sp.nrgroups = (nrows + 31) / 32;
    std::vector<int32_t> rrow((size_t)std::max<int64_t>(sp.nrgroups * 32, 1), -1);
    for (int64_t r = 0; r < n; r++) {
      const int32_t d = co[r + 1] - co[r];
      if (d < T) rrow[start[dmax - d]++] = (int32_t)r;
    }
    std::vector<int64_t> rg((size_t)sp.nrgroups + 1, 0);
    sp.nrgroups_e = 0;
    sp.nrgroups_l = 0;
    for (int64_t gi = 0; gi < sp.nrgroups; gi++) {
      const int32_t r0 = rrow[gi * 32];  // the group's longest row
      rg[gi + 1] = rg[gi] + 32 * (int64_t)(co[r0 + 1] - co[r0]);
      if (co[r0 + 1] > co[r0]) sp.nrgroups_e = gi + 1;
      if (co[r0 + 1] - co[r0] > SEG_SHORT) sp.nrgroups_l = gi + 1;
    }
    sp.nrell = rg[sp.nrgroups];
    sp.npos = sp.nrgroups * 32 + nh;
    // positions: phase 2's lanes (rrow), then the hubs; prow and its inverse ppos
    // are formed on the device
    const size_t nprow = (size_t)std::max<int64_t>(sp.npos, 1), nppos = (size_t)std::max<int64_t>(n, 1);
    MG_TRY(dev_alloc(g, (void **)&sp.rrow, sizeof(int32_t) * rrow.size()));
    MG_TRY(dev_alloc(g, (void **)&sp.rgofs, sizeof(int64_t) * rg.size()));
    MG_TRY(dev_alloc(g, (void **)&sp.ridx, sizeof(int32_t) * (size_t)std::max<int64_t>(sp.nrell, 1)));
    if (weighted) MG_TRY(dev_alloc(g, (void **)&sp.rwts, sizeof(float) * (size_t)std::max<int64_t>(sp.nrell, 1)));
    MG_TRY(dev_alloc(g, (void **)&sp.rgrab, sizeof(int32_t)));
    MG_TRY(dev_alloc(g, (void **)&sp.ppos, sizeof(int32_t) * nppos));
    MG_TRY(dev_alloc(g, (void **)&sp.prow, sizeof(int32_t) * nprow));
    MG_TRY(dev_alloc(g, (void **)&sp.pslot, sizeof(int32_t) * nprow));
    MG_CUDA_TRY(cudaMemsetAsync(sp.rgrab, 0, sizeof(int32_t), s));
    MG_CUDA_TRY(cudaMemsetAsync(sp.ridx, 0xff, sizeof(int32_t) * (size_t)std::max<int64_t>(sp.nrell, 1), s));
    if (weighted) MG_CUDA_TRY(cudaMemsetAsync(sp.rwts, 0, sizeof(float) * (size_t)std::max<int64_t>(sp.nrell, 1), s));
    MG_CUDA_TRY(cudaMemcpyAsync(sp.rrow, rrow.data(), sizeof(int32_t) * rrow.size(), cudaMemcpyHostToDevice, s));
    MG_CUDA_TRY(cudaMemcpyAsync(sp.rgofs, rg.data(), sizeof(int64_t) * rg.size(), cudaMemcpyHostToDevice, s));
    MG_CUDA_TRY(cudaMemsetAsync(sp.ppos, 0xff, sizeof(int32_t) * nppos, s));
    MG_CUDA_TRY(cudaMemsetAsync(sp.prow, 0xff, sizeof(int32_t) * nprow, s));
    if (sp.nrgroups > 0)
      MG_CUDA_TRY(cudaMemcpyAsync(sp.prow, sp.rrow, sizeof(int32_t) * (size_t)(sp.nrgroups * 32),
                                  cudaMemcpyDeviceToDevice, s));
    if (nh > 0)
      MG_CUDA_TRY(cudaMemcpyAsync(sp.prow + sp.nrgroups * 32, sp.bins.hrows, sizeof(int32_t) * (size_t)nh,
                                  cudaMemcpyDeviceToDevice, s));
    if (sp.nrgroups > 0)
      seg_rows_fill_kernel<<<g->num_sms * 8, 256, 0, s>>>(sp.rrow, sp.rgofs, sp.nrgroups, g->co, sp.sidx, sp.swts,
                                                          sp.ridx, sp.rwts);
    if (sp.npos > 0)
      seg_pos_slot_kernel<<<g->num_sms * 4, 256, 0, s>>>(sp.prow, sp.npos, hc.slot, sp.pslot, sp.ppos);
    MG_CUDA_TRY(cudaGetLastError());
    MG_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
  }
  // Dense blocks are staged in shared memory; phase 1's groups are cut into one
  // contiguous range per CTA by estimated cost: sliced-ELL entries (a global
  // gather counting SEG_GLOBAL_FACTOR), a fixed cost per group, and a block load
  // wherever a CTA's range enters a dense block.
  std::vector<uint8_t> dense((size_t)std::max<int64_t>(B, 1), 0);
  std::vector<int32_t> gblock((size_t)grp);
  for (int64_t b = 0; b < B; b++) {
    dense[b] = (gofs[bgrp[b + 1]] - gofs[bgrp[b]]) >= SEG_DENSE ? 1 : 0;
    for (int64_t gi = bgrp[b]; gi < bgrp[b + 1]; gi++) gblock[gi] = (int32_t)b;
  }
  auto gcost = [&](int64_t gi) {
    return 32 * (int64_t)gdepth[gi] * (dense[gblock[gi]] ? 1 : SEG_GLOBAL_FACTOR) + SEG_GROUP_COST;
  };
  // Greedy cut for a cost cap per CTA (a range closes before the group that would
  // pass the cap); the smallest cap that needs at most `grid` ranges is kept.
  std::vector<int32_t> cta((size_t)sp.grid + 1, (int32_t)grp);
  auto cut = [&](int64_t cap, bool write) {
    int64_t acc = 0, start = 0;
    int32_t used = grp > 0 ? 1 : 0;
    if (write) cta[0] = 0;
    for (int64_t gi = 0; gi < grp; gi++) {
      const bool enters = gi == start || gblock[gi] != gblock[gi - 1];
      int64_t c = gcost(gi) + ((enters && dense[gblock[gi]]) ? SEG_LOAD_COST : 0);
      if (acc + c > cap && gi > start) {  // close the range before gi
        if (write && used < sp.grid) cta[used] = (int32_t)gi;
        used++;
        start = gi;
        acc = 0;
        c = gcost(gi) + (dense[gblock[gi]] ? SEG_LOAD_COST : 0);
      }
      acc += c;
    }
    return used;
  };
  int64_t lo = 1, hi = 1;
  for (int64_t gi = 0; gi < grp; gi++) hi += gcost(gi) + SEG_LOAD_COST;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (cut(mid, false) <= sp.grid) hi = mid;
    else lo = mid + 1;
  }
  cut(lo, true);
  MG_CUDA_TRY(cudaMemcpyAsync(sp.bdense, dense.data(), dense.size(), cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaMemcpyAsync(sp.cta, cta.data(), sizeof(int32_t) * cta.size(), cudaMemcpyHostToDevice, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  sp.ok = true;
  return MG_OK;
}

// Segmented plan for (T, S), rebuilt when either changes; a failed build leaves
// nothing behind.
static mg_status get_seg_plan(mg_graph *g, int32_t T, int32_t S, bool weighted, const mg::HubCache &hc,
                              mg::SegPlan **out) {
  mg::SegPlan &sp = plans_of(g)->seg;
  if (!sp.ok || sp.T != T || sp.S != S || sp.weighted != weighted) {
    seg_plan_release(g, sp);
    const mg_status st = seg_plan_build(g, T, S, weighted, hc, sp);
    if (st != MG_OK) {
      seg_plan_release(g, sp);
      return st;
    }
  }
  *out = &sp;
  return MG_OK;
}

// Capacity of the column cache: half of an SM's shared memory per CTA (two CTAs
// of PRB_HUB_NT threads per SM), less the kernel's own static shared memory.
static int32_t hub_cache_limit(mg_graph *g) {
  int per_sm = 0, per_block = 0;
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, g->device);
  cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, g->device);
  cudaGetLastError();
  const int bytes = std::min(per_sm / PRB_HUB_MINB - 2048, per_block - 1024);
  return std::max(0, bytes / 4) & ~63;
}

static int32_t hub_cache_capacity(mg_graph *g) { return std::min(PRB_HUB_CAP, hub_cache_limit(g)); }

// Default shape of the segmented gather: hub rows of at least 512 edges, column
// blocks as wide as the column cache (the kernel then asks for the cached gather's
// shared memory, leaving L1 the same room for phase 2's uncached gathers).
constexpr int32_t SEG_DEFAULT_T = 512;
static int32_t seg_block_default(mg_graph *g) { return std::max<int32_t>(1024, hub_cache_capacity(g) & ~1023); }

// Carves the solver's buffers out of ws_main (every per-vertex array padded to
// n + 8 entries for the widened tile copies), copies the teleport vector and the
// adjoint right-hand side into padded buffers, computes the row sums s_u and picks
// the gather variant.
static mg_status solve_setup(mg_graph *g, bool adjoint, bool weighted, const float *tele_src,
                             const float *wvec_src, int variant, SolvePlan &sp, int32_t hub_cap = -1,
                             int32_t seg_T = 0, int32_t seg_S = 0) {
  using namespace mg;
  const bool use_tma = variant == 1;
  const bool use_seg = variant == 3 && !adjoint && g->n > 0;
  const bool use_hub = (variant == 2 || use_seg) && !adjoint && g->n > 0;
  GatherPlan *plan = nullptr;
  BinPlan *bins = nullptr, *rbins = nullptr;
  HubCache *hubs = nullptr;
  SegPlan *seg = nullptr;
  if (use_hub) MG_TRY(get_hub_cache(g, hub_cap > 0 ? hub_cap : hub_cache_capacity(g), &hubs));
  if (use_tma) MG_TRY(get_plan(g, adjoint, &plan));
  else if (use_seg) {
    MG_TRY(get_seg_plan(g, seg_T > 0 ? seg_T : SEG_DEFAULT_T, seg_S > 0 ? seg_S : seg_block_default(g), weighted,
                        *hubs, &seg));
    bins = &seg->bins;
  } else MG_TRY(get_bin_plan(g, adjoint, &bins));
  if (weighted) MG_TRY(get_bin_plan(g, true, &rbins));
  const int64_t n = g->n;
  // whole 32-entry chunks (seg_swz) and a pad; a segmented solve keeps x in its
  // position order (phase 2's lanes, then the hubs)
  const size_t np = (size_t)std::max<int64_t>((n + 31) & ~(int64_t)31, seg ? seg->npos : 0) + 8;
  const int32_t nt = plan ? plan->ntiles : 1;
  const bool symmetric = (g->flags & MG_GRAPH_SYMMETRIC) != 0;
  SolveArgs &a = sp.a;
  std::memset(&a, 0, sizeof(a));
  a.soff = adjoint ? !weighted : (symmetric && !weighted);
  int nr = 1;
  a.ri_srow = a.soff ? -1 : nr++;
  a.ri_tele = tele_src ? nr++ : -1;
  a.ri_wvec = adjoint ? nr++ : -1;
  int occ = 0;
  sp.use_tma = use_tma;
  sp.use_hub = use_hub && !use_seg;
  sp.use_seg = use_seg;
  sp.hub_bytes = use_hub ? (int32_t)(sizeof(float) * hubs->K) : 0;
  sp.seg_bytes = use_seg ? (int32_t)(sizeof(float) * seg->S) : 0;
  sp.weighted = weighted;
  sp.gather = nullptr;
  if (use_tma) sp.gather = gather_variant(weighted, nr, &occ);
  else if (use_seg) {
    occ = weighted ? seg_occupancy<true>(sp.seg_bytes) : seg_occupancy<false>(sp.seg_bytes);
    if (occ < 1) {
      mg_set_error("segmented gather: a CTA of %d threads with %d bytes of shared memory does not fit an SM", SEG_NT,
                   sp.seg_bytes);
      return MG_ERR_UNSUPPORTED;
    }
    // phase 1's ranges are cut for one CTA per SM; phase 2 runs one CTA per SM too
    int occ2 = 0;
    if (weighted) {
      cudaFuncSetAttribute(solve_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp.hub_bytes);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, solve_rows_kernel<true>, SEG_NT, sp.hub_bytes);
    } else {
      cudaFuncSetAttribute(solve_rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp.hub_bytes);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, solve_rows_kernel<false>, SEG_NT, sp.hub_bytes);
    }
    cudaGetLastError();
    if (occ2 < 1) {
      mg_set_error("segmented gather: the row kernel does not fit an SM with %d bytes of shared memory", sp.hub_bytes);
      return MG_ERR_UNSUPPORTED;
    }
    occ = 1;
  } else if (use_hub) occ = weighted ? hub_occupancy<true>(sp.hub_bytes) : hub_occupancy<false>(sp.hub_bytes);
  else occ = weighted ? binned_occupancy<true>() : binned_occupancy<false>();
  const int g1 = g->num_sms * std::max(1, std::min(occ, 8));
  const int g2 = use_tma ? std::max(1, (nt + PRG_NT - 1) / PRG_NT) : 0;
  const int ginit = g->num_sms * 8;
  const int gp = std::max(std::max(g1, g2), ginit);
  const size_t need = Carve::need({sizeof(float) * np, sizeof(float) * np, sizeof(float) * np, sizeof(float) * np,
                                   sizeof(float) * np, sizeof(float) * np, sizeof(float) * np,
                                   sizeof(int32_t) * (size_t)nt, sizeof(int32_t) * (size_t)nt,
                                   sizeof(Comp) * (size_t)nt, sizeof(Comp) * (size_t)nt,
                                   sizeof(double) * 2 * (size_t)gp, sizeof(double) * 2 * (size_t)gp,
                                   sizeof(float) * (size_t)(use_hub ? hubs->K + 8 : 0),
                                   sizeof(float) * (size_t)(use_hub ? hubs->K + 8 : 0),
                                   sizeof(float) * (size_t)(use_seg ? seg->npos + 8 : 0),
                                   sizeof(float) * (size_t)(use_seg && tele_src ? seg->npos + 8 : 0)});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  a.v0 = cv.take<float>(np);
  a.v1 = cv.take<float>(np);
  a.g0 = cv.take<float>(np);
  a.g1 = cv.take<float>(np);
  float *srow = cv.take<float>(np);
  float *tele = cv.take<float>(np);
  float *wvec = cv.take<float>(np);
  a.carry_row = cv.take<int32_t>(nt);
  a.head_row = cv.take<int32_t>(nt);
  a.carry_val = cv.take<Comp>(nt);
  a.head_val = cv.take<Comp>(nt);
  a.part1 = cv.take<double>(2 * (size_t)gp);
  a.part2 = cv.take<double>(2 * (size_t)gp);
  if (use_hub) {
    a.gh0 = cv.take<float>((size_t)hubs->K + 8);
    a.gh1 = cv.take<float>((size_t)hubs->K + 8);
    a.hslot = hubs->slot;
    a.nhub = hubs->K;
  }
  float *pos_s = use_seg ? cv.take<float>((size_t)seg->npos + 8) : nullptr;
  float *pos_t = use_seg && tele_src ? cv.take<float>((size_t)seg->npos + 8) : nullptr;
  a.n = n;
  a.srow = srow;
  a.tele = tele_src ? tele : nullptr;
  a.wvec = adjoint ? wvec : nullptr;
  a.grid1 = g1;
  a.grid2 = g2;
  a.ctl = g->ctl;
  cudaStream_t s = g->stream;
  if (tele_src) MG_CUDA_TRY(cudaMemcpyAsync(tele, tele_src, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  if (adjoint && wvec_src)
    MG_CUDA_TRY(cudaMemcpyAsync(wvec, wvec_src, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  fill_i32_kernel<<<g->num_sms * 4, 256, 0, s>>>(a.head_row, nt, -1);
  if (!weighted) {
    outdeg_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ro, n, srow);
  } else {
    const PrbArgs rp = prb_args_of(g, *rbins, true, (const float *)g->vals);
    rowsum_binned_kernel<<<g->num_sms * 8, PRB_NT, 0, s>>>(rp, srow);
  }
  a.off = adjoint ? g->ro : g->co;
  a.idx = adjoint ? g->ci : g->ri;
  a.wts = weighted ? (const float *)(adjoint ? g->vals : g->cvals) : nullptr;
  if (plan) {
    a.tx = plan->tx;
    a.ty = plan->ty;
    a.ntiles = plan->ntiles;
  } else {
    sp.p = prb_args_of(g, *bins, adjoint, a.wts);
#if PRB_DYNAMIC
    sp.p.grab = bins->grab;  // the solve kernels' last CTA resets it
#endif
    if (use_seg) {
      sp.p.idx = seg->sidx;
      if (weighted) sp.p.wts = seg->swts;
      sp.p.grab = bins->grab;  // phase 2 always takes items from the counter
      sp.p.wstart[PRB_BINS] = sp.p.wstart[6];  // hub rows are phase 1's, not work items of phase 2
      sp.sg = SegArgs{seg->ent,  seg->gofs, seg->pidx,   seg->pwts,  seg->bgrp,  seg->cta,
                      seg->bdense, (n + 31) & ~(int64_t)31, seg->S, seg->nblocks, seg->rrow, seg->rgofs,
                      seg->ridx, seg->rwts, seg->rgrab, seg->nrgroups, seg->nrgroups_e, seg->nrgroups_l,
                      seg->pslot, pos_s, pos_t};
      a.gswz = 1;
      a.vpos = seg->ppos;
      sp.ppos = seg->ppos;
      if (seg->npos > 0)
        seg_pos_rows_kernel<<<g->num_sms * 4, 256, 0, s>>>(a, seg->prow, seg->npos, pos_s, pos_t);
    } else if (use_hub) {
      sp.p.idx = hubs->cidx;
    }
  }
  MG_CUDA_TRY(cudaGetLastError());
  return MG_OK;
}

// Runs the solver loop described by `sp` (initial iterate set up by the init
// kernels). Returns after the loop; results stay in a.v0/a.v1 at ctl->cur.
static mg_status solve_run(mg_graph *g, SolvePlan &sp, int use_graph, int slot) {
  using namespace mg;
  const SolveArgs &a = sp.a;
  cudaStream_t s = g->stream;
  const int ginit = g->num_sms * 8;
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  solve_init_kernel<<<ginit, 256, 0, s>>>(a);
  solve_init_reduce_kernel<<<1, 256, 0, s>>>(a, ginit);
  if (sp.use_hub || sp.use_seg) {
    const HubCache &hc = plans_of(g)->hubs;
    hub_fill_kernel<<<g->num_sms, 256, 0, s>>>(hc.hv, hc.K, a.g0, a.gh0, a.gswz);
  }
  MG_CUDA_TRY(cudaGetLastError());
  struct Sig {
    SolveArgs a;
    GatherLaunch gl;
    PrbArgs p;
    SegArgs sg;
    int w, tma, hub, seg;
  } sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.a = a;
  sig.gl = sp.gather;
  sig.p = sp.p;
  sig.w = sp.weighted;
  sig.tma = sp.use_tma;
  sig.hub = sp.use_hub;
  sig.seg = sp.use_seg;
  if (sp.use_seg) sig.sg = sp.sg;
  const int g1 = a.grid1, g2 = a.grid2;
  const GatherLaunch gl = sp.gather;
  const PrbArgs p = sp.p;
  const SegArgs sg = sp.sg;
  const bool tma = sp.use_tma, w = sp.weighted, hub = sp.use_hub, seg = sp.use_seg;
  const int32_t hb = sp.hub_bytes, sb = sp.seg_bytes;
  LoopBody body = [a, gl, p, sg, g1, g2, tma, w, hub, seg, hb, sb](cudaStream_t st, cudaGraphConditionalHandle h,
                                                                  int use_cond) {
    SolveArgs b = a;
    b.h = h;
    b.use_cond = use_cond;
    if (tma) {
      gl(g1, st, b);
      solve_fixup_kernel<<<g2, PRG_NT, 0, st>>>(b);
    } else if (seg) {
      // phase 1 (hub fragments), then the other rows and the iteration's end
      if (w) {
        solve_segment_kernel<true><<<g1, SEG_NT, sb, st>>>(b, p, sg);
        solve_rows_kernel<true><<<g1, SEG_NT, hb, st>>>(b, p, sg);
      } else {
        solve_segment_kernel<false><<<g1, SEG_NT, sb, st>>>(b, p, sg);
        solve_rows_kernel<false><<<g1, SEG_NT, hb, st>>>(b, p, sg);
      }
    } else if (hub) {
      if (w) solve_binned_hub_kernel<true><<<g1, PRB_HUB_NT, hb, st>>>(b, p);
      else solve_binned_hub_kernel<false><<<g1, PRB_HUB_NT, hb, st>>>(b, p);
    } else if (w) {
      solve_binned_kernel<true><<<g1, PRB_NT, 0, st>>>(b, p);
    } else {
      solve_binned_kernel<false><<<g1, PRB_NT, 0, st>>>(b, p);
    }
  };
  MG_TRY(run_loop(g, slot, &sig, sizeof(sig), use_graph >= 0, body, (int64_t)a.max_iter + 2));
  return MG_OK;
}

// ---------------------------------------------------------------------------
// REFCOMPAT: the reference program's delta-frontier iteration.
namespace mg {

constexpr int PRR_NT = 256;

struct RefArgs {
  const int32_t *ro, *ci, *co, *ri;
  int32_t both;
  float *x, *xn;
  const float *deg;
  uint8_t *chg;
  uint32_t *inq0, *inq1;
  int32_t *q0, *q1;
  int32_t qcap;
  int64_t n;
  float delta;
  int32_t compensated;
  DevCtl *ctl;
  cudaGraphConditionalHandle h;
  int32_t use_cond;
};

__device__ __forceinline__ void warp_comp_reduce(Comp &c) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Comp d{__shfl_xor_sync(FULL, c.hi, o), __shfl_xor_sync(FULL, c.lo, o)};
    comp_add(c, d);
  }
}

__device__ __forceinline__ void ref_term(Comp &acc, const RefArgs &a, int32_t u) {
  const float t = a.x[u] / a.deg[u];
  if (a.compensated) two_sum_add(acc, t);
  else acc.hi += t;
}

// Gather + apply for a tile of frontier vertices: thread bin (< 32 in-edges)
// sums sequentially, warp bin with a fixed shuffle tree, CTA bin with a fixed
// shared-memory tree, so every sum has a fixed order.
__global__ void __launch_bounds__(PRR_NT) prr_gather_kernel(RefArgs a) {
  __shared__ float s_hi[PRR_NT], s_lo[PRR_NT];
  __shared__ int32_t s_v, s_owner;
  __shared__ int64_t s_sum[PRR_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  const int lane = lane_id();
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * PRR_NT; tile < nin; tile += (int64_t)gridDim.x * PRR_NT) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < nin ? qin[i] : -1;
    int32_t d1 = 0, d2 = 0;
    if (v >= 0) {
      d1 = a.co[v + 1] - a.co[v];
      d2 = a.both ? a.ro[v + 1] - a.ro[v] : 0;
      insp += d1 + d2;
    }
    int32_t deg = d1 + d2;
    Comp acc{0.f, 0.f};
    bool mine = v >= 0 && deg < 32;
    if (mine) {
      for (int32_t e = a.co[v]; e < a.co[v + 1]; e++) ref_term(acc, a, a.ri[e]);
      if (a.both)
        for (int32_t e = a.ro[v]; e < a.ro[v + 1]; e++) ref_term(acc, a, a.ci[e]);
    }
    // CTA bin.
    while (__syncthreads_or(deg >= 2048 && !mine)) {
      if (deg >= 2048 && !mine) s_owner = threadIdx.x;
      __syncthreads();
      const int owner = s_owner;
      if (threadIdx.x == owner) s_v = v;
      __syncthreads();
      const int32_t vv = s_v;
      Comp part{0.f, 0.f};
      for (int32_t e = a.co[vv] + threadIdx.x; e < a.co[vv + 1]; e += PRR_NT) ref_term(part, a, a.ri[e]);
      if (a.both)
        for (int32_t e = a.ro[vv] + threadIdx.x; e < a.ro[vv + 1]; e += PRR_NT) ref_term(part, a, a.ci[e]);
      s_hi[threadIdx.x] = part.hi;
      s_lo[threadIdx.x] = part.lo;
      __syncthreads();
      for (int st = PRR_NT / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
          Comp x{s_hi[threadIdx.x], s_lo[threadIdx.x]};
          comp_add(x, Comp{s_hi[threadIdx.x + st], s_lo[threadIdx.x + st]});
          s_hi[threadIdx.x] = x.hi;
          s_lo[threadIdx.x] = x.lo;
        }
        __syncthreads();
      }
      if (threadIdx.x == owner) {
        acc = Comp{s_hi[0], s_lo[0]};
        mine = true;
      }
      __syncthreads();
    }
    // Warp bin.
    for (;;) {
      const unsigned wm = __ballot_sync(FULL, deg >= 32 && !mine);
      if (!wm) break;
      const int l = __ffs(wm) - 1;
      const int32_t wv = __shfl_sync(FULL, v, l);
      Comp part{0.f, 0.f};
      for (int32_t e = a.co[wv] + lane; e < a.co[wv + 1]; e += 32) ref_term(part, a, a.ri[e]);
      if (a.both)
        for (int32_t e = a.ro[wv] + lane; e < a.ro[wv + 1]; e += 32) ref_term(part, a, a.ci[e]);
      warp_comp_reduce(part);
      if (lane == l) {
        acc = part;
        mine = true;
      }
    }
    if (v >= 0) {
      const float g = acc.hi + acc.lo;
      const float nv = 0.15f + (1.0f - 0.15f) * g;
      a.chg[v] = fabsf(a.x[v] - nv) >= a.delta ? 1 : 0;
      a.xn[v] = nv;
    }
  }
  const int64_t b = block_sum<PRR_NT>(insp, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd((unsigned long long *)&c->edges_inspected, (unsigned long long)b);
}

__global__ void __launch_bounds__(PRR_NT) prr_expand_kernel(RefArgs a) {
  __shared__ ExpandSmem<PRR_NT> sm;
  __shared__ int64_t s_sum[PRR_NT / 32 + 1];
  DevCtl *c = a.ctl;
  if (vload(&c->done)) {
    if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.h, 0u);
    return;
  }
  const int cur = vload(&c->cur);
  const int32_t nin = vload(&c->qlen[cur]);
  const int32_t *qin = cur ? a.q1 : a.q0;
  uint32_t *inq_cur = cur ? a.inq1 : a.inq0;
  uint32_t *inq_next = cur ? a.inq0 : a.inq1;
  int32_t *qout = cur ? a.q0 : a.q1;
  int32_t *qlen_out = &c->qlen[cur ^ 1];
  int64_t insp = 0, nchg = 0;
  const int32_t *ci = a.ci, *ri = a.ri;
  auto claim = [&](int32_t, int32_t u) {
    const uint32_t bit = 1u << (u & 31);
    const bool push = !(atomicOr(inq_next + (u >> 5), bit) & bit);
    warp_append(push, u, qout, qlen_out, a.qcap, &c->overflow);
  };
  for (int64_t tile = (int64_t)blockIdx.x * PRR_NT; tile < nin; tile += (int64_t)gridDim.x * PRR_NT) {
    const int64_t i = tile + threadIdx.x;
    int32_t v = i < nin ? qin[i] : -1;
    if (v >= 0) {
      inq_cur[v >> 5] = 0u;
      a.x[v] = a.xn[v];
      if (a.chg[v]) nchg++;
      else v = -1;
    }
    expand_tile<PRR_NT, 1024>(sm, a.ro, v, insp, [&](int32_t sv, int32_t k) { claim(sv, ci[k]); });
    if (a.both) expand_tile<PRR_NT, 1024>(sm, a.co, v, insp, [&](int32_t sv, int32_t k) { claim(sv, ri[k]); });
  }
  const int64_t b = block_sum<PRR_NT>(nchg, s_sum);
  if (threadIdx.x == 0 && b) atomicAdd((unsigned long long *)&c->vertices_updated, (unsigned long long)b);
  if (last_block(&c->blocks_done) && threadIdx.x == 0) {
    const int32_t nf = vload(&c->qlen[cur ^ 1]);
    const int lvl = c->level + 1;
    c->level = lvl;
    c->qlen[cur] = 0;
    c->cur = cur ^ 1;
    c->blocks_done = 0;
    const bool over = vload(&c->overflow) != 0;
    if (over) c->status = MG_ERR_QUEUE_OVERFLOW;
    const bool done = nf == 0 || lvl >= c->iter_cap || over;
    __threadfence();
    c->done = done ? 1 : 0;
    if (a.use_cond) cudaGraphSetConditional(a.h, done ? 0u : 1u);
  }
}

__global__ void prr_init_kernel(RefArgs a, float *deg, int32_t iter_cap) {
  const int64_t nw = (a.n + 31) >> 5;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    a.x[i] = 0.15f;
    a.q0[i] = (int32_t)i;
    a.chg[i] = 0;
    int32_t d = a.ro[i + 1] - a.ro[i];
    if (a.both) d += a.co[i + 1] - a.co[i];
    deg[i] = (float)d;
    if (i < nw) {
      a.inq0[i] = 0;
      a.inq1[i] = 0;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->qlen[0] = (int32_t)a.n;
    a.ctl->iter_cap = iter_cap;
    a.ctl->done = (a.n == 0 || iter_cap <= 0) ? 1 : 0;
  }
}

}  // namespace mg

static mg_status pagerank_refcompat(mg_graph *g, float *ranks, const mg_pr_opts &o, mg_stats *stats) {
  using namespace mg;
  if (!g->has_csc) {
    mg_set_error("mg_pagerank: the gather over in-edges needs the CSC");
    return MG_ERR_UNSUPPORTED;
  }
  const int64_t n = g->n;
  const int64_t nwords = (n + 31) / 32;
  const size_t need = Carve::need({4 * (size_t)n, 4 * (size_t)n, 4 * (size_t)n, (size_t)n, 4 * (size_t)nwords,
                                   4 * (size_t)nwords, 4 * (size_t)n, 4 * (size_t)n});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  RefArgs a;
  std::memset(&a, 0, sizeof(a));
  float *xws = cv.take<float>(n);
  a.xn = cv.take<float>(n);
  float *deg = cv.take<float>(n);
  a.chg = cv.take<uint8_t>(n);
  a.inq0 = cv.take<uint32_t>(nwords);
  a.inq1 = cv.take<uint32_t>(nwords);
  a.q0 = cv.take<int32_t>(n);
  a.q1 = cv.take<int32_t>(n);
  a.x = o.device_output ? ranks : xws;
  a.deg = deg;
  a.ro = g->ro;
  a.ci = g->ci;
  a.co = g->co;
  a.ri = g->ri;
  a.both = o.directed == 0 ? 1 : 0;
  a.qcap = (int32_t)std::max<int64_t>(n, 1);
  a.n = n;
  a.delta = o.tol > 0 ? (float)o.tol : 0.01f;
  a.compensated = o.compensated >= 0 ? 1 : 0;
  a.ctl = g->ctl;
  cudaStream_t s = g->stream;
  // The reference iterates until the frontier empties (iter_num = INT_MAX); the
  // delta rule always empties it, far below this bound.
  const int32_t cap = o.max_iter > 0 ? o.max_iter : 100000;
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
  prr_init_kernel<<<g->num_sms * 8, 256, 0, s>>>(a, deg, cap);
  MG_CUDA_TRY(cudaGetLastError());
  const int grid = g->num_sms * 4;
  struct Sig {
    RefArgs a;
    int grid;
  } sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.a = a;
  sig.grid = grid;
  LoopBody body = [a, grid](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
    RefArgs b = a;
    b.h = h;
    b.use_cond = use_cond;
    prr_gather_kernel<<<grid, PRR_NT, 0, st>>>(b);
    prr_expand_kernel<<<grid, PRR_NT, 0, st>>>(b);
  };
  MG_TRY(run_loop(g, SLOT_PR_REF, &sig, sizeof(sig), o.use_graph >= 0, body, (int64_t)cap + 2));
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  if (!o.device_output) MG_TRY(copy_out(g, ranks, a.x, sizeof(float) * n, 0));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = hc.edges_inspected;
    stats->edges_inspected = hc.edges_inspected;
    stats->bytes_compulsory = 8 * hc.edges_inspected;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->launches = 1 + (o.use_graph >= 0 ? 3 * (int64_t)hc.body_iters : 2 * (int64_t)hc.level);
  }
  if (hc.status != 0) {
    mg_set_error("mg_pagerank: device status %d", hc.status);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// NORMALIZED, one vector.
// Gather autotuner (mg_pr_opts.autotune): times the forward solve's gather
// variants on this graph -- the column cache at several capacities and the binned
// kernel without a cache -- over four iterations each (second of two runs, so the
// executable graph is cached) and keeps the fastest for the graph's later solves.
// Results do not depend on the choice beyond rounding.
static mg_status pr_autotune(mg_graph *g, const float *tele_dev, const mg_pr_opts &o) {
  using namespace mg;
  const bool weighted = o.weighted != 0;
  const int32_t limit = hub_cache_limit(g);
  struct Cand {
    int variant;
    int32_t cap, T, S;
  };
  std::vector<Cand> cands;
  std::vector<int32_t> caps;
  for (int32_t c : {20480, 32768, PRB_HUB_CAP})
    if (c > 0 && c <= limit && std::find(caps.begin(), caps.end(), c) == caps.end()) caps.push_back(c);
  cands.push_back({0, 0, 0, 0});  // no cache
  cands.push_back({1, 0, 0, 0});  // merge-path tiles staged by TMA bulk copies
  for (int32_t c : caps) cands.push_back({2, c, 0, 0});
  // segmented: hub thresholds (blocks as wide as the column cache; wider blocks
  // measured slower on R-MAT s22, 389 vs 344 us per iteration at T = 512)
  const int32_t sdef = seg_block_default(g);
  if (g->n > 0 && (g->n + sdef - 1) / sdef <= SEG_MAXB)
    for (int32_t T : {512, 1024, 2048}) cands.push_back({3, hub_cache_capacity(g), T, sdef});
  float best = 0.f;
  size_t best_i = 0;
  for (size_t i = 0; i < cands.size(); i++) {
    const Cand &cd = cands[i];
    float ms = 0.f;
    bool skip = false;
    for (int rep = 0; rep < 2 && !skip; rep++) {
      SolvePlan sp;
      const mg_status st =
          solve_setup(g, false, weighted, tele_dev, nullptr, cd.variant, sp, cd.cap > 0 ? cd.cap : -1, cd.T, cd.S);
      if (st == MG_ERR_UNSUPPORTED) {  // a shape this graph cannot take
        skip = true;
        break;
      }
      MG_TRY(st);
      SolveArgs &a = sp.a;
      a.tn = g->n > 0 ? 1.0 / (double)g->n : 0.0;
      a.alpha = o.alpha > 0 ? o.alpha : 0.85;
      a.tol = 1e-300;  // run all four iterations
      a.max_iter = 4;
      a.adjoint = 0;
      MG_CUDA_TRY(cudaEventRecord(g->ev0, g->stream));
      MG_TRY(solve_run(g, sp, 0, SLOT_PR));
      MG_CUDA_TRY(cudaEventRecord(g->ev1, g->stream));
      MG_CUDA_TRY(cudaEventSynchronize(g->ev1));
      MG_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    }
    if (skip) continue;
    if (i == 0 || ms < best) {
      best = ms;
      best_i = i;
    }
  }
  PlanSet *ps = plans_of(g);
  const Cand &b = cands[best_i];
  ps->tuned_variant = b.variant;
  ps->tuned_cap = b.cap;
  ps->tuned_seg_T = b.variant == 3 ? b.T : 0;
  ps->tuned_seg_S = b.variant == 3 ? b.S : 0;
  // keep only the kept variant's segmented plan
  if (b.variant != 3) seg_plan_release(g, ps->seg);
  return MG_OK;
}

static mg_status pagerank_normalized(mg_graph *g, const float *tele_dev, float *ranks_out, int out_is_device,
                                     const mg_pr_opts &o, mg_stats *stats) {
  using namespace mg;
  const bool weighted = o.weighted != 0;
  if (!g->has_csc) {
    mg_set_error("mg_pagerank: the gather over in-edges needs the CSC");
    return MG_ERR_UNSUPPORTED;
  }
  if (weighted && g->vtype != MG_DTYPE_F32) {
    mg_set_error("mg_pagerank: weighted mode needs float edge values");
    return MG_ERR_ARG;
  }
  PlanSet *ps = plans_of(g);
  if (o.gather_kernel == 0 && o.autotune && ps->tuned_variant < 0) MG_TRY(pr_autotune(g, tele_dev, o));
  int variant = o.gather_kernel;
  int32_t cap = -1, segT = 0, segS = 0;
  if (variant == 0 && ps->tuned_variant > 0) {  // the autotuner's pick
    variant = ps->tuned_variant;
    cap = ps->tuned_cap > 0 ? ps->tuned_cap : -1;
    segT = ps->tuned_seg_T;
    segS = ps->tuned_seg_S;
  }
  if (variant == 3) {  // explicit segmented shape
    if (o.seg_hub_edges > 0) segT = o.seg_hub_edges;
    if (o.seg_block_cols > 0) segS = o.seg_block_cols;
  }
  SolvePlan sp;
  MG_TRY(solve_setup(g, false, weighted, tele_dev, nullptr, variant, sp, cap, segT, segS));
  SolveArgs &a = sp.a;
  a.tn = g->n > 0 ? 1.0 / (double)g->n : 0.0;
  a.alpha = o.alpha > 0 ? o.alpha : 0.85;
  a.tol = o.tol > 0 ? o.tol : 1e-6;
  a.max_iter = o.max_iter > 0 ? o.max_iter : 50;
  a.adjoint = 0;
  cudaStream_t s = g->stream;
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  MG_TRY(solve_run(g, sp, o.use_graph, SLOT_PR));
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  MG_TRY(fetch_ctl(g));
  const DevCtl &hc = *g->ctl_host;
  const float *res = hc.cur ? a.v1 : a.v0;
  if (sp.use_seg && g->n > 0) {  // x is in the solve's position order: back to row order
    float *rowx = hc.cur ? a.v0 : a.v1;  // the other iterate buffer is free now
    seg_unpermute_kernel<<<g->num_sms * 4, 256, 0, s>>>(res, sp.ppos, g->n, rowx);
    MG_CUDA_TRY(cudaGetLastError());
    res = rowx;
  }
  MG_CUDA_TRY(cudaMemcpyAsync(ranks_out, res, sizeof(float) * g->n,
                              out_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = g->m * hc.level;
    stats->edges_inspected = g->m * hc.level;
    stats->residual = hc.dsum[0];
    // per iteration: offsets 4(n+1), indices 4m (+4m weights), x read, x and x/s written
    stats->bytes_compulsory = hc.level * (4 * (g->n + 1) + (weighted ? 8 : 4) * g->m + 12 * g->n);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    // fill + row sums + init + init reduce, then per iteration the gather (merge-path:
    // gather + fix-up), plus the loop guard when the loop runs as a graph
    const int64_t per_it = (variant == 1 || sp.use_seg) ? 2 : 1;
    stats->status_detail = (sp.use_hub || sp.use_seg) ? sp.a.nhub : 0;
    stats->variant = variant;
    stats->launches = 4 + ((sp.use_hub || sp.use_seg) ? 1 : 0) +
                      (o.use_graph >= 0 ? (per_it + 1) * (int64_t)hc.body_iters : per_it * (int64_t)hc.level);
  }
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Batched personalised PageRank (nvec > 1): groups of up to 256 vectors solved
// together over the vertex-major layout of ppr.cuh.
template <int VPL, bool W>
static int ppr_occupancy() {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mg::ppr_iter_kernel<VPL, W>, mg::PPR_NT, 0);
  cudaGetLastError();
  return std::max(1, std::min(occ, 8));
}

template <int VPL, bool W>
static void ppr_launch_iter(const mg::PprArgs &a, cudaStream_t st) {
  mg::ppr_iter_kernel<VPL, W><<<a.grid, mg::PPR_NT, 0, st>>>(a);
}

template <int VPL>
static void ppr_launch_init(const mg::PprArgs &a, int grid, cudaStream_t st) {
  mg::ppr_init_kernel<VPL><<<grid, mg::PPR_NT, 0, st>>>(a);
}

static mg_status pagerank_ppr(mg_graph *g, const float *tele_dev, int32_t nvec, float *ranks_out, int out_is_device,
                              const mg_pr_opts &o, mg_stats *stats, int32_t gw);

// Group-width autotuner of the batched personalised PageRank (mg_pr_opts.autotune
// with nvec > 1): runs the first vectors at 64, 128 and 256 vectors per pass for
// four iterations each (second of two runs, so the executable graph is cached)
// and keeps the width with the most vector-iterations per second for the graph.
static mg_status ppr_autotune(mg_graph *g, const float *tele_dev, int32_t nvec, float *ranks, const mg_pr_opts &o) {
  using namespace mg;
  mg_pr_opts t = o;
  t.max_iter = 4;
  t.tol = 1e-300;  // run all four iterations
  double best = -1.0;
  int32_t best_w = PPR_MAXW;
  const int32_t cap = std::min<int32_t>(((nvec + 31) / 32) * 32, PPR_MAXW);
  for (int32_t w : {64, 128, 256}) {
    if (w > cap) continue;
    const int32_t nv = std::min(nvec, w);
    mg_stats st;
    for (int rep = 0; rep < 2; rep++) MG_TRY(pagerank_ppr(g, tele_dev, nv, ranks, o.device_output, t, &st, w));
    const double rate = st.kernel_ms > 0 ? (double)nv * (double)st.iterations / st.kernel_ms : 0.0;
    if (rate > best) {
      best = rate;
      best_w = w;
    }
  }
  plans_of(g)->tuned_ppr_w = best_w;
  return MG_OK;
}

static mg_status pagerank_ppr(mg_graph *g, const float *tele_dev, int32_t nvec, float *ranks_out, int out_is_device,
                              const mg_pr_opts &o, mg_stats *stats, int32_t gw) {
  using namespace mg;
  const bool weighted = o.weighted != 0;
  if (!g->has_csc) {
    mg_set_error("mg_pagerank: the gather over in-edges needs the CSC");
    return MG_ERR_UNSUPPORTED;
  }
  if (weighted && g->vtype != MG_DTYPE_F32) {
    mg_set_error("mg_pagerank: weighted mode needs float edge values");
    return MG_ERR_ARG;
  }
  BinPlan *bins = nullptr, *rbins = nullptr;
  MG_TRY(get_bin_plan(g, false, &bins));
  if (weighted) MG_TRY(get_bin_plan(g, true, &rbins));
  const int64_t n = g->n;
  const int32_t kmax = std::min<int32_t>(nvec, gw);
  const int vpl = kmax > 128 ? 8 : kmax > 64 ? 4 : kmax > 32 ? 2 : 1;
  const int32_t W = 32 * vpl;
  int occ = 1;
  switch (vpl * 2 + (weighted ? 1 : 0)) {
    case 2: occ = ppr_occupancy<1, false>(); break;
    case 3: occ = ppr_occupancy<1, true>(); break;
    case 4: occ = ppr_occupancy<2, false>(); break;
    case 5: occ = ppr_occupancy<2, true>(); break;
    case 8: occ = ppr_occupancy<4, false>(); break;
    case 9: occ = ppr_occupancy<4, true>(); break;
    case 16: occ = ppr_occupancy<8, false>(); break;
    default: occ = ppr_occupancy<8, true>(); break;
  }
  const int grid = g->num_sms * occ;
  const int ginit = g->num_sms * 8;
  const int gpart = std::max(grid, ginit);
  const size_t nw = (size_t)n * W;
  const int64_t nchunks = bins->ntasks, nheavy = bins->nheavy;
  const size_t need = Carve::need({sizeof(float) * nw, sizeof(float) * nw, sizeof(float) * nw, sizeof(float) * nw,
                                   sizeof(float) * nw, sizeof(float) * ((size_t)n + 8), sizeof(double) * W,
                                   sizeof(double) * 2 * W * (size_t)gpart,
                                   sizeof(Comp) * W * (size_t)std::max<int64_t>(nchunks, 1),
                                   sizeof(int32_t) * (size_t)(std::max<int64_t>(nheavy, 1) + 1),
                                   sizeof(double) * 2 * W * (size_t)std::max<int64_t>(nheavy, 1),
                                   out_is_device ? 0 : sizeof(float) * (size_t)kmax * n});
  MG_TRY(ws_reserve(g, g->ws_main, need));
  Carve cv(g->ws_main.ptr);
  PprArgs a;
  std::memset(&a, 0, sizeof(a));
  float *tele = cv.take<float>(nw);
  a.x0 = cv.take<float>(nw);
  a.x1 = cv.take<float>(nw);
  a.g0 = cv.take<float>(nw);
  a.g1 = cv.take<float>(nw);
  float *srow = cv.take<float>((size_t)n + 8);
  a.dang = cv.take<double>(W);
  a.part = cv.take<double>(2 * (size_t)W * gpart);
  a.hpart = cv.take<Comp>((size_t)W * std::max<int64_t>(nchunks, 1));
  a.hcount = cv.take<int32_t>(std::max<int64_t>(nheavy, 1) + 1);
  a.grab = a.hcount + std::max<int64_t>(nheavy, 1);
  a.hres = cv.take<double>(2 * (size_t)W * std::max<int64_t>(nheavy, 1));
  float *stage = out_is_device ? nullptr : cv.take<float>((size_t)kmax * n);
  a.off = g->co;
  a.idx = g->ri;
  a.wts = weighted ? (const float *)g->cvals : nullptr;
  a.rows = bins->rows;
  a.nlight = bins->boff[6];
  a.hrows = bins->hrows;
  a.hbase = bins->hbase;
  a.nheavy = nheavy;
  a.nchunks = nchunks;
  a.srow = srow;
  a.tele = tele;
  a.n = n;
  a.W = W;
  a.alpha = o.alpha > 0 ? o.alpha : 0.85;
  a.tol = o.tol > 0 ? o.tol : 1e-6;
  a.max_iter = o.max_iter > 0 ? o.max_iter : 50;
  a.grid = grid;
  a.ctl = g->ctl;
  cudaStream_t s = g->stream;
  MG_CUDA_TRY(cudaMemsetAsync(a.hcount, 0, sizeof(int32_t) * (std::max<int64_t>(nheavy, 1) + 1), s));
  if (!weighted) {
    outdeg_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ro, n, srow);
  } else {
    const PrbArgs rp = prb_args_of(g, *rbins, true, (const float *)g->vals);
    rowsum_binned_kernel<<<g->num_sms * 8, PRB_NT, 0, s>>>(rp, srow);
  }
  MG_CUDA_TRY(cudaGetLastError());
  mg_stats total;
  std::memset(&total, 0, sizeof(total));
  const dim3 tblk(32, 8), tgrid((unsigned)((n + 31) / 32), (unsigned)(W / 32));
  for (int32_t c0 = 0; c0 < nvec; c0 += kmax) {
    const int32_t k = std::min<int32_t>(kmax, nvec - c0);
    MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
    ppr_pack_kernel<<<tgrid, tblk, 0, s>>>(tele_dev ? tele_dev + (size_t)c0 * n : nullptr, k, n, W, tele);
    MG_CUDA_TRY(cudaMemsetAsync(g->ctl, 0, sizeof(DevCtl), s));
    switch (vpl) {
      case 1: ppr_launch_init<1>(a, ginit, s); break;
      case 2: ppr_launch_init<2>(a, ginit, s); break;
      case 4: ppr_launch_init<4>(a, ginit, s); break;
      default: ppr_launch_init<8>(a, ginit, s); break;
    }
    ppr_init_reduce_kernel<<<1, 256, 0, s>>>(a, ginit);
    MG_CUDA_TRY(cudaGetLastError());
    struct Sig {
      PprArgs a;
      int vpl, w;
    } sig;
    std::memset(&sig, 0, sizeof(sig));
    sig.a = a;
    sig.vpl = vpl;
    sig.w = weighted;
    LoopBody body = [a, vpl, weighted](cudaStream_t st, cudaGraphConditionalHandle h, int use_cond) {
      PprArgs b = a;
      b.h = h;
      b.use_cond = use_cond;
      switch (vpl * 2 + (weighted ? 1 : 0)) {
        case 2: ppr_launch_iter<1, false>(b, st); break;
        case 3: ppr_launch_iter<1, true>(b, st); break;
        case 4: ppr_launch_iter<2, false>(b, st); break;
        case 5: ppr_launch_iter<2, true>(b, st); break;
        case 8: ppr_launch_iter<4, false>(b, st); break;
        case 9: ppr_launch_iter<4, true>(b, st); break;
        case 16: ppr_launch_iter<8, false>(b, st); break;
        default: ppr_launch_iter<8, true>(b, st); break;
      }
    };
    MG_TRY(run_loop(g, SLOT_PPR, &sig, sizeof(sig), o.use_graph >= 0, body, (int64_t)a.max_iter + 2));
    MG_TRY(fetch_ctl(g));
    const DevCtl &hc = *g->ctl_host;
    const float *res = hc.cur ? a.x1 : a.x0;
    float *dst = out_is_device ? ranks_out + (size_t)c0 * n : stage;
    ppr_unpack_kernel<<<tgrid, tblk, 0, s>>>(res, k, n, W, dst);
    MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
    MG_CUDA_TRY(cudaGetLastError());
    if (!out_is_device)
      MG_CUDA_TRY(cudaMemcpyAsync(ranks_out + (size_t)c0 * n, stage, sizeof(float) * (size_t)k * n,
                                  cudaMemcpyDeviceToHost, s));
    MG_CUDA_TRY(cudaStreamSynchronize(s));
    if (hc.status != 0) {
      mg_set_error("mg_pagerank: device status %d", hc.status);
      return (mg_status)hc.status;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    total.kernel_ms += ms;
    total.iterations = std::max<int64_t>(total.iterations, hc.level);
    total.edges_traversed += g->m * hc.level * k;
    total.edges_inspected += g->m * hc.level;
    total.residual = std::max(total.residual, hc.dsum[0]);
    // per iteration: offsets, indices (+ weights), W-wide rows gathered per edge,
    // and x read, x, g written and t read per vertex
    total.bytes_compulsory += hc.level * (4 * (n + 1) + (weighted ? 8 : 4) * g->m + (int64_t)4 * W * g->m +
                                          (int64_t)16 * W * n);
    total.launches += 5 + (o.use_graph >= 0 ? 2 * (int64_t)hc.body_iters : (int64_t)hc.level);
  }
  if (stats) *stats = total;
  return MG_OK;
}

extern "C" mg_status mg_pagerank(mg_graph *g, const float *teleport, int32_t nvec, float *ranks,
                                 const mg_pr_opts *opts, mg_stats *stats) {
  if (!g || !ranks || nvec <= 0) {
    mg_set_error("mg_pagerank: null argument or nvec <= 0");
    return MG_ERR_ARG;
  }
  mg_pr_opts o;
  std::memset(&o, 0, sizeof(o));
  o.directed = 1;
  if (opts) o = *opts;
  if (o.mode != MG_PR_REFCOMPAT && o.mode != MG_PR_NORMALIZED) {
    mg_set_error("mg_pagerank: unknown mode %d", o.mode);
    return MG_ERR_ARG;
  }
  if (o.alpha < 0 || o.alpha >= 1) {
    mg_set_error("mg_pagerank: alpha must be in [0, 1)");
    return MG_ERR_ARG;
  }
  if (o.gather_kernel < 0 || o.gather_kernel > 3) {
    mg_set_error("mg_pagerank: gather_kernel must be 0..3");
    return MG_ERR_ARG;
  }
  if (o.seg_hub_edges < 0 || o.seg_block_cols < 0 || o.seg_block_cols % 32 != 0) {
    mg_set_error("mg_pagerank: seg_hub_edges must be >= 0 and seg_block_cols a multiple of 32");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  if (o.device_output) {
    MG_TRY(check_device_ptr(g, ranks, "mg_pagerank", "ranks"));
    MG_TRY(check_device_ptr(g, teleport, "mg_pagerank", "teleport"));
  }
  if (o.mode == MG_PR_REFCOMPAT) {
    if (nvec != 1 || teleport) {
      mg_set_error("mg_pagerank: REFCOMPAT takes no teleport vector and nvec == 1");
      return MG_ERR_ARG;
    }
    return pagerank_refcompat(g, ranks, o, stats);
  }
  const int64_t n = g->n;
  // Teleport vectors and outputs are staged through device memory.
  float *tele_dev = nullptr;
  if (teleport) {
    if (o.device_output) tele_dev = const_cast<float *>(teleport);
    else {
      MG_TRY(ws_reserve(g, g->ws_out, sizeof(float) * (size_t)n * nvec + 256));
      tele_dev = (float *)g->ws_out.ptr;
      MG_CUDA_TRY(cudaMemcpyAsync(tele_dev, teleport, sizeof(float) * n * nvec, cudaMemcpyHostToDevice, g->stream));
    }
  }
  if (nvec > 1) {
    int32_t gw = o.group_width > 0 ? o.group_width : mg::PPR_MAXW;
    if (gw % 32 != 0 || gw > mg::PPR_MAXW) {
      mg_set_error("mg_pagerank: group_width must be a multiple of 32 up to %d", mg::PPR_MAXW);
      return MG_ERR_ARG;
    }
    if (o.group_width <= 0 && o.autotune) {
      mg::PlanSet *ps = plans_of(g);
      if (ps->tuned_ppr_w < 0) MG_TRY(ppr_autotune(g, tele_dev, nvec, ranks, o));
      gw = ps->tuned_ppr_w;
    }
    MG_TRY(pagerank_ppr(g, tele_dev, nvec, ranks, o.device_output, o, stats, gw));
    if (stats) stats->status_detail = gw;
    return MG_OK;
  }
  mg_stats total;
  std::memset(&total, 0, sizeof(total));
  for (int32_t k = 0; k < nvec; k++) {
    mg_stats st;
    MG_TRY(pagerank_normalized(g, tele_dev ? tele_dev + (size_t)k * n : nullptr, ranks + (size_t)k * n,
                               o.device_output, o, &st));
    total.iterations += st.iterations;
    total.edges_traversed += st.edges_traversed;
    total.edges_inspected += st.edges_inspected;
    total.bytes_compulsory += st.bytes_compulsory;
    total.kernel_ms += st.kernel_ms;
    total.launches += st.launches;
    total.residual = std::max(total.residual, st.residual);
    total.status_detail = st.status_detail;  // cached columns of the gather (same for every vector)
    total.variant = st.variant;
  }
  if (stats) *stats = total;
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Adjoint (mg_pagerank_backward).
namespace mg {

// Per-row products of the converged adjoint: pl[u] = sum_k a_uk lambda_k / s_u and
// coef[u] = alpha * x_u / s_u (both 0 for dangling rows), in FP64.
struct AdjRowStore {
  const float *srow, *x;
  double *pl, *coef;
  double alpha;
  __device__ __forceinline__ void operator()(int32_t r, Comp v) {
    const double s = (double)srow[r];
    if (s > 0.0) {
      pl[r] = ((double)v.hi + (double)v.lo) / s;
      coef[r] = alpha * (double)x[r] / s;
    } else {
      pl[r] = 0.0;
      coef[r] = 0.0;
    }
  }
};

template <bool WEIGHTED>
__global__ void __launch_bounds__(PRB_NT) adj_rows_kernel(PrbArgs p, const float *lam, AdjRowStore st) {
  prb_run<WEIGHTED>(p, [&](int32_t c) { return __ldg(lam + c); }, st,
                    [&](int64_t, int32_t row, Comp v) { st(row, v); });
}

// dL/da_uv = coef[u] * (lambda_v - pl[u]) for every CSR edge, rows expanded with
// the degree-binned tile expansion (coalesced index loads and gradient stores).
__global__ void __launch_bounds__(256) adj_edge_grad_kernel(const int32_t *__restrict__ ro,
                                                            const int32_t *__restrict__ ci, int64_t n,
                                                            const float *__restrict__ lam,
                                                            const double *__restrict__ pl,
                                                            const double *__restrict__ coef, float *__restrict__ grad) {
  __shared__ ExpandSmem<256> sm;
  int64_t insp = 0;
  for (int64_t tile = (int64_t)blockIdx.x * 256; tile < n; tile += (int64_t)gridDim.x * 256) {
    const int64_t i = tile + threadIdx.x;
    const int32_t v = i < n ? (int32_t)i : -1;
    expand_tile<256, 1024>(sm, ro, v, insp, [&](int32_t u, int32_t k) {
      grad[k] = (float)(coef[u] * ((double)__ldg(lam + ci[k]) - pl[u]));
    });
  }
}

// Dangling rank mass of x: per-block partials, then one block.
__global__ void __launch_bounds__(256) adj_dangling_kernel(const float *x, const float *srow, int64_t n,
                                                           double *part) {
  __shared__ double s_red[256 / 32 + 1];
  double d = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (srow[i] == 0.f) d += (double)x[i];
  d = block_sum<256>(d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = d;
}

// dL/dt_i = lambda_i * (1 - alpha + alpha * d).
__global__ void __launch_bounds__(256) adj_tele_grad_kernel(const float *lam, const double *part, int nparts,
                                                            int64_t n, double alpha, float *gt) {
  __shared__ double s_d;
  if (threadIdx.x == 0) {
    double d = 0.0;
    for (int i = 0; i < nparts; i++) d += part[i];
    s_d = d;
  }
  __syncthreads();
  const double f = 1.0 - alpha + alpha * s_d;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    gt[i] = (float)((double)lam[i] * f);
}

}  // namespace mg

extern "C" mg_status mg_pagerank_backward(mg_graph *g, const float *teleport, const float *ranks,
                                          const float *dL_dranks, float *dL_dweights, float *dL_dteleport,
                                          const mg_pr_opts *opts, mg_stats *stats) {
  using namespace mg;
  if (!g || !ranks || !dL_dranks) {
    mg_set_error("mg_pagerank_backward: null argument");
    return MG_ERR_ARG;
  }
  mg_pr_opts o;
  std::memset(&o, 0, sizeof(o));
  o.mode = MG_PR_NORMALIZED;
  if (opts) o = *opts;
  if (o.mode != MG_PR_NORMALIZED) {
    mg_set_error("mg_pagerank_backward: only the NORMALIZED fixed point has an adjoint");
    return MG_ERR_ARG;
  }
  if (o.alpha < 0 || o.alpha >= 1) {
    mg_set_error("mg_pagerank_backward: alpha must be in [0, 1)");
    return MG_ERR_ARG;
  }
  const bool weighted = o.weighted != 0;
  if (weighted && g->vtype != MG_DTYPE_F32) {
    mg_set_error("mg_pagerank_backward: weighted mode needs float edge values");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  if (o.device_output) {
    const char *fn = "mg_pagerank_backward";
    MG_TRY(check_device_ptr(g, ranks, fn, "ranks"));
    MG_TRY(check_device_ptr(g, dL_dranks, fn, "dL_dranks"));
    MG_TRY(check_device_ptr(g, teleport, fn, "teleport"));
    MG_TRY(check_device_ptr(g, dL_dweights, fn, "dL_dweights"));
    MG_TRY(check_device_ptr(g, dL_dteleport, fn, "dL_dteleport"));
  }
  const int64_t n = g->n, m = g->m;
  cudaStream_t s = g->stream;
  // Inputs staged on the device.
  const float *x_dev = ranks, *w_dev = dL_dranks, *t_dev = teleport;
  if (!o.device_output) {
    MG_TRY(ws_reserve(g, g->ws_out, Carve::need({4 * (size_t)n, 4 * (size_t)n, 4 * (size_t)n})));
    Carve cv(g->ws_out.ptr);
    float *xs = cv.take<float>(n), *ws = cv.take<float>(n), *ts = cv.take<float>(n);
    MG_CUDA_TRY(cudaMemcpyAsync(xs, ranks, 4 * n, cudaMemcpyHostToDevice, s));
    MG_CUDA_TRY(cudaMemcpyAsync(ws, dL_dranks, 4 * n, cudaMemcpyHostToDevice, s));
    if (teleport) MG_CUDA_TRY(cudaMemcpyAsync(ts, teleport, 4 * n, cudaMemcpyHostToDevice, s));
    x_dev = xs;
    w_dev = ws;
    t_dev = teleport ? ts : nullptr;
  }
  MG_CUDA_TRY(cudaEventRecord(g->ev0, s));
  SolvePlan sp;
  MG_TRY(solve_setup(g, true, weighted, t_dev, w_dev, o.gather_kernel == 1 ? 1 : 0, sp));  // no cache in the adjoint
  SolveArgs &a = sp.a;
  a.tn = n > 0 ? 1.0 / (double)n : 0.0;
  a.alpha = o.alpha > 0 ? o.alpha : 0.85;
  a.tol = o.tol > 0 ? o.tol : 1e-7;
  a.max_iter = o.max_iter > 0 ? o.max_iter : 200;
  a.adjoint = 1;
  MG_TRY(solve_run(g, sp, o.use_graph, SLOT_ADJ));
  MG_TRY(fetch_ctl(g));
  const DevCtl hc = *g->ctl_host;
  const float *lam = hc.cur ? a.v1 : a.v0;
  // Per-row products and gradients (scratch in ws_aux).
  const int nparts = g->num_sms * 4;
  MG_TRY(ws_reserve(g, g->ws_aux, Carve::need({8 * (size_t)n, 8 * (size_t)n, 8 * (size_t)nparts, 4 * (size_t)m,
                                            4 * (size_t)n})));
  Carve cv(g->ws_aux.ptr);
  double *pl = cv.take<double>(n), *coef = cv.take<double>(n), *part = cv.take<double>(nparts);
  float *gw_ws = cv.take<float>(m), *gt_ws = cv.take<float>(n);
  float *gw = o.device_output ? dL_dweights : gw_ws;
  float *gt = o.device_output ? dL_dteleport : gt_ws;
  int64_t launches = 0;
  if (dL_dweights) {
    BinPlan *rb = nullptr;
    MG_TRY(get_bin_plan(g, true, &rb));
    const PrbArgs rp = prb_args_of(g, *rb, true, weighted ? (const float *)g->vals : nullptr);
    AdjRowStore st{a.srow, x_dev, pl, coef, a.alpha};
    if (weighted) adj_rows_kernel<true><<<g->num_sms * 8, PRB_NT, 0, s>>>(rp, lam, st);
    else adj_rows_kernel<false><<<g->num_sms * 8, PRB_NT, 0, s>>>(rp, lam, st);
    adj_edge_grad_kernel<<<g->num_sms * 8, 256, 0, s>>>(g->ro, g->ci, n, lam, pl, coef, gw);
    launches += 2;
  }
  if (dL_dteleport) {
    adj_dangling_kernel<<<nparts, 256, 0, s>>>(x_dev, a.srow, n, part);
    adj_tele_grad_kernel<<<g->num_sms * 8, 256, 0, s>>>(lam, part, nparts, n, a.alpha, gt);
    launches += 2;
  }
  MG_CUDA_TRY(cudaGetLastError());
  MG_CUDA_TRY(cudaEventRecord(g->ev1, s));
  if (!o.device_output) {
    if (dL_dweights) MG_CUDA_TRY(cudaMemcpyAsync(dL_dweights, gw, 4 * m, cudaMemcpyDeviceToHost, s));
    if (dL_dteleport) MG_CUDA_TRY(cudaMemcpyAsync(dL_dteleport, gt, 4 * n, cudaMemcpyDeviceToHost, s));
  }
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = hc.level;
    stats->edges_traversed = m * (hc.level + (dL_dweights ? 2 : 0));
    stats->edges_inspected = stats->edges_traversed;
    stats->residual = hc.dsum[0];
    // per solve iteration as the forward; the gradient pass reads col + weight,
    // writes the gradient, and reads/writes per-row state
    stats->bytes_compulsory = hc.level * (4 * (n + 1) + (weighted ? 8 : 4) * m + 12 * n) +
                              (dL_dweights ? 12 * m + 24 * n : 0);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    stats->kernel_ms = ms;
    stats->launches = 4 + launches + (o.use_graph >= 0 ? 2 * (int64_t)hc.body_iters : (int64_t)hc.level);
  }
  if (hc.status != 0) {
    mg_set_error("mg_pagerank_backward: device status %d", hc.status);
    return (mg_status)hc.status;
  }
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Test hook: host-side check of a segmented gather plan (mg_debug_seg_plan).
extern "C" mg_status mg_debug_seg_plan(mg_graph *g, int32_t hub_edges, int32_t block_cols, int64_t *out) {
  using namespace mg;
  if (!g || !out || hub_edges <= 0 || block_cols <= 0 || block_cols % 32 != 0) {
    mg_set_error("mg_debug_seg_plan: bad argument");
    return MG_ERR_ARG;
  }
  MG_TRY(graph_enter(g));
  HubCache *hubs = nullptr;
  MG_TRY(get_hub_cache(g, hub_cache_capacity(g), &hubs));
  SegPlan *sp = nullptr;
  const bool weighted = plans_of(g)->seg.ok ? plans_of(g)->seg.weighted : false;
  MG_TRY(get_seg_plan(g, hub_edges, block_cols, weighted, *hubs, &sp));
  cudaStream_t s = g->stream;
  const int64_t nh = sp->bins.nheavy, ng = sp->ngroups, m = g->m;
  auto d2h = [&](void *dst, const void *src, size_t bytes) -> mg_status {
    if (bytes) MG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    return MG_OK;
  };
  std::vector<int32_t> hrows(nh), hbase(nh + 1), hcount(nh), co(g->n + 1), ri(m), bgrp(sp->nblocks + 1),
      cta(sp->grid + 1);
  std::vector<uint16_t> pidx(sp->nell);
  std::vector<int2> ent((size_t)ng * 32);
  std::vector<int64_t> gofs(ng + 1);
  MG_TRY(d2h(hrows.data(), sp->bins.hrows, 4 * nh));
  MG_TRY(d2h(hbase.data(), sp->bins.hbase, 4 * (nh + 1)));
  MG_TRY(d2h(hcount.data(), sp->bins.hcount, 4 * nh));
  MG_TRY(d2h(co.data(), g->co, 4 * (g->n + 1)));
  MG_TRY(d2h(ri.data(), g->ri, 4 * m));
  MG_TRY(d2h(bgrp.data(), sp->bgrp, 4 * bgrp.size()));
  MG_TRY(d2h(cta.data(), sp->cta, 4 * cta.size()));
  MG_TRY(d2h(pidx.data(), sp->pidx, 2 * pidx.size()));
  MG_TRY(d2h(ent.data(), sp->ent, sizeof(int2) * ent.size()));
  MG_TRY(d2h(gofs.data(), sp->gofs, 8 * gofs.size()));
  MG_CUDA_TRY(cudaStreamSynchronize(s));
  const int64_t nfrag = nh ? hbase[nh] : 0;
  std::vector<int32_t> seen(nfrag, 0);
  // per fragment: its block and the multiset of its (permuted) columns
  std::vector<std::vector<int32_t>> fcols(nfrag);
  std::vector<int32_t> fblock(nfrag, -1), fhub(nfrag, -1);
  for (int64_t b = 0; b < sp->nblocks; b++)
    for (int64_t gi = bgrp[b]; gi < bgrp[b + 1]; gi++)
      for (int l = 0; l < 32; l++) {
        const int2 e = ent[gi * 32 + l];
        if (e.x < 0) continue;
        if (e.x >= nfrag) continue;
        seen[e.x]++;
        fblock[e.x] = (int32_t)b;
        fhub[e.x] = e.y;
        const int64_t depth = (gofs[gi + 1] - gofs[gi]) / 32;
        for (int64_t i = 0; i < depth; i++) {
          const uint16_t off = pidx[seg_pk(gofs[gi], l, i)];
          if (off != 0xffffu) fcols[e.x].push_back((int32_t)(b * sp->S + off));
        }
      }
  int64_t once = 0, match = 0;
  for (int64_t f = 0; f < nfrag; f++) once += seen[f] == 1;
  // expected: per hub, its edges of each block (permuted), split at SEG_FMAX, in block order
  for (int64_t h = 0; h < nh; h++) {
    const int32_t r = hrows[h];
    std::vector<std::vector<int32_t>> byb(sp->nblocks);
    for (int32_t k = co[r]; k < co[r + 1]; k++) byb[ri[k] / sp->S].push_back(seg_swz(ri[k]));
    int64_t f = hbase[h];
    for (int64_t b = 0; b < sp->nblocks; b++) {
      for (size_t q = 0; q < byb[b].size(); q += SEG_FMAX, f++) {
        if (f >= hbase[h + 1]) break;
        std::vector<int32_t> want(byb[b].begin() + q, byb[b].begin() + std::min(byb[b].size(), q + SEG_FMAX));
        std::vector<int32_t> got = fcols[f];
        std::sort(want.begin(), want.end());
        std::sort(got.begin(), got.end());
        match += (got == want && fblock[f] == b && fhub[f] == h) ? 1 : 0;
      }
    }
  }
  int64_t nonzero = 0;
  for (int32_t c : hcount) nonzero += c != 0;
  bool cover = cta[0] == 0 && cta[sp->grid] == ng;
  for (int i = 0; i < sp->grid; i++) cover = cover && cta[i] <= cta[i + 1];
  out[0] = nh;
  out[1] = nfrag;
  out[2] = ng;
  out[3] = sp->nell;
  out[4] = once;
  out[5] = match;
  out[6] = nonzero;
  out[7] = cover ? 1 : 0;
  return MG_OK;
}
