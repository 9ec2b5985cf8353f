/*
 * mapgraph_b200.h -- C ABI of the B200 (sm_100a) Gather-Apply-Scatter engine.
 *
 * This is the drop-in boundary for MapGraph's GAS hot path. The reference exposes
 * it as C++ templates (CsrProblem, EnactorVertexCentric and the four bundled
 * vertex programs); here the same operations are plain extern "C" functions with
 * pointers and sizes, no CUDA or C++ types in the signatures. Each entry cites the
 * reference interface it replaces (paths inside the MapGraph tree).
 *
 * Conventions
 *   - Vertex ids and offsets are int32 (the reference's VertexId/SizeT = int).
 *   - Every call returns an mg_status; nothing throws or exits. mg_last_error()
 *     gives a human-readable detail for the calling thread's last failure.
 *   - A graph lives on the CUDA device that was current when it was created and
 *     owns one CUDA stream; calls on one graph are serialised by the caller
 *     (a graph is not thread-safe, distinct graphs are). Calls are synchronous:
 *     results are complete when the call returns, like EnactIterativeSearch.
 *   - Output pointers are host pointers unless opts->device_output is set, in
 *     which case they are device pointers on the graph's device.
 *   - The engine never falls back to CPU code: without a usable GPU every compute
 *     call returns MG_ERR_NO_DEVICE.
 */
#ifndef MAPGRAPH_B200_H
#define MAPGRAPH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mg_status {
  MG_OK = 0,
  MG_ERR_ARG = 1,            /* bad argument: null pointer, size, out-of-range source */
  MG_ERR_OOM = 2,            /* device or host allocation failed */
  MG_ERR_QUEUE_OVERFLOW = 3, /* a frontier exceeded the capacity set by queue_sizing */
  MG_ERR_TIMEOUT = 4,        /* a bounded device-side wait ran out */
  MG_ERR_CUDA = 5,           /* CUDA runtime error; see mg_last_error() */
  MG_ERR_NO_DEVICE = 6,      /* no CUDA device / driver available */
  MG_ERR_UNSUPPORTED = 7     /* option combination not supported */
} mg_status;

typedef enum mg_dtype {
  MG_DTYPE_NONE = 0, /* no edge values (unit weights) */
  MG_DTYPE_I32 = 1,  /* int32 edge values (BFS/SSSP/CC programs: Value = int) */
  MG_DTYPE_F32 = 2   /* float edge values (PageRank program: Value = float) */
} mg_dtype;

/* mg_graph_create flags */
#define MG_GRAPH_SYMMETRIC 0x1u    /* caller asserts the CSR equals its transpose; the CSC aliases it */
#define MG_GRAPH_NO_CSC 0x2u       /* skip the transpose (then directed == 0, pull BFS and PageRank are refused) */
#define MG_GRAPH_DEVICE_INPUT 0x4u /* input arrays are device pointers on the current device */
#define MG_GRAPH_ASYNC_UPLOAD 0x8u /* with MG_GRAPH_SYMMETRIC or MG_GRAPH_NO_CSC: mg_graph_create returns once
                                      the upload and the validation are enqueued on the graph's stream, so the
                                      copy overlaps work on other graphs; the input arrays must stay valid and
                                      unchanged until mg_graph_sync or the first call on the graph returns,
                                      and an invalid CSR is reported there (MG_ERR_ARG). Other graphs upload
                                      synchronously whatever the flag. */

/* BFS direction policy (mg_opts.direction) */
#define MG_DIR_AUTO 0 /* push/pull switch chosen on the device each level (Beamer's rule); graphs of mean
                         out-degree <= 8 run top-down only */
#define MG_DIR_PUSH 1 /* top-down only (the reference engine's only mode) */
#define MG_DIR_PULL 2 /* bottom-up wherever possible (after the first level) */

/* PageRank modes (mg_pr_opts.mode) */
#define MG_PR_REFCOMPAT 0  /* x = 0.15 + 0.85 * sum x_u/deg_u, delta frontier (reference semantics) */
#define MG_PR_NORMALIZED 1 /* x = alpha (P^T x + d t) + (1 - alpha) t, L1-residual stop */

typedef struct mg_graph mg_graph;

/* Options shared by the traversal programs. Zero-initialised means defaults. */
typedef struct mg_opts {
  int32_t directed;      /* 1: follow out-edges; 0: out- and in-edges (reference "directed", default 1) */
  int32_t iter_num;      /* iteration cap (reference "iter_num"); <= 0 means unbounded */
  int32_t direction;     /* BFS only: MG_DIR_AUTO / MG_DIR_PUSH / MG_DIR_PULL */
  int32_t device_output; /* 1: output arrays are device pointers */
  double queue_sizing;   /* frontier capacity = queue_sizing * n (reference "max_queue_sizing");
                            <= 0 means n, which cannot overflow */
  int32_t threshold;     /* reference "threshold": accepted for compatibility; strategy is chosen on the device */
  int32_t use_graph;     /* 1 (default when 0): run the iteration loop as a CUDA graph with a device-side while node;
                            -1: host-driven loop (one frontier-size read per iteration) */
  int32_t delta;         /* SSSP only (int32 weights, iter_num unbounded): > 0 runs the near-far schedule with
                            this bucket width; 0 (default) chooses near-far with 8 x the mean weight on sparse
                            graphs (mean out-degree <= 8) and plain frontier Bellman-Ford otherwise; < 0 always
                            plain Bellman-Ford, whose rounds are the reference's (an iteration cap keeps it) */
  int32_t reserved[3];
} mg_opts;

/* Counters returned by every compute call (may be NULL). */
typedef struct mg_stats {
  int64_t iterations;       /* GAS iterations (BFS levels, relaxation rounds, PR sweeps) */
  int64_t edges_traversed;  /* TEPS numerator: BFS/SSSP sum of outdeg over reached vertices; CC m; PR m * iterations */
  int64_t edges_inspected;  /* edges actually read by the kernels */
  int64_t bytes_compulsory; /* algorithmic DRAM bytes (see the engine's documentation) */
  double kernel_ms;         /* device time of the iteration loop (CUDA events) */
  double residual;          /* PageRank: last L1 residual (normalised mode) */
  int64_t launches;         /* kernels launched by the call */
  int32_t status_detail;    /* BFS: levels run bottom-up; otherwise detail of a non-OK status */
  int32_t variant;          /* NORMALIZED PageRank (nvec == 1): the gather_kernel that ran (after
                               autotuning); 0 for the other programs */
} mg_stats;

/* PageRank options. Zero-initialised fields take the defaults in brackets. */
typedef struct mg_pr_opts {
  int32_t mode;          /* MG_PR_REFCOMPAT [default] or MG_PR_NORMALIZED */
  int32_t directed;      /* REFCOMPAT: 1 in-edges only, 0 both directions with deg = out+in [1] */
  int32_t max_iter;      /* iteration cap [REFCOMPAT: unbounded; NORMALIZED: 50] */
  int32_t weighted;      /* NORMALIZED: 1 uses F32 edge values a_uv, P_uv = a_uv / sum_k a_uk [0] */
  double alpha;          /* NORMALIZED damping [0.85] */
  double tol;            /* NORMALIZED: stop when the L1 change < tol [1e-6]; REFCOMPAT: active
                            while |dx| >= tol [0.01] */
  int32_t compensated;   /* 1: two-sum compensated FP32 accumulation [1]; -1 plain FP32 sums */
  int32_t device_output; /* 1: ranks/teleport/gradient arrays are device pointers */
  int32_t use_graph;     /* as mg_opts.use_graph */
  int32_t gather_kernel; /* NORMALIZED/adjoint gather: 0 degree-binned warps [default]; 1 merge-path tiles
                            staged in shared memory by TMA bulk copies; 2 degree-binned with the most-gathered
                            columns cached in shared memory; 3 segmented: rows of >= 512 edges gathered one
                            column block at a time from shared-memory copies of the block (TMA bulk copies),
                            the other rows one lane per row with the column cache of 2 (2 and 3 are forward
                            solves; the adjoint uses 0) */
  int32_t autotune;      /* NORMALIZED forward with gather_kernel 0: 1 makes the first such solve on a graph
                            time the gathers (degree-binned without and with column caches of 20K, 32K and
                            40K columns, merge-path, segmented with hub thresholds 512 / 1024 / 2048 edges;
                            4 iterations each) and keep the fastest for every later
                            solve;
                            stats->status_detail reports the column-cache size used (0 for none);
                            with nvec > 1 and group_width 0 it picks the group width instead (64, 128
                            or 256 vectors per pass, timed over 4 iterations each) [0] */
  int32_t group_width;   /* nvec > 1: vectors iterated together per pass, a multiple of 32 up to 256
                            [0: 256, or the autotuned width]; stats->status_detail reports it */
  int32_t seg_hub_edges; /* gather_kernel 3: rows of at least this many in-edges are gathered column block
                            by column block [0: 512, or the autotuned value] */
  int32_t seg_block_cols;/* gather_kernel 3: columns per block, a multiple of 32 whose values fit one CTA's
                            shared memory [0: the column cache's width, or the autotuned value] */
} mg_pr_opts;

/* ---- status ------------------------------------------------------------- */
const char *mg_status_string(mg_status s);
const char *mg_last_error(void);
const char *mg_version(void);
/* Number of usable CUDA devices (0 when there is no driver or GPU). */
int32_t mg_device_count(void);

/* ---- graph storage -------------------------------------------------------
 * Replaces CsrProblem::FromHostProblem (GASengine/csr_problem.cuh:401-621) and
 * the GPU CSC build it runs (util.cuh:55-126: offsets_to_indices, sort_by_column).
 * Copies n+1 row offsets, m column indices and m edge values (vals_t != NONE)
 * to the current device, validates them, and builds the transpose (CSC, its
 * edge permutation and the permuted values) unless MG_GRAPH_NO_CSC or
 * MG_GRAPH_SYMMETRIC. The caller keeps ownership of its arrays. */
mg_status mg_graph_create(const int32_t *row_offsets, const int32_t *col_idx, const void *edge_vals,
                          mg_dtype vals_t, int64_t n, int64_t m, uint32_t flags, mg_graph **out);

/* Replaces ~CsrProblem / ~GraphSlice (GASengine/csr_problem.cuh:217-309). NULL is a no-op. */
mg_status mg_graph_destroy(mg_graph *g);
/* Waits for an MG_GRAPH_ASYNC_UPLOAD upload and its validation (no-op otherwise). */
mg_status mg_graph_sync(mg_graph *g);

/* The CUDA stream (a cudaStream_t) every call on g is issued on, so a caller can
 * order its own work or CUDA events with the engine's. Owned by the graph. */
mg_status mg_graph_stream(const mg_graph *g, void **stream);

/* Sizes and flags of a graph (CsrProblem::nodes/edges, csr_problem.cuh:312-314). */
mg_status mg_graph_info(const mg_graph *g, int64_t *n, int64_t *m, uint32_t *flags, int32_t *device);

/* Out-degree statistics of a graph, computed on the device (synchronises the
 * graph's stream): the largest out-degree and the number of vertices without
 * out-edges. Either pointer may be NULL. */
mg_status mg_graph_degree_stats(mg_graph *g, int64_t *max_out_degree, int64_t *no_out_edges);

/* Device arrays of a graph, as GraphSlice exposes them (csr_problem.cuh:154-163):
 * row_offsets, column_indices, edge_values (NULL without values), column_offsets,
 * row_indices and the CSC->CSR edge permutation (the last three NULL without CSC;
 * equal to the CSR arrays / identity-free NULL perm for symmetric graphs).
 * Any output pointer may be NULL. */
mg_status mg_graph_device_arrays(const mg_graph *g, const int32_t **row_offsets,
                                 const int32_t **col_idx, const void **edge_vals,
                                 const int32_t **col_offsets, const int32_t **row_idx,
                                 const int32_t **csc_perm);

/* ---- the four bundled vertex programs ------------------------------------
 * Each replaces EnactorVertexCentric<CsrProblem, Program>::EnactIterativeSearch
 * (GASengine/enactor_vertex_centric.cuh:2398-2966) for its Program, followed by
 * CsrProblem::ExtractResults (csr_problem.cuh:371-396). */

/* struct bfs (Algorithms/BFS/bfs.h:28-262): depth[v] = hops from the nearest of
 * the nsrc sources (all seeded at 0), -1 when unreached. n outputs. */
mg_status mg_bfs(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth,
                 const mg_opts *opts, mg_stats *stats);

/* struct sssp (Algorithms/SSSP/sssp.h:33-409): dist[v] = shortest path length from
 * the nearest source over int32 edge values (unit weights without values),
 * INT_MAX (2147483647) when unreached. Weights must be >= 0; the graph must carry
 * I32 values or none. n outputs. */
mg_status mg_sssp(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist,
                  const mg_opts *opts, mg_stats *stats);

/* struct cc (Algorithms/CC/cc.h:32-349) as driven by Algorithms/CC/cc.cu:289-330
 * (directed forced to 0, every vertex a source): label[v] = smallest vertex id in
 * v's weakly connected component. n outputs. */
mg_status mg_cc(mg_graph *g, int32_t *label, const mg_opts *opts, mg_stats *stats);

/* struct pagerank (Algorithms/PageRank/PageRank.h:33-409).
 * REFCOMPAT: the reference's x = 0.15 + 0.85 * sum_{u->v} x_u / deg_u with its
 *   delta frontier (a vertex stays active while |dx| >= tol, default 0.01);
 *   nvec must be 1 and teleport NULL.
 * NORMALIZED: x = alpha * (P^T x + d * t) + (1 - alpha) * t with t the teleport
 *   vector (uniform when NULL), d the rank mass on dangling vertices, x_0 = t,
 *   stopping after the first iteration whose L1 change is < tol, or max_iter.
 *   nvec > 1 runs nvec personalised vectors at once: teleport is nvec x n
 *   (row-major, each row summing to 1) and ranks is nvec x n.
 * FP32 values with compensated per-destination accumulation; the residual and
 * the dangling mass are reduced in FP64. */
mg_status mg_pagerank(mg_graph *g, const float *teleport, int32_t nvec, float *ranks,
                      const mg_pr_opts *opts, mg_stats *stats);

/* BFS predecessors from a depth array (mg_bfs output), replacing the reference's
 * pred_extract (Algorithms/BFS/predextract.cuh:246-373, called at
 * Algorithms/BFS/bfs.cu:463-468): pred[v] = the largest in-neighbour u with
 * depth[v] - depth[u] == 1, else -1 (sources get their largest unreached
 * in-neighbour, as in the reference). depth and pred are host arrays unless
 * opts->device_output is set; other options are ignored. */
mg_status mg_bfs_predecessors(mg_graph *g, const int32_t *depth, int32_t *pred, const mg_opts *opts);

/* ---- batching (no reference counterpart: the reference loops the engine once
 * per source, Algorithms/BFS/bfs.cu:442-456) ---------------------------------
 * nsrc independent single-source instances in one device run; depth / dist are
 * nsrc x n, row i for srcs[i]. */
mg_status mg_bfs_batch(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth,
                       const mg_opts *opts, mg_stats *stats);
mg_status mg_sssp_batch(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dist,
                        const mg_opts *opts, mg_stats *stats);

/* A ragged batch of independent graphs stored as one disjoint union on the device.
 * Graph i has n[i] vertices and m[i] edges; its vertex v becomes vertex
 * vertex_base[i] + v of the union (vertex_base = exclusive prefix sum of n,
 * retrievable with mg_graph_ragged_bases). */
mg_status mg_graph_create_ragged(int32_t ngraphs, const int32_t *const *row_offsets,
                                 const int32_t *const *col_idx, const int64_t *n, const int64_t *m,
                                 uint32_t flags, mg_graph **out);
mg_status mg_graph_ragged_bases(const mg_graph *g, int64_t *vertex_base /* ngraphs + 1 */);
/* One BFS per member graph, from local source srcs[i], all in one device run.
 * depth is laid out like the union's vertices (sum of n[i] entries). */
mg_status mg_bfs_ragged(mg_graph *g, const int32_t *srcs, int32_t *depth, const mg_opts *opts,
                        mg_stats *stats);

/* ---- differentiation (no reference counterpart) ----------------------------
 * Adjoint of the NORMALIZED PageRank fixed point for L = sum_i dL_dranks[i]*x_i:
 * lambda solves lambda = w + alpha * (P lambda + 1_D (t . lambda)) (the gather
 * kernel run on the reversed graph), then
 *   dL/da_uv = alpha * x_u / s_u * (lambda_v - sum_k P_uk lambda_k)   (m, CSR order)
 *   dL/dt_i  = lambda_i * (1 - alpha + alpha * d)                      (n)
 * with a the F32 edge values (unit weights when opts->weighted == 0), s_u their
 * row sums, x = ranks from mg_pagerank with the same options, d its dangling mass.
 * Either gradient pointer may be NULL. nvec must be 1. */
mg_status mg_pagerank_backward(mg_graph *g, const float *teleport, const float *ranks,
                               const float *dL_dranks, float *dL_dweights, float *dL_dteleport,
                               const mg_pr_opts *opts, mg_stats *stats);

/* ---- BFS over a fixed scratch area (no reference counterpart) --------------
 * The same traversal and results as mg_bfs, for callers that must not allocate
 * device memory while they run (memory reserved up front, code running inside
 * an allocator). Frontier queues, visited bitmap, sources and the deferred-hub
 * list live in one static device array of 8.54 MB; the call allocates nothing.
 * - The array belongs to the library's device code: every process that loads
 *   the library holds 8.54 MB of it on each device where the library's kernels
 *   get loaded, whether or not it calls this function. With CUDA's lazy module
 *   loading (the default since CUDA 12) that memory is reserved when the module
 *   first loads on a device, which can be inside the first call here. Make one
 *   call (or any other engine call) on each device during set-up, before the
 *   region that must not allocate.
 * - depth must be DEVICE memory (n entries) of the graph's device; a host
 *   pointer is rejected with MG_ERR_ARG before anything runs. opts->device_output
 *   and opts->use_graph are ignored (the level loop is driven from the host).
 * - Graphs of more than MG_BFS_NOALLOC_MAX_VERTICES vertices, or more than
 *   MG_BFS_NOALLOC_MAX_SOURCES sources, are rejected with MG_ERR_ARG.
 * - The first call on a device looks up the array's device address
 *   (cudaGetSymbolAddress) and caches it; make that first call before any
 *   stream capture on the device.
 * - The array is shared by every graph on a device: two calls in flight on the
 *   same device at the same time (other threads or streams) race on it and
 *   corrupt each other's results. Serialise them. Every return, an error
 *   included, waits for the work the call queued, so serialised calls never
 *   overlap on the GPU. */
#define MG_BFS_NOALLOC_MAX_VERTICES (1 << 20)
#define MG_BFS_NOALLOC_MAX_SOURCES 1024
mg_status mg_bfs_noalloc(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depth, const mg_opts *opts,
                         mg_stats *stats);

/* ---- BFS over a 1-D vertex partition (one rank per GPU) ----------------------
 * For graphs split over several GPUs. The reference lays out, but never runs,
 * per-GPU vertex ranges (GASengine/csr_problem.cuh:339-365, GraphSlice per GPU;
 * its driver loops run on GPU 0 only, enactor_vertex_centric.cuh:2398-2966).
 * Rank r holds the out-edges and in-edges of its vertices [lo, hi) with global
 * vertex ids and the global out-degree of all n vertices. A BFS is
 *   mg_part_bfs_begin, then while !level.done:
 *     mg_part_bfs_step(bits)                 this rank's discoveries, n bits
 *     all-gather bits over the ranks         world x words, rank-major (NCCL on
 *                                            mg_part_stream's stream, or one shared
 *                                            buffer when the partitions share a GPU)
 *     mg_part_bfs_merge(gathered, world)     next frontier, same on every rank
 *   mg_part_bfs_result
 * Every rank must pass the same sources and options; the levels, directions and
 * depths then agree on all ranks (the merge folds the same words everywhere). */
typedef struct mg_part mg_part;

typedef struct mg_part_level {
  int64_t frontier;       /* vertices of the frontier the next step expands */
  int64_t frontier_edges; /* their out-edges */
  int32_t level;          /* levels completed */
  int32_t done;           /* 1: frontier empty or iter_num reached */
  int32_t direction;      /* BFS: MG_DIR_PUSH or MG_DIR_PULL for the next step */
  int32_t reserved;
  double residual;        /* PageRank: L1 change of the last iteration */
} mg_part_level;

/* lo must be a multiple of 32, hi a multiple of 32 or n. out_offsets / in_offsets
 * have hi - lo + 1 entries (row v - lo), out_idx / in_idx global ids in [0, n).
 * With MG_GRAPH_SYMMETRIC the in-edges are the out-edges (in_* may be NULL).
 * out_degree (n entries) may be NULL only when [lo, hi) = [0, n).
 * MG_GRAPH_DEVICE_INPUT: the arrays are device pointers on the current device. */
mg_status mg_part_create(int64_t n, int64_t lo, int64_t hi, const int32_t *out_offsets, const int32_t *out_idx,
                         const int32_t *in_offsets, const int32_t *in_idx, const int32_t *out_degree,
                         uint32_t flags, mg_part **out);
mg_status mg_part_destroy(mg_part *p);
/* The stream the partition's kernels run on (a cudaStream_t). */
mg_status mg_part_stream(const mg_part *p, void **stream);
/* Words of the n-bit bitmaps exchanged per level: (n + 31) / 32. */
mg_status mg_part_words(const mg_part *p, int64_t *words);
/* Resets the run and seeds the sources (opts: direction, iter_num). */
mg_status mg_part_bfs_begin(mg_part *p, const int32_t *srcs, int32_t nsrc, const mg_opts *opts,
                            mg_part_level *level);
/* This rank's discoveries of the pending level into bits (device, words entries). */
mg_status mg_part_bfs_step(mg_part *p, uint32_t *bits);
/* Folds the world's bitmaps (device, world x words) into the next frontier. */
mg_status mg_part_bfs_merge(mg_part *p, const uint32_t *gathered, int32_t world, mg_part_level *level);
/* Depths of all n vertices (replicated; host or device output) and the run's counters. */
mg_status mg_part_bfs_result(mg_part *p, int32_t *depth, int32_t device_output, mg_stats *stats);

/* PageRank over the partition: MG_PR_NORMALIZED with the uniform teleport,
 * unweighted (opts: alpha, tol, max_iter). Per iteration
 *     mg_part_pr_step(slice)                 this rank's new ranks of [lo, hi)
 *                                            into slice (device, hi - lo floats)
 *     all-gather the slices, each padded to `stride` floats (>= the largest
 *     slice), rank-major
 *     mg_part_pr_merge(gathered, world, stride, cuts)   cuts (host, world + 1)
 *                                            as in the partition, [0, ..., n]
 * until level.done (L1 change below tol, or max_iter). Every rank keeps the
 * whole iterate; the merge's sums run in a fixed order, so all ranks stop at the
 * same iteration. */
mg_status mg_part_pr_begin(mg_part *p, const mg_pr_opts *opts, mg_part_level *level);
mg_status mg_part_pr_step(mg_part *p, float *slice);
mg_status mg_part_pr_merge(mg_part *p, const float *gathered, int32_t world, int64_t stride, const int64_t *cuts,
                           mg_part_level *level);
/* Ranks of all n vertices (host or device output) and the run's counters. */
mg_status mg_part_pr_result(mg_part *p, float *ranks, int32_t device_output, mg_stats *stats);

/* ---- Per-level trace of the last run ----------------------------------------
 * What the reference prints with verbose=1 (frontier size per iteration,
 * GASengine/enactor_vertex_centric.cuh:2528-2546), recorded on the device by the
 * level-end code of mg_bfs, mg_sssp and single-vector mg_pagerank (MG_PR_NORMALIZED)
 * on a graph, for the first MG_TRACE_LEVELS levels. One record per level:
 *   BFS:      frontier = vertices expanded, frontier_edges = their out-edges,
 *             direction = MG_DIR_PUSH / MG_DIR_PULL;
 *   SSSP:     frontier = vertices relaxed, frontier_edges = their out-edges (the
 *             edges the round inspects; both directions with directed = 0);
 *   PageRank: frontier = n, value = the iteration's L1 change;
 *   every record: time_ns, the device clock at the level's end.
 * *count = records written (min(levels, cap, MG_TRACE_LEVELS)). */
#define MG_TRACE_LEVELS 4096
typedef struct mg_level_record {
  int32_t level;
  int32_t direction;
  int64_t frontier;
  int64_t frontier_edges;
  double value;
  uint64_t time_ns; /* device clock (PTX %globaltimer) when the level ended: differences give per-level
                       durations */
} mg_level_record;
mg_status mg_graph_trace(mg_graph *g, mg_level_record *out, int32_t cap, int32_t *count);

/* ---- Traversal tuning (per graph) -------------------------------------------
 * Thresholds and launch shapes of the traversal kernels, read by every later call
 * on the graph (the reference fixes its equivalents at compile time, e.g. the
 * expand/contract tile sizes of GASengine/vertex_centric/*_problem_type.cuh).
 * mg_tuning_defaults fills the defaults; mg_graph_set_tuning checks each field
 * against its range (MG_ERR_ARG, nothing changed, on a bad value). The Python
 * package's tuning module times candidate sets on the device for a graph class
 * and caches the fastest in a JSON file. */
typedef struct mg_tuning {
  int32_t sssp_heavy;       /* SSSP round: frontier vertices of at least this many edges are cut into chunks of
                               256 edges that every warp of the grid relaxes; lighter ones are walked by the warp
                               that drew them [256; 1 .. 2^30] */
  int32_t sssp_heavy_small; /* the same for a frontier of fewer vertices than the grid has threads [32; 1 ..
                               sssp_heavy] */
  int32_t sssp_ctas_per_sm; /* CTAs of 256 threads per SM of the SSSP round kernels [4; 1 .. 8] */
  int32_t sssp_chunk_cap;   /* SSSP chunk list capacity in chunks; 0: the bound of the graph's edges (at most
                               2^23); past it a warp walks its heavy vertices itself [0; 0 .. 2^30] */
  int32_t sssp_batch_heavy; /* mg_sssp_batch (interleaved rows): frontier items of at least this many edges are cut
                               into chunks of 128 edges for every warp of the grid [32; 1 .. 2^30] */
  int32_t bfs_cta_th;       /* BFS push levels: out-degree from which the whole CTA expands a frontier vertex
                               [512; 32 .. 2^30] */
  int32_t bfs_grid_th;      /* out-degree from which a vertex of a large frontier is spread over the whole grid
                               [4096; 32 .. 2^30] */
  int32_t bfs_defer_warp;   /* 1: a frontier filling under an eighth of the grid's threads sends every vertex of
                               32+ edges to the grid-wide pass; 0: only those of bfs_cta_th+ edges [1; 0 .. 1] */
  int32_t bfs_persist_max;  /* push levels of at most this many frontier vertices ... [65536; 0 .. 2^30] */
  int32_t bfs_persist_edges;/* ... and at most this many frontier out-edges run in one persistent cooperative
                               launch (0: never) [131072; 0 .. 2^30] */
  int32_t bfs_alpha;        /* direction rule: pull once the frontier's out-edges exceed the unvisited vertices'
                               out-edges / alpha [14; 1 .. 2^20] */
  int32_t bfs_beta;         /* ... and back to push when the frontier holds fewer than n / beta vertices
                               [24; 1 .. 2^20] */
  int32_t bfs_sparse_degree;/* MG_DIR_AUTO stays top-down on graphs of mean out-degree <= this [8; 0 .. 2^20] */
  int32_t bfs_ctas_per_sm;  /* CTAs of 256 threads per SM of the BFS level kernels [4; 1 .. 8] */
  int32_t bfs_tail_max;     /* push levels of at most this many frontier vertices ... [512; 0 .. 2^30] */
  int32_t bfs_tail_edges;   /* ... and out-edges run one after another in a single CTA, one launch for the
                               run of them, wherever they occur (0: never) [16384; 0 .. 2^30] */
  int32_t cc_rounds;        /* CC: rounds that link every vertex to its next neighbour before the largest sampled
                               component is picked and only the vertices outside it read their other edges
                               [1; 0 .. 8] */
  int32_t reserved[15];
} mg_tuning;
void mg_tuning_defaults(mg_tuning *t);
mg_status mg_graph_set_tuning(mg_graph *g, const mg_tuning *t);
mg_status mg_graph_get_tuning(mg_graph *g, mg_tuning *t);

/* ---- Test hooks: host-side fault injection ----------------------------------
 * For failure-path tests; nothing here faults, traps or hangs a device.
 * mg_debug_fail_alloc(k): the k-th device allocation from now, and every later
 *   one, fails as if the device were out of memory (the call in progress returns
 *   MG_ERR_OOM); k = 0 disarms.
 * mg_debug_barrier_skew(extra, poll_limit): the persistent BFS kernel's grid
 *   barriers wait for `extra` arrivals more than there are blocks, polling at
 *   most poll_limit times, so the next mg_bfs that takes the persistent path
 *   returns MG_ERR_TIMEOUT and leaves the device usable; extra = 0 restores. */
mg_status mg_debug_fail_alloc(int64_t k);
mg_status mg_debug_barrier_skew(int32_t extra, int64_t poll_limit);
/* mg_debug_seg_plan(g, hub_edges, block_cols, out): builds (or reuses) the graph's
 * segmented PageRank gather plan for that shape and checks it on the host; out[8]
 * receives {hub rows, fragments, groups, sliced-ELL entries, fragments listed
 * once, fragments whose entries match their row's edges in that block, hub arrival
 * counters not at zero, CTA ranges covering every group (1/0)}. Test hook. */
mg_status mg_debug_seg_plan(mg_graph *g, int32_t hub_edges, int32_t block_cols, int64_t *out);

#ifdef __cplusplus
}
#endif
#endif /* MAPGRAPH_B200_H */
