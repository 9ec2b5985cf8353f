/*
 * mapgraph_b200_io.h -- host-side graph ingest and seeded synthetic generators.
 *
 * Host C ABI (no CUDA types). All generators are counter-based (splitmix64 of
 * (seed, stream, index)), so the same seed gives the same graph on any machine
 * and any thread count. Every routine returns a CSR whose rows list their edges in
 * a canonical order, ready for mg_graph_create() (mapgraph_b200.h).
 */
#ifndef MAPGRAPH_B200_IO_H
#define MAPGRAPH_B200_IO_H

#include <stdint.h>
#include "mapgraph_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A host CSR owned by the library; release with mg_host_csr_free(). */
typedef struct mg_host_csr {
  int64_t n;               /* vertices */
  int64_t m;               /* directed edges */
  int32_t *row_offsets;    /* n + 1 */
  int32_t *col_idx;        /* m */
  int32_t *weights_i32;    /* m, or NULL */
  float *weights_f32;      /* m, or NULL */
} mg_host_csr;

void mg_host_csr_free(mg_host_csr *g);

/* Weight kinds for the generators. */
#define MG_W_NONE 0        /* no weights */
#define MG_W_UNIFORM_INT 1 /* int32 uniform in [p0, p1] */
#define MG_W_LOGNORMAL 2   /* float exp(N(p0, p1)) (mean p0, sigma p1 of the log) */

/* Directed Erdos-Renyi multigraph: m edges with uniform endpoints; a self-loop
 * draw is redrawn, so exactly m edges come back; duplicates are kept. */
mg_status mg_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t wkind, double p0, double p1,
                    mg_host_csr *out);

/* R-MAT: 2^scale vertices, edge_factor * 2^scale generated edges, quadrant
 * probabilities (a, b, c, 1-a-b-c) at each of the scale levels, no noise and no
 * vertex-id permutation. Self-loops are dropped, duplicates kept. symmetrize != 0
 * adds the reverse of every edge with the same weight. */
mg_status mg_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                      uint64_t seed, int32_t symmetrize, int32_t wkind, double p0, double p1,
                      mg_host_csr *out);

/* rows x cols 2-D lattice, id = r * cols + c, 4-neighbour edges in both
 * directions, plus round(longrange_frac * lattice directed edges) uniform random
 * vertex pairs added in both directions. One weight per undirected edge. */
mg_status mg_gen_lattice(int32_t rows, int32_t cols, double longrange_frac, uint64_t seed,
                         int32_t wkind, double p0, double p1, mg_host_csr *out);

/* Matrix Market ingest with the reference's semantics
 * (b40c/graph/builder/market.cuh:43-166, b40c/graph/csr_graph.cuh:74-164):
 * '%' lines are comments; the first other line is "rows cols entries" and must
 * be square; entries are 1-based "row col [value]" with value 1 when absent;
 * values are read as double and stored both truncated to int32 and as float;
 * undirected != 0 also inserts every reverse edge; rows keep file order
 * (stable sort by row). Returns MG_ERR_ARG for a malformed or truncated file. */
mg_status mg_read_market(const char *path, int32_t undirected, mg_host_csr *out);

/* Writes a host CSR as a Matrix Market file (1-based "row col [value]" lines in
 * CSR order; values: 0 none ("pattern"), 1 the int32 weights, 2 the float
 * weights). Reading it back with mg_read_market(path, 0, ...) gives the same CSR. */
mg_status mg_write_market(const char *path, const mg_host_csr *g, int32_t values);

/* Binary CSR cache (no reference counterpart: the reference re-parses the text
 * file on every run): mg_save_csr writes the arrays of a host CSR, mg_load_csr
 * reads them back (release with mg_host_csr_free). Native byte order. */
mg_status mg_save_csr(const char *path, const mg_host_csr *g);
mg_status mg_load_csr(const char *path, mg_host_csr *out);

/* Host CSR -> CSC (stable: within a column, edges in CSR order, as the
 * reference's std::stable_sort by column, csr_graph.cuh:128-153). perm[k] is the
 * CSR edge id of CSC slot k. Arrays are caller-allocated (n+1, m, m). */
mg_status mg_host_csr_to_csc(int64_t n, int64_t m, const int32_t *row_offsets,
                             const int32_t *col_idx, int32_t *col_offsets, int32_t *row_idx,
                             int32_t *perm);

#ifdef __cplusplus
}
#endif
#endif /* MAPGRAPH_B200_IO_H */
