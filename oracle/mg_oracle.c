/*
 * mg_oracle.c -- test infrastructure (the checker), never on the product path.
 *
 * A plain-C restatement of the reference's algorithms for the GAS hot path, used
 * only by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg to
 * check and time the CUDA engine. Every routine is serial and works on host CSR
 * arrays (int32 row offsets / column indices). It is pinned against the
 * reference's own CPU functions (oracle/_ref, built from the reference tree) and
 * against golden vectors recorded from them (tests/golden/).
 *
 * Conventions shared with the engine:
 *   - BFS depth of an unreached vertex is -1; sources have depth 0
 *     (Algorithms/BFS/bfs.h:36, :71-78).
 *   - SSSP distance of an unreached vertex is INT_MAX, the GPU engine's
 *     INIT_VALUE (Algorithms/SSSP/sssp.h:43). The reference CPU check writes
 *     100000000 instead (Algorithms/SSSP/sssp.cu:139); tests map that sentinel.
 *   - CC labels are the minimum vertex id of each weakly connected component
 *     (Algorithms/CC/cc.h:93-148 starts from labels = ids and propagates minima
 *     over CSR and CSC; Algorithms/CC/cc.cu:132-199 iterates to the same fixed point).
 *   - directed == 0 follows out-edges and in-edges (the CSC), each in-edge with
 *     its own weight (the engine indexes weights through the CSC->CSR edge
 *     permutation, GASengine/vertex_centric/expand_atomic/cta.cuh:327-331).
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* BFS: restates CPUBFS (Algorithms/BFS/bfs.cu:56-143) with num_srcs sources all
 * seeded at depth 0, which is what the engine does for a multi-source
 * EnactIterativeSearch (Algorithms/BFS/bfs.h:71-78).                        */
void mgo_bfs(int n, const int *ro, const int *ci, const int *co, const int *ri,
             int directed, int nsrc, const int *srcs, int *depth) {
  int *queue = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int head = 0, tail = 0;
  for (int i = 0; i < n; i++) depth[i] = -1;
  for (int s = 0; s < nsrc; s++) {
    if (depth[srcs[s]] == -1) {
      depth[srcs[s]] = 0;
      queue[tail++] = srcs[s];
    }
  }
  while (head < tail) {
    int v = queue[head++];
    int nd = depth[v] + 1;
    for (int e = ro[v]; e < ro[v + 1]; e++) {
      int u = ci[e];
      if (depth[u] == -1) {
        depth[u] = nd;
        queue[tail++] = u;
      }
    }
    if (!directed) {
      for (int e = co[v]; e < co[v + 1]; e++) {
        int u = ri[e];
        if (depth[u] == -1) {
          depth[u] = nd;
          queue[tail++] = u;
        }
      }
    }
  }
  free(queue);
}

/* ------------------------------------------------------------------------- */
/* SSSP: exact shortest distances by Dijkstra with a binary heap. The reference
 * CPU check (Algorithms/SSSP/sssp.cu:127-199) is an O(n^2) Dijkstra and the GPU
 * engine a frontier Bellman-Ford (Algorithms/SSSP/sssp.h:242-402); all three
 * reach the same unique fixed point for non-negative integer weights.
 * w is indexed by CSR edge; cw (CSC weights, already permuted) is read only when
 * directed == 0.                                                             */
typedef struct { int64_t d; int v; } heap_item;

static void heap_push(heap_item *h, int *size, heap_item it) {
  int i = (*size)++;
  while (i > 0) {
    int p = (i - 1) / 2;
    if (h[p].d <= it.d) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = it;
}

static heap_item heap_pop(heap_item *h, int *size) {
  heap_item top = h[0];
  heap_item last = h[--(*size)];
  int i = 0;
  for (;;) {
    int c = 2 * i + 1;
    if (c >= *size) break;
    if (c + 1 < *size && h[c + 1].d < h[c].d) c++;
    if (h[c].d >= last.d) break;
    h[i] = h[c];
    i = c;
  }
  if (*size > 0) h[i] = last;
  return top;
}

void mgo_sssp(int n, const int *ro, const int *ci, const int *w, const int *co,
              const int *ri, const int *cw, int directed, int nsrc, const int *srcs,
              int *dist) {
  int64_t m_total = (int64_t)ro[n] + (directed ? 0 : (int64_t)co[n]);
  heap_item *h = (heap_item *)malloc(sizeof(heap_item) * (size_t)(m_total + nsrc + 1));
  int size = 0;
  int64_t *d = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) d[i] = INT64_MAX;
  for (int s = 0; s < nsrc; s++) {
    if (d[srcs[s]] != 0) {
      d[srcs[s]] = 0;
      heap_item it = {0, srcs[s]};
      heap_push(h, &size, it);
    }
  }
  while (size > 0) {
    heap_item it = heap_pop(h, &size);
    if (it.d != d[it.v]) continue;
    int v = it.v;
    for (int e = ro[v]; e < ro[v + 1]; e++) {
      int64_t nd = it.d + (int64_t)w[e];
      if (nd < d[ci[e]]) {
        d[ci[e]] = nd;
        heap_item ni = {nd, ci[e]};
        heap_push(h, &size, ni);
      }
    }
    if (!directed) {
      for (int e = co[v]; e < co[v + 1]; e++) {
        int64_t nd = it.d + (int64_t)cw[e];
        if (nd < d[ri[e]]) {
          d[ri[e]] = nd;
          heap_item ni = {nd, ri[e]};
          heap_push(h, &size, ni);
        }
      }
    }
  }
  for (int i = 0; i < n; i++) dist[i] = d[i] == INT64_MAX ? INT_MAX : (int)d[i];
  free(d);
  free(h);
}

/* ------------------------------------------------------------------------- */
/* CC: minimum vertex id per weakly connected component. CPUCC
 * (Algorithms/CC/cc.cu:132-199) reaches it by min-label sweeps over the CSR and
 * the CSC; here a union-find that always links the larger root under the smaller
 * one reaches the same labels, since every root is its component's minimum.   */
static int uf_find(int *p, int x) {
  while (p[x] != x) {
    p[x] = p[p[x]];
    x = p[x];
  }
  return x;
}

void mgo_cc(int n, const int *ro, const int *ci, int *label) {
  for (int i = 0; i < n; i++) label[i] = i;
  for (int v = 0; v < n; v++) {
    for (int e = ro[v]; e < ro[v + 1]; e++) {
      int a = uf_find(label, v), b = uf_find(label, ci[e]);
      if (a < b) label[b] = a;
      else if (b < a) label[a] = b;
    }
  }
  for (int v = 0; v < n; v++) label[v] = uf_find(label, v);
}

/* ------------------------------------------------------------------------- */
/* PageRank, reference-compatible mode, FP64, on the GPU engine's schedule:
 *   frontier F_0 = all vertices (Algorithms/PageRank/PageRank.h:130-139);
 *   each iteration, for v in F: g_v = sum over in-edges u->v of x_u / deg_u
 *   (gather_edge, PageRank.h:233-243), x_v' = 0.15 + 0.85 g_v (apply,
 *   PageRank.h:257-283), changed_v = |x_v' - x_v| >= 0.01; all gathers read the
 *   previous iterate (gather, then apply: GASengine/enactor_vertex_centric.cuh
 *   2561-2575);
 *   F_{i+1} = out-neighbours of the changed vertices, without duplicates
 *   (expand_edge PageRank.h:328-363, allow_duplicates = false);
 *   stop when F is empty or after iter_num iterations.
 * directed == 0: deg = outdeg + indeg and the gather and the expansion run over
 * both directions (PageRank.h:141-161).
 * Returns the number of iterations run.                                      */
int mgo_pr_refcompat(int n, const int *ro, const int *ci, const int *co, const int *ri,
                     int directed, int iter_num, double delta, double *x) {
  double *g = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int *deg = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *front = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *next = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  unsigned char *flag = (unsigned char *)calloc((size_t)(n > 0 ? n : 1), 1);
  unsigned char *chg = (unsigned char *)calloc((size_t)(n > 0 ? n : 1), 1);
  int nf = n, it = 0;
  for (int v = 0; v < n; v++) {
    x[v] = 0.15;
    front[v] = v;
    deg[v] = (ro[v + 1] - ro[v]) + (directed ? 0 : (co[v + 1] - co[v]));
  }
  while (nf > 0 && it < iter_num) {
    for (int i = 0; i < nf; i++) {
      int v = front[i];
      double s = 0.0;
      for (int e = co[v]; e < co[v + 1]; e++) s += x[ri[e]] / (double)deg[ri[e]];
      if (!directed)
        for (int e = ro[v]; e < ro[v + 1]; e++) s += x[ci[e]] / (double)deg[ci[e]];
      g[v] = s;
    }
    for (int i = 0; i < nf; i++) {
      int v = front[i];
      double nv = 0.15 + 0.85 * g[v];
      chg[v] = fabs(nv - x[v]) >= delta;
      x[v] = nv;
    }
    int nn = 0;
    for (int i = 0; i < nf; i++) {
      int v = front[i];
      if (!chg[v]) continue;
      for (int e = ro[v]; e < ro[v + 1]; e++) {
        int u = ci[e];
        if (!flag[u]) { flag[u] = 1; next[nn++] = u; }
      }
      if (!directed)
        for (int e = co[v]; e < co[v + 1]; e++) {
          int u = ri[e];
          if (!flag[u]) { flag[u] = 1; next[nn++] = u; }
        }
    }
    for (int i = 0; i < nf; i++) chg[front[i]] = 0;
    for (int i = 0; i < nn; i++) flag[next[i]] = 0;
    int *t = front; front = next; next = t;
    nf = nn;
    it++;
  }
  free(g); free(deg); free(front); free(next); free(flag); free(chg);
  return it;
}

/* ------------------------------------------------------------------------- */
/* PageRank, normalised mode, FP64 (no reference counterpart; the engine's
 * normalised mode is specified by the power iteration
 *   x_{k+1} = alpha * (P^T x_k + d_k * t) + (1 - alpha) * t,
 *   d_k = sum of x_k over dangling vertices (no out-edges / zero weight sum),
 *   P_uv = a_uv / s_u with s_u = sum_k a_uk (a_uv = 1 when a == NULL),
 * with x_0 = t, t the teleport vector (uniform 1/n when t == NULL), stopping
 * after the first iteration whose L1 change sum|x_{k+1} - x_k| is below tol, or
 * after max_iter iterations). Push form over the CSR.
 * Returns the number of iterations; *resid gets the last L1 change.          */
int mgo_pr_normalized(int n, const int *ro, const int *ci, const float *a, double alpha,
                      double tol, int max_iter, const double *t, double *x, double *resid) {
  double *s = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *xn = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *tt = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int v = 0; v < n; v++) {
    double sv = 0.0;
    for (int e = ro[v]; e < ro[v + 1]; e++) sv += a ? (double)a[e] : 1.0;
    s[v] = sv;
    tt[v] = t ? t[v] : 1.0 / (double)n;
    x[v] = tt[v];
  }
  int it = 0;
  double r = 0.0;
  while (it < max_iter) {
    double dang = 0.0;
    for (int v = 0; v < n; v++) {
      xn[v] = 0.0;
      if (s[v] == 0.0) dang += x[v];
    }
    for (int u = 0; u < n; u++) {
      if (s[u] == 0.0) continue;
      double xu = x[u] / s[u];
      for (int e = ro[u]; e < ro[u + 1]; e++) xn[ci[e]] += xu * (a ? (double)a[e] : 1.0);
    }
    r = 0.0;
    for (int v = 0; v < n; v++) {
      double nv = alpha * (xn[v] + dang * tt[v]) + (1.0 - alpha) * tt[v];
      r += fabs(nv - x[v]);
      x[v] = nv;
    }
    it++;
    if (r < tol) break;
  }
  if (resid) *resid = r;
  free(s); free(xn); free(tt);
  return it;
}

/* Same power iteration started from a given x (warm start), run until the L1
 * change drops below tol or max_iter; returns L = sum_i w_i x_i. Used for central
 * finite differences of the PageRank adjoint.                                 */
double mgo_pr_loss(int n, const int *ro, const int *ci, const float *a, double alpha,
                   double tol, int max_iter, const double *t, const double *w, double *x) {
  double *s = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *xn = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int v = 0; v < n; v++) {
    double sv = 0.0;
    for (int e = ro[v]; e < ro[v + 1]; e++) sv += a ? (double)a[e] : 1.0;
    s[v] = sv;
  }
  for (int it = 0; it < max_iter; it++) {
    double dang = 0.0;
    for (int v = 0; v < n; v++) {
      xn[v] = 0.0;
      if (s[v] == 0.0) dang += x[v];
    }
    for (int u = 0; u < n; u++) {
      if (s[u] == 0.0) continue;
      double xu = x[u] / s[u];
      for (int e = ro[u]; e < ro[u + 1]; e++) xn[ci[e]] += xu * (a ? (double)a[e] : 1.0);
    }
    double r = 0.0;
    for (int v = 0; v < n; v++) {
      double tv = t ? t[v] : 1.0 / (double)n;
      double nv = alpha * (xn[v] + dang * tv) + (1.0 - alpha) * tv;
      r += fabs(nv - x[v]);
      x[v] = nv;
    }
    if (r < tol) break;
  }
  double L = 0.0;
  for (int v = 0; v < n; v++) L += w[v] * x[v];
  free(s); free(xn);
  return L;
}

/* ------------------------------------------------------------------------- */
/* PageRank adjoint, FP64. For L = sum_i w_i x_i at the fixed point of the
 * normalised iteration above, the adjoint lambda solves
 *   lambda = w + alpha * (P lambda + 1_D (t . lambda))
 * (the transpose of the forward system; 1_D marks dangling vertices). Then
 *   dL/da_uv = alpha * x_u / s_u * (lambda_v - sum_k P_uk lambda_k)
 *   dL/dt_i  = lambda_i * (1 - alpha + alpha * d),   d = sum_{u in D} x_u.
 * x is the forward solution supplied by the caller. Iterates until the L1
 * change of lambda is below tol or max_iter. Returns the iterations run.      */
int mgo_pr_adjoint(int n, const int *ro, const int *ci, const float *a, double alpha,
                   const double *t, const double *x, const double *w, double tol,
                   int max_iter, double *lambda, double *grad_a, double *grad_t) {
  double *s = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *ln = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double d = 0.0;
  for (int v = 0; v < n; v++) {
    double sv = 0.0;
    for (int e = ro[v]; e < ro[v + 1]; e++) sv += a ? (double)a[e] : 1.0;
    s[v] = sv;
    if (sv == 0.0) d += x[v];
    lambda[v] = w[v];
  }
  int it = 0;
  while (it < max_iter) {
    double tl = 0.0;
    for (int v = 0; v < n; v++) tl += (t ? t[v] : 1.0 / (double)n) * lambda[v];
    double r = 0.0;
    for (int u = 0; u < n; u++) {
      double acc;
      if (s[u] == 0.0) {
        acc = tl;
      } else {
        acc = 0.0;
        for (int e = ro[u]; e < ro[u + 1]; e++)
          acc += (a ? (double)a[e] : 1.0) * lambda[ci[e]];
        acc /= s[u];
      }
      ln[u] = w[u] + alpha * acc;
    }
    for (int v = 0; v < n; v++) {
      r += fabs(ln[v] - lambda[v]);
      lambda[v] = ln[v];
    }
    it++;
    if (r < tol) break;
  }
  for (int u = 0; u < n; u++) {
    if (s[u] == 0.0) continue;
    double pl = 0.0;
    for (int e = ro[u]; e < ro[u + 1]; e++) pl += (a ? (double)a[e] : 1.0) * lambda[ci[e]];
    pl /= s[u];
    double c = alpha * x[u] / s[u];
    for (int e = ro[u]; e < ro[u + 1]; e++) grad_a[e] = c * (lambda[ci[e]] - pl);
  }
  for (int v = 0; v < n; v++) grad_t[v] = lambda[v] * (1.0 - alpha + alpha * d);
  free(s); free(ln);
  return it;
}
