// host_io.cpp -- host-side ingest (Matrix Market) and seeded synthetic graph
// generators. Plain C++17 + OpenMP; no CUDA.
//
// Generators are counter-based: every random draw is splitmix64 of a key derived
// from (seed, stream) mixed with the draw's index, so the graph is a pure
// function of the seed, independent of thread count and scheduling.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <omp.h>

#include "mapgraph_b200_io.h"
#include "mg_internal.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Stream keys: one independent random sequence per purpose.
enum : uint64_t { S_SRC = 1, S_DST = 2, S_WEIGHT = 3, S_RMAT = 4, S_LONG = 5, S_REDRAW = 6 };

inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return splitmix64(seed * 0xD1B54A32D192ED03ull + stream * 0x632BE59BD9B4E019ull);
}
inline uint64_t draw(uint64_t key, uint64_t idx) { return splitmix64(key ^ (idx * 0x9E3779B97F4A7C15ull)); }
inline double unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)

struct WeightGen {
  int32_t kind;
  double p0, p1;
  uint64_t key;
  bool is_float() const { return kind == MG_W_LOGNORMAL; }
  int32_t ival(uint64_t idx) const {
    int64_t lo = (int64_t)p0, hi = (int64_t)p1;
    return (int32_t)(lo + (int64_t)(draw(key, idx) % (uint64_t)(hi - lo + 1)));
  }
  float fval(uint64_t idx) const {
    // Box-Muller from two independent draws.
    double u1 = unit(draw(key, 2 * idx)), u2 = unit(draw(key, 2 * idx + 1));
    if (u1 < 1e-300) u1 = 1e-300;
    double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    return (float)std::exp(p0 + p1 * z);
  }
};

bool valid_weights(int32_t wkind, double p0, double p1) {
  if (wkind == MG_W_NONE) return true;
  if (wkind == MG_W_UNIFORM_INT) return p0 <= p1 && p0 >= -2147483648.0 && p1 <= 2147483647.0;
  if (wkind == MG_W_LOGNORMAL) return p1 >= 0.0;
  return false;
}

// COO edge list with one weight slot.
struct Coo {
  std::vector<int32_t> src, dst, wi;
  std::vector<float> wf;
};

// Builds a CSR from COO. Rows come out sorted by (column, weight) when
// canonical != 0 (generated graphs), or in COO order (stable by row) otherwise
// (file ingest, matching the reference's std::stable_sort by row).
mg_status coo_to_csr(int64_t n, Coo &coo, int32_t wkind, bool canonical, mg_host_csr *out) {
  const int64_t m = (int64_t)coo.src.size();
  if (n < 0 || n > INT32_MAX - 1 || m > INT32_MAX) return MG_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  out->n = n;
  out->m = m;
  out->row_offsets = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(n + 1));
  out->col_idx = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  bool has_i = wkind == MG_W_UNIFORM_INT, has_f = wkind == MG_W_LOGNORMAL;
  if (has_i) out->weights_i32 = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  if (has_f) out->weights_f32 = (float *)std::malloc(sizeof(float) * (size_t)std::max<int64_t>(m, 1));
  if (!out->row_offsets || !out->col_idx || (has_i && !out->weights_i32) || (has_f && !out->weights_f32)) {
    mg_host_csr_free(out);
    return MG_ERR_OOM;
  }
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  if (canonical) {
    // GCC atomic builtins on the plain counters (no std::atomic aliasing).
    int64_t *acnt = cnt.data();
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) __atomic_fetch_add(&acnt[coo.src[e]], (int64_t)1, __ATOMIC_RELAXED);
  } else {
    for (int64_t e = 0; e < m; e++) cnt[coo.src[e]]++;
  }
  int64_t run = 0;
  for (int64_t v = 0; v < n; v++) {
    int64_t c = cnt[v];
    out->row_offsets[v] = (int32_t)run;
    cnt[v] = run;
    run += c;
  }
  out->row_offsets[n] = (int32_t)run;
  if (canonical) {
    std::vector<int64_t> slot((size_t)m);
    int64_t *cur = cnt.data();
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) slot[e] = __atomic_fetch_add(&cur[coo.src[e]], (int64_t)1, __ATOMIC_RELAXED);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) {
      out->col_idx[slot[e]] = coo.dst[e];
      if (has_i) out->weights_i32[slot[e]] = coo.wi[e];
      if (has_f) out->weights_f32[slot[e]] = coo.wf[e];
    }
    // Canonical row order: sort each row by (column, weight).
#pragma omp parallel
    {
      std::vector<std::pair<int32_t, int32_t>> bi;
      std::vector<std::pair<int32_t, float>> bf;
#pragma omp for schedule(dynamic, 4096)
      for (int64_t v = 0; v < n; v++) {
        int64_t b = out->row_offsets[v], e = out->row_offsets[v + 1];
        if (e - b < 2) continue;
        if (has_f) {
          bf.clear();
          for (int64_t k = b; k < e; k++) bf.emplace_back(out->col_idx[k], out->weights_f32[k]);
          std::sort(bf.begin(), bf.end());
          for (int64_t k = b; k < e; k++) { out->col_idx[k] = bf[k - b].first; out->weights_f32[k] = bf[k - b].second; }
        } else if (has_i) {
          bi.clear();
          for (int64_t k = b; k < e; k++) bi.emplace_back(out->col_idx[k], out->weights_i32[k]);
          std::sort(bi.begin(), bi.end());
          for (int64_t k = b; k < e; k++) { out->col_idx[k] = bi[k - b].first; out->weights_i32[k] = bi[k - b].second; }
        } else {
          std::sort(out->col_idx + b, out->col_idx + e);
        }
      }
    }
  } else {
    for (int64_t e = 0; e < m; e++) {
      int64_t s = cnt[coo.src[e]]++;
      out->col_idx[s] = coo.dst[e];
      if (has_i) out->weights_i32[s] = coo.wi[e];
      if (has_f) out->weights_f32[s] = coo.wf[e];
    }
  }
  return MG_OK;
}

}  // namespace

extern "C" {

void mg_host_csr_free(mg_host_csr *g) {
  if (!g) return;
  std::free(g->row_offsets);
  std::free(g->col_idx);
  std::free(g->weights_i32);
  std::free(g->weights_f32);
  std::memset(g, 0, sizeof(*g));
}

mg_status mg_gen_er(int64_t n, int64_t m, uint64_t seed, int32_t wkind, double p0, double p1,
                    mg_host_csr *out) {
  if (!out || n < 2 || m < 0 || m > INT32_MAX || n > INT32_MAX - 1 || !valid_weights(wkind, p0, p1)) {
    mg_set_error("mg_gen_er: invalid arguments");
    return MG_ERR_ARG;
  }
  Coo coo;
  coo.src.resize(m);
  coo.dst.resize(m);
  WeightGen wg{wkind, p0, p1, stream_key(seed, S_WEIGHT)};
  if (wkind == MG_W_UNIFORM_INT) coo.wi.resize(m);
  if (wkind == MG_W_LOGNORMAL) coo.wf.resize(m);
  const uint64_t ks = stream_key(seed, S_SRC), kd = stream_key(seed, S_DST), kr = stream_key(seed, S_REDRAW);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    int64_t u = (int64_t)(draw(ks, e) % (uint64_t)n);
    int64_t v = (int64_t)(draw(kd, e) % (uint64_t)n);
    for (uint64_t t = 1; v == u; t++) v = (int64_t)(draw(kr, (uint64_t)e * 64 + t) % (uint64_t)n);
    coo.src[e] = (int32_t)u;
    coo.dst[e] = (int32_t)v;
    if (wkind == MG_W_UNIFORM_INT) coo.wi[e] = wg.ival(e);
    if (wkind == MG_W_LOGNORMAL) coo.wf[e] = wg.fval(e);
  }
  return coo_to_csr(n, coo, wkind, true, out);
}

mg_status mg_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                      uint64_t seed, int32_t symmetrize, int32_t wkind, double p0, double p1,
                      mg_host_csr *out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
      !valid_weights(wkind, p0, p1)) {
    mg_set_error("mg_gen_rmat: invalid arguments");
    return MG_ERR_ARG;
  }
  const int64_t n = (int64_t)1 << scale;
  const int64_t mg = n * (int64_t)edge_factor;
  if (mg * (symmetrize ? 2 : 1) > INT32_MAX) {
    mg_set_error("mg_gen_rmat: edge count exceeds int32");
    return MG_ERR_ARG;
  }
  const uint64_t kq = stream_key(seed, S_RMAT);
  WeightGen wg{wkind, p0, p1, stream_key(seed, S_WEIGHT)};
  // Pass 1: endpoints of every generated edge (self-loops flagged by u == v).
  std::vector<int32_t> gu(mg), gv(mg);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < mg; e++) {
    uint32_t u = 0, v = 0;
    for (int l = 0; l < scale; l++) {
      double r = unit(draw(kq, (uint64_t)e * (uint64_t)scale + (uint64_t)l));
      uint32_t bu, bv;
      if (r < a) { bu = 0; bv = 0; }
      else if (r < ab) { bu = 0; bv = 1; }
      else if (r < abc) { bu = 1; bv = 0; }
      else { bu = 1; bv = 1; }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    gu[e] = (int32_t)u;
    gv[e] = (int32_t)v;
  }
  // Pass 2: compact away self-loops (prefix count per block keeps it deterministic).
  const int nt = omp_get_max_threads();
  std::vector<int64_t> keep(nt + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    int64_t lo = mg * t / nt, hi = mg * (t + 1) / nt, k = 0;
    for (int64_t e = lo; e < hi; e++) k += gu[e] != gv[e];
    keep[t + 1] = k;
  }
  for (int t = 0; t < nt; t++) keep[t + 1] += keep[t];
  const int64_t mk = keep[nt];
  const int64_t mult = symmetrize ? 2 : 1;
  Coo coo;
  coo.src.resize(mk * mult);
  coo.dst.resize(mk * mult);
  if (wkind == MG_W_UNIFORM_INT) coo.wi.resize(mk * mult);
  if (wkind == MG_W_LOGNORMAL) coo.wf.resize(mk * mult);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    int64_t lo = mg * t / nt, hi = mg * (t + 1) / nt, k = keep[t];
    for (int64_t e = lo; e < hi; e++) {
      if (gu[e] == gv[e]) continue;
      int64_t s = k * mult;
      coo.src[s] = gu[e];
      coo.dst[s] = gv[e];
      if (symmetrize) { coo.src[s + 1] = gv[e]; coo.dst[s + 1] = gu[e]; }
      if (wkind == MG_W_UNIFORM_INT) { int32_t w = wg.ival(e); coo.wi[s] = w; if (symmetrize) coo.wi[s + 1] = w; }
      if (wkind == MG_W_LOGNORMAL) { float w = wg.fval(e); coo.wf[s] = w; if (symmetrize) coo.wf[s + 1] = w; }
      k++;
    }
  }
  std::vector<int32_t>().swap(gu);
  std::vector<int32_t>().swap(gv);
  return coo_to_csr(n, coo, wkind, true, out);
}

mg_status mg_gen_lattice(int32_t rows, int32_t cols, double longrange_frac, uint64_t seed,
                         int32_t wkind, double p0, double p1, mg_host_csr *out) {
  if (!out || rows < 1 || cols < 1 || longrange_frac < 0 || !valid_weights(wkind, p0, p1)) {
    mg_set_error("mg_gen_lattice: invalid arguments");
    return MG_ERR_ARG;
  }
  const int64_t n = (int64_t)rows * cols;
  const int64_t und = (int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols;  // undirected lattice edges
  const int64_t nlong = (int64_t)std::llround(longrange_frac * 2.0 * (double)und);
  if (n > INT32_MAX - 1 || 2 * (und + nlong) > INT32_MAX || (nlong > 0 && n < 2)) {
    mg_set_error("mg_gen_lattice: size exceeds int32");
    return MG_ERR_ARG;
  }
  const int64_t mu = und + nlong;  // undirected edges, each emitted in both directions
  Coo coo;
  coo.src.resize(2 * mu);
  coo.dst.resize(2 * mu);
  if (wkind == MG_W_UNIFORM_INT) coo.wi.resize(2 * mu);
  if (wkind == MG_W_LOGNORMAL) coo.wf.resize(2 * mu);
  WeightGen wg{wkind, p0, p1, stream_key(seed, S_WEIGHT)};
  const int64_t horiz = (int64_t)rows * (cols - 1);
  const uint64_t kl = stream_key(seed, S_LONG), kr = stream_key(seed, S_REDRAW);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < mu; k++) {
    int64_t u, v;
    if (k < horiz) {
      int64_t r = k / (cols - 1), c = k % (cols - 1);
      u = r * cols + c;
      v = u + 1;
    } else if (k < und) {
      int64_t q = k - horiz;
      int64_t r = q / cols, c = q % cols;
      u = r * cols + c;
      v = u + cols;
    } else {
      int64_t j = k - und;
      u = (int64_t)(draw(kl, 2 * (uint64_t)j) % (uint64_t)n);
      v = (int64_t)(draw(kl, 2 * (uint64_t)j + 1) % (uint64_t)n);
      for (uint64_t t = 1; v == u; t++) v = (int64_t)(draw(kr, (uint64_t)j * 64 + t) % (uint64_t)n);
    }
    coo.src[2 * k] = (int32_t)u;
    coo.dst[2 * k] = (int32_t)v;
    coo.src[2 * k + 1] = (int32_t)v;
    coo.dst[2 * k + 1] = (int32_t)u;
    if (wkind == MG_W_UNIFORM_INT) { int32_t w = wg.ival(k); coo.wi[2 * k] = w; coo.wi[2 * k + 1] = w; }
    if (wkind == MG_W_LOGNORMAL) { float w = wg.fval(k); coo.wf[2 * k] = w; coo.wf[2 * k + 1] = w; }
  }
  return coo_to_csr(n, coo, wkind, true, out);
}

namespace {

// One Matrix Market entry line: "row col [value]" with sscanf("%lld %lld %lf")
// semantics (leading blanks skipped, a missing or unparsable value means 1.0).
// Returns the number of fields read (2 or 3), or fewer on a malformed line.
int parse_entry(const char *p, const char *eol, long long *r, long long *c, double *v) {
  char *q = nullptr;
  std::string tmp;  // strtoll/strtod stop at the first character they do not take
  *r = std::strtoll(p, &q, 10);
  if (q == p || q > eol) return 0;
  const char *p2 = q;
  *c = std::strtoll(p2, &q, 10);
  if (q == p2 || q > eol) return 1;
  const char *p3 = q;
  const double x = std::strtod(p3, &q);
  if (q == p3 || q > eol) return 2;
  *v = x;
  return 3;
}

bool blank_line(const char *p, const char *eol) {
  while (p < eol && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
  return p == eol;
}

}  // namespace

// Parallel reader: the header is parsed first; the body is cut into chunks at
// line boundaries, each thread counts its entry lines, and after a prefix sum
// every thread parses its lines into their file positions, so the result equals
// a line-by-line read (rows then keep file order, as the reference's stable sort).
mg_status mg_read_market(const char *path, int32_t undirected, mg_host_csr *out) {
  if (!path || !out) {
    mg_set_error("mg_read_market: null argument");
    return MG_ERR_ARG;
  }
  int fd = open(path, O_RDONLY);
  if (fd < 0) {
    mg_set_error("mg_read_market: cannot open %s: %s", path, std::strerror(errno));
    return MG_ERR_ARG;
  }
  struct stat st;
  if (fstat(fd, &st) != 0) {
    close(fd);
    mg_set_error("mg_read_market: cannot stat %s", path);
    return MG_ERR_ARG;
  }
  size_t len = (size_t)st.st_size;
  std::vector<char> buf(len + 1);
  size_t got = 0;
  while (got < len) {
    ssize_t r = read(fd, buf.data() + got, len - got);
    if (r <= 0) break;
    got += (size_t)r;
  }
  close(fd);
  buf[got] = '\0';
  const char *p = buf.data(), *end = buf.data() + got;
  // Problem line: the first line that is neither blank nor a '%' comment.
  int64_t n = -1, declared = 0;
  while (p < end) {
    const char *eol = (const char *)std::memchr(p, '\n', (size_t)(end - p));
    if (!eol) eol = end;
    if (blank_line(p, eol) || *p == '%') {
      p = eol + 1;
      continue;
    }
    long long rx, cy, ne;
    std::string line(p, eol);
    p = eol + 1;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &rx, &cy, &ne) != 3) {
      mg_set_error("mg_read_market: invalid problem description");
      return MG_ERR_ARG;
    }
    if (rx != cy) {
      mg_set_error("mg_read_market: not square (%lld, %lld)", rx, cy);
      return MG_ERR_ARG;
    }
    if (rx < 0 || rx > INT32_MAX - 1 || ne < 0 || ne * (undirected ? 2 : 1) > INT32_MAX) {
      mg_set_error("mg_read_market: sizes exceed int32");
      return MG_ERR_ARG;
    }
    n = rx;
    declared = ne;
    break;
  }
  if (n < 0) {
    mg_set_error("mg_read_market: no graph found");
    return MG_ERR_ARG;
  }
  const char *body = std::min(p, end);
  const size_t blen = (size_t)(end - body);
  const int nth = std::max(1, omp_get_max_threads());
  const int nchunk = (int)std::min<size_t>((size_t)nth * 8, std::max<size_t>(1, blen / 4096 + 1));
  std::vector<const char *> cb(nchunk + 1);
  cb[0] = body;
  for (int i = 1; i < nchunk; i++) {
    const char *c = body + blen * (size_t)i / (size_t)nchunk;
    c = std::max(c, cb[i - 1]);
    const char *nl = c < end ? (const char *)std::memchr(c, '\n', (size_t)(end - c)) : nullptr;
    cb[i] = nl ? nl + 1 : end;
  }
  cb[nchunk] = end;
  std::vector<int64_t> cnt(nchunk + 1, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < nchunk; i++) {
    int64_t k = 0;
    for (const char *q = cb[i]; q < cb[i + 1];) {
      const char *eol = (const char *)std::memchr(q, '\n', (size_t)(cb[i + 1] - q));
      if (!eol) eol = cb[i + 1];
      if (!blank_line(q, eol) && *q != '%') k++;
      q = eol + 1;
    }
    cnt[i + 1] = k;
  }
  for (int i = 0; i < nchunk; i++) cnt[i + 1] += cnt[i];
  const int64_t entries = cnt[nchunk];
  if (entries > declared) {
    mg_set_error("mg_read_market: more than %lld entries", (long long)declared);
    return MG_ERR_ARG;
  }
  if (entries < declared) {
    mg_set_error("mg_read_market: only %lld/%lld entries read", (long long)entries, (long long)declared);
    return MG_ERR_ARG;
  }
  const int64_t dup = undirected ? 2 : 1;
  Coo coo;
  coo.src.resize((size_t)(entries * dup));
  coo.dst.resize((size_t)(entries * dup));
  std::vector<double> vals((size_t)(entries * dup));
  std::atomic<int64_t> bad{INT64_MAX};
  std::atomic<int> bad_kind{0};
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < nchunk; i++) {
    int64_t k = cnt[i];
    for (const char *q = cb[i]; q < cb[i + 1];) {
      const char *eol = (const char *)std::memchr(q, '\n', (size_t)(cb[i + 1] - q));
      if (!eol) eol = cb[i + 1];
      if (blank_line(q, eol) || *q == '%') {
        q = eol + 1;
        continue;
      }
      long long r = 0, c = 0;
      double v = 1.0;
      const int nr = parse_entry(q, eol, &r, &c, &v);
      int kind = 0;
      if (nr != 2 && nr != 3) kind = 1;
      else if (r < 1 || r > n || c < 1 || c > n) kind = 2;
      if (kind) {
        int64_t prev = bad.load();
        while (k < prev && !bad.compare_exchange_weak(prev, k)) {
        }
        if (k <= bad.load()) bad_kind.store(kind);
      } else {
        const size_t at = (size_t)(k * dup);
        coo.src[at] = (int32_t)(r - 1);
        coo.dst[at] = (int32_t)(c - 1);
        vals[at] = v;
        if (undirected) {
          coo.src[at + 1] = (int32_t)(c - 1);
          coo.dst[at + 1] = (int32_t)(r - 1);
          vals[at + 1] = v;
        }
      }
      k++;
      q = eol + 1;
    }
  }
  if (bad.load() != INT64_MAX) {
    if (bad_kind.load() == 1) mg_set_error("mg_read_market: badly formed entry %lld", (long long)bad.load());
    else mg_set_error("mg_read_market: entry %lld out of range", (long long)bad.load());
    return MG_ERR_ARG;
  }
  const size_t mm = coo.src.size();
  coo.wi.resize(mm);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)mm; e++) coo.wi[e] = (int32_t)vals[e];
  mg_status st2 = coo_to_csr(n, coo, MG_W_UNIFORM_INT, false, out);
  if (st2 != MG_OK) return st2;
  // Float view of the same values (the PageRank program reads Value = float).
  out->weights_f32 = (float *)std::malloc(sizeof(float) * std::max<size_t>(mm, 1));
  if (!out->weights_f32) {
    mg_host_csr_free(out);
    return MG_ERR_OOM;
  }
  // Re-run the stable row placement for the float values.
  std::vector<int64_t> cur((size_t)n + 1);
  for (int64_t v = 0; v <= n; v++) cur[v] = out->row_offsets[v];
  for (size_t e = 0; e < mm; e++) out->weights_f32[cur[coo.src[e]]++] = (float)vals[e];
  return MG_OK;
}

mg_status mg_write_market(const char *path, const mg_host_csr *g, int32_t values) {
  if (!path || !g || g->n < 0 || g->m < 0 || !g->row_offsets || (g->m > 0 && !g->col_idx)) {
    mg_set_error("mg_write_market: invalid arguments");
    return MG_ERR_ARG;
  }
  const bool vi = values == 1 && g->weights_i32, vf = values == 2 && g->weights_f32;
  if (values != 0 && !vi && !vf) {
    mg_set_error("mg_write_market: the graph has no %s weights", values == 1 ? "int32" : "float");
    return MG_ERR_ARG;
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    mg_set_error("mg_write_market: cannot open %s: %s", path, std::strerror(errno));
    return MG_ERR_ARG;
  }
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate %s general\n%lld %lld %lld\n",
               vf ? "real" : (vi ? "integer" : "pattern"), (long long)g->n, (long long)g->n, (long long)g->m);
  // Rows are formatted in parallel blocks, then written in order.
  const int64_t n = g->n;
  const int64_t block = 1 << 16;
  const int64_t nblk = (n + block - 1) / block;
  bool ok = true;
  for (int64_t b0 = 0; b0 < nblk && ok; b0 += 64) {
    const int64_t b1 = std::min<int64_t>(nblk, b0 + 64);
    std::vector<std::string> text((size_t)(b1 - b0));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = b0; b < b1; b++) {
      std::string &t = text[(size_t)(b - b0)];
      char line[96];
      for (int64_t v = b * block; v < std::min(n, (b + 1) * block); v++) {
        for (int64_t k = g->row_offsets[v]; k < g->row_offsets[v + 1]; k++) {
          int len;
          if (vi) len = std::snprintf(line, sizeof(line), "%lld %d %d\n", (long long)v + 1, g->col_idx[k] + 1, g->weights_i32[k]);
          else if (vf) len = std::snprintf(line, sizeof(line), "%lld %d %.9g\n", (long long)v + 1, g->col_idx[k] + 1, (double)g->weights_f32[k]);
          else len = std::snprintf(line, sizeof(line), "%lld %d\n", (long long)v + 1, g->col_idx[k] + 1);
          t.append(line, (size_t)len);
        }
      }
    }
    for (const std::string &t : text)
      if (!t.empty() && std::fwrite(t.data(), 1, t.size(), f) != t.size()) ok = false;
  }
  if (std::fclose(f) != 0) ok = false;
  if (!ok) {
    mg_set_error("mg_write_market: write to %s failed", path);
    return MG_ERR_ARG;
  }
  return MG_OK;
}

// Binary CSR cache: "MGB200C1", int64 n, int64 m, int32 flags (1: int32
// weights, 2: float weights), int32 0, then row_offsets (n + 1), col_idx (m),
// weights_i32 (m, if flagged), weights_f32 (m, if flagged); native byte order.
static const char kCsrMagic[8] = {'M', 'G', 'B', '2', '0', '0', 'C', '1'};

mg_status mg_save_csr(const char *path, const mg_host_csr *g) {
  if (!path || !g || g->n < 0 || g->m < 0 || !g->row_offsets || (g->m > 0 && !g->col_idx)) {
    mg_set_error("mg_save_csr: invalid arguments");
    return MG_ERR_ARG;
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    mg_set_error("mg_save_csr: cannot open %s: %s", path, std::strerror(errno));
    return MG_ERR_ARG;
  }
  const int32_t flags = (g->weights_i32 ? 1 : 0) | (g->weights_f32 ? 2 : 0), zero = 0;
  const int64_t n = g->n, m = g->m;
  bool ok = std::fwrite(kCsrMagic, 1, 8, f) == 8 && std::fwrite(&n, 8, 1, f) == 1 && std::fwrite(&m, 8, 1, f) == 1 &&
            std::fwrite(&flags, 4, 1, f) == 1 && std::fwrite(&zero, 4, 1, f) == 1;
  ok = ok && std::fwrite(g->row_offsets, 4, (size_t)n + 1, f) == (size_t)n + 1;
  ok = ok && std::fwrite(g->col_idx, 4, (size_t)m, f) == (size_t)m;
  if (g->weights_i32) ok = ok && std::fwrite(g->weights_i32, 4, (size_t)m, f) == (size_t)m;
  if (g->weights_f32) ok = ok && std::fwrite(g->weights_f32, 4, (size_t)m, f) == (size_t)m;
  if (std::fclose(f) != 0) ok = false;
  if (!ok) {
    mg_set_error("mg_save_csr: write to %s failed", path);
    return MG_ERR_ARG;
  }
  return MG_OK;
}

mg_status mg_load_csr(const char *path, mg_host_csr *out) {
  if (!path || !out) {
    mg_set_error("mg_load_csr: null argument");
    return MG_ERR_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    mg_set_error("mg_load_csr: cannot open %s: %s", path, std::strerror(errno));
    return MG_ERR_ARG;
  }
  char magic[8];
  int64_t n = 0, m = 0;
  int32_t flags = 0, zero = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCsrMagic, 8) == 0 &&
            std::fread(&n, 8, 1, f) == 1 && std::fread(&m, 8, 1, f) == 1 && std::fread(&flags, 4, 1, f) == 1 &&
            std::fread(&zero, 4, 1, f) == 1 && n >= 0 && n <= INT32_MAX - 1 && m >= 0 && m <= INT32_MAX;
  if (!ok) {
    std::fclose(f);
    mg_set_error("mg_load_csr: %s is not a mapgraph_b200 CSR file", path);
    return MG_ERR_ARG;
  }
  out->n = n;
  out->m = m;
  out->row_offsets = (int32_t *)std::malloc(4 * ((size_t)n + 1));
  out->col_idx = (int32_t *)std::malloc(4 * std::max<size_t>((size_t)m, 1));
  if (flags & 1) out->weights_i32 = (int32_t *)std::malloc(4 * std::max<size_t>((size_t)m, 1));
  if (flags & 2) out->weights_f32 = (float *)std::malloc(4 * std::max<size_t>((size_t)m, 1));
  ok = out->row_offsets && out->col_idx && (!(flags & 1) || out->weights_i32) && (!(flags & 2) || out->weights_f32);
  ok = ok && std::fread(out->row_offsets, 4, (size_t)n + 1, f) == (size_t)n + 1;
  ok = ok && std::fread(out->col_idx, 4, (size_t)m, f) == (size_t)m;
  if (flags & 1) ok = ok && std::fread(out->weights_i32, 4, (size_t)m, f) == (size_t)m;
  if (flags & 2) ok = ok && std::fread(out->weights_f32, 4, (size_t)m, f) == (size_t)m;
  std::fclose(f);
  if (ok && (out->row_offsets[0] != 0 || out->row_offsets[n] != m)) ok = false;
  if (!ok) {
    mg_host_csr_free(out);
    mg_set_error("mg_load_csr: %s is truncated or inconsistent", path);
    return MG_ERR_ARG;
  }
  return MG_OK;
}

mg_status mg_host_csr_to_csc(int64_t n, int64_t m, const int32_t *row_offsets, const int32_t *col_idx,
                             int32_t *col_offsets, int32_t *row_idx, int32_t *perm) {
  if (n < 0 || m < 0 || !row_offsets || !col_offsets || (m > 0 && (!col_idx || !row_idx || !perm))) {
    mg_set_error("mg_host_csr_to_csc: invalid arguments");
    return MG_ERR_ARG;
  }
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  for (int64_t e = 0; e < m; e++) cnt[col_idx[e]]++;
  int64_t run = 0;
  for (int64_t v = 0; v < n; v++) {
    int64_t c = cnt[v];
    col_offsets[v] = (int32_t)run;
    cnt[v] = run;
    run += c;
  }
  col_offsets[n] = (int32_t)run;
  for (int64_t v = 0; v < n; v++) {
    for (int64_t e = row_offsets[v]; e < row_offsets[v + 1]; e++) {
      int64_t s = cnt[col_idx[e]]++;
      row_idx[s] = (int32_t)v;
      perm[s] = (int32_t)e;
    }
  }
  return MG_OK;
}

}  // extern "C"
