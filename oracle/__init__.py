"""CPU oracle of the GAS hot path -- TEST INFRASTRUCTURE ONLY (the checker).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
package, and only to check or time the CUDA engine; the engine never calls it.

Two layers:

* ``libmgoracle.so`` (mg_oracle.c): a plain-C restatement of the reference's
  algorithms -- BFS, Dijkstra SSSP, min-label CC, the reference-compatible
  PageRank schedule in FP64, and the FP64 normalised/personalised PageRank and
  its adjoint. Each routine cites the reference lines it restates.
* ``_ref/libmgref.so`` (build_ref.sh + ref_wrap.cpp): the reference's own CPU
  correctness functions CPUBFS / CPUSSSP / CPUCC / CPUPR and its Matrix Market
  ingest, compiled from the reference tree when it is present. It pins the
  restatement; tests/golden/ holds vectors recorded from it so the pin also holds
  where the reference tree is absent.
* ``_ref/gas_ref_tuned`` and ``_ref/gas_ref_generic``: the reference's own bundled
  vertex programs (Algorithms/*/*.h, unchanged) compiled against this
  repository's compat GASengine headers, to check that they run on the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libmgoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmgref.so")
# The reference checkout: MG_REFERENCE_DIR, else a "reference" directory beside
# this repository's checkout.
REFERENCE_DIR = os.environ.get("MG_REFERENCE_DIR",
                               os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
INT_MAX = 2**31 - 1
REF_SSSP_UNREACHED = 100000000  # Algorithms/SSSP/sssp.cu:139

_I = C.POINTER(C.c_int32)
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)


def build(force: bool = False) -> None:
    """Compiles the restatement, and the reference's CPU path when the tree is present."""
    src = os.path.join(HERE, "mg_oracle.c")
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", LIB, src, "-lm"], check=True)
    if os.path.isdir(REFERENCE_DIR):
        root = os.path.dirname(HERE)
        deps = [os.path.join(HERE, "ref_wrap.cpp"), os.path.join(HERE, "build_ref.sh"),
                os.path.join(root, "tests", "cpp", "gas_ref_programs.cu"),
                os.path.join(root, "include", "compat", "GASengine", "csr_problem.cuh"),
                os.path.join(root, "include", "compat", "GASengine", "enactor_vertex_centric.cuh")]
        outs = [REF_LIB] + [os.path.join(HERE, "_ref", f"gas_ref_{m}") for m in ("tuned", "generic")]
        newest = max(map(os.path.getmtime, [d for d in deps if os.path.exists(d)]))
        if force or any(not os.path.exists(o) or os.path.getmtime(o) < newest for o in outs):
            subprocess.run(["sh", os.path.join(HERE, "build_ref.sh")], check=True, capture_output=True)


_lib = None
_ref = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.mgo_bfs.argtypes = [C.c_int, _I, _I, _I, _I, C.c_int, C.c_int, _I, _I]
        lib.mgo_sssp.argtypes = [C.c_int, _I, _I, _I, _I, _I, _I, C.c_int, C.c_int, _I, _I]
        lib.mgo_cc.argtypes = [C.c_int, _I, _I, _I]
        lib.mgo_pr_refcompat.argtypes = [C.c_int, _I, _I, _I, _I, C.c_int, C.c_int, C.c_double, _D]
        lib.mgo_pr_refcompat.restype = C.c_int
        lib.mgo_pr_normalized.argtypes = [C.c_int, _I, _I, _F, C.c_double, C.c_double, C.c_int, _D, _D, _D]
        lib.mgo_pr_normalized.restype = C.c_int
        lib.mgo_pr_loss.argtypes = [C.c_int, _I, _I, _F, C.c_double, C.c_double, C.c_int, _D, _D, _D]
        lib.mgo_pr_loss.restype = C.c_double
        lib.mgo_pr_adjoint.argtypes = [C.c_int, _I, _I, _F, C.c_double, _D, _D, _D, C.c_double, C.c_int, _D, _D,
                                       _D]
        lib.mgo_pr_adjoint.restype = C.c_int
        _lib = lib
    return _lib


def have_ref() -> bool:
    if os.path.exists(REF_LIB):
        return True
    if os.path.isdir(REFERENCE_DIR):
        try:
            build()
        except Exception:
            return False
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _ref
    if _ref is None:
        if not have_ref():
            raise RuntimeError("reference CPU oracle (oracle/_ref/libmgref.so) unavailable")
        lib = C.CDLL(REF_LIB)
        lib.mgref_bfs.argtypes = [C.c_int, C.c_int, _I, _I, _I, _I, C.c_int, C.c_int, _I]
        lib.mgref_bfs.restype = C.c_double
        lib.mgref_sssp.argtypes = [C.c_int, C.c_int, _I, _I, _I, _I, _I, C.c_int, C.c_int, _I]
        lib.mgref_sssp.restype = C.c_double
        lib.mgref_cc.argtypes = [C.c_int, C.c_int, _I, _I, _I, _I, _I]
        lib.mgref_cc.restype = C.c_double
        lib.mgref_pr.argtypes = [C.c_int, C.c_int, _I, _I, _I, _I, _F, _I]
        lib.mgref_pr.restype = C.c_double
        lib.mgref_load_market.argtypes = [C.c_char_p, _I, _I]
        lib.mgref_load_market.restype = C.c_void_p
        lib.mgref_graph_get.argtypes = [C.c_void_p, _I, _I, _I, _I, _I]
        lib.mgref_graph_free.argtypes = [C.c_void_p]
        _ref = lib
    return _ref


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_I)


def _keep_i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_I)


def csc_of(ro, ci):
    """Stable transpose (col_offsets, row_idx, perm): within a column, CSR edge order."""
    ro = np.asarray(ro, dtype=np.int64)
    ci = np.asarray(ci, dtype=np.int64)
    n = ro.size - 1
    perm = np.argsort(ci, kind="stable").astype(np.int32)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(ro))
    co = np.zeros(n + 1, dtype=np.int64)
    np.add.at(co, ci + 1, 1)
    co = np.cumsum(co).astype(np.int32)
    return co, rows[perm].astype(np.int32), perm


# ---------------------------------------------------------------------------
# Restatement (libmgoracle.so)
def bfs(ro, ci, srcs, directed=1, csc=None):
    lib = _load()
    n = len(ro) - 1
    co, ri, _ = csc if csc is not None else (csc_of(ro, ci) if not directed else (ro, ci, None))
    out = np.empty(n, dtype=np.int32)
    ro_, p_ro = _keep_i(ro)
    ci_, p_ci = _keep_i(ci)
    co_, p_co = _keep_i(co)
    ri_, p_ri = _keep_i(ri)
    s_, p_s = _keep_i(np.atleast_1d(srcs))
    lib.mgo_bfs(n, p_ro, p_ci, p_co, p_ri, int(directed), s_.size, p_s, out.ctypes.data_as(_I))
    return out


def sssp(ro, ci, w, srcs, directed=1, csc=None):
    lib = _load()
    n = len(ro) - 1
    w = np.ones(len(ci), dtype=np.int32) if w is None else np.asarray(w, dtype=np.int32)
    if directed:
        co, ri, cw = ro, ci, w
    else:
        co, ri, perm = csc if csc is not None else csc_of(ro, ci)
        cw = w[perm]
    out = np.empty(n, dtype=np.int32)
    keep = [_keep_i(x) for x in (ro, ci, w, co, ri, cw, np.atleast_1d(srcs))]
    p = [k[1] for k in keep]
    lib.mgo_sssp(n, p[0], p[1], p[2], p[3], p[4], p[5], int(directed), keep[6][0].size, p[6],
                 out.ctypes.data_as(_I))
    return out


def cc(ro, ci):
    lib = _load()
    n = len(ro) - 1
    out = np.empty(n, dtype=np.int32)
    ro_, p_ro = _keep_i(ro)
    ci_, p_ci = _keep_i(ci)
    lib.mgo_cc(n, p_ro, p_ci, out.ctypes.data_as(_I))
    return out


def pr_refcompat(ro, ci, directed=1, iter_num=2**31 - 1, delta=0.01, csc=None):
    """FP64 replay of the reference engine's PageRank schedule; returns (x, iterations)."""
    lib = _load()
    n = len(ro) - 1
    co, ri, _ = csc if csc is not None else csc_of(ro, ci)
    x = np.empty(n, dtype=np.float64)
    keep = [_keep_i(a) for a in (ro, ci, co, ri)]
    it = lib.mgo_pr_refcompat(n, keep[0][1], keep[1][1], keep[2][1], keep[3][1], int(directed), int(iter_num),
                              float(delta), x.ctypes.data_as(_D))
    return x, it


def _fptr(a):
    if a is None:
        return None, None
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_F)


def _dptr(a):
    if a is None:
        return None, None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_D)


def pr_normalized(ro, ci, weights=None, alpha=0.85, tol=1e-6, max_iter=50, teleport=None):
    """FP64 normalised PageRank; returns (x, iterations, last L1 change)."""
    lib = _load()
    n = len(ro) - 1
    x = np.empty(n, dtype=np.float64)
    r = C.c_double()
    ro_, p_ro = _keep_i(ro)
    ci_, p_ci = _keep_i(ci)
    w_, p_w = _fptr(weights)
    t_, p_t = _dptr(teleport)
    it = lib.mgo_pr_normalized(n, p_ro, p_ci, p_w, alpha, tol, int(max_iter), p_t, x.ctypes.data_as(_D),
                               C.byref(r))
    return x, it, r.value


def pr_loss(ro, ci, weights, w, x0, alpha=0.85, tol=1e-14, max_iter=10000, teleport=None):
    """L = sum w_i x_i at the FP64 fixed point, power iteration warm-started from x0."""
    lib = _load()
    n = len(ro) - 1
    x = np.array(x0, dtype=np.float64, copy=True)
    ro_, p_ro = _keep_i(ro)
    ci_, p_ci = _keep_i(ci)
    a_, p_a = _fptr(weights)
    t_, p_t = _dptr(teleport)
    w_, p_wv = _dptr(w)
    return lib.mgo_pr_loss(n, p_ro, p_ci, p_a, alpha, tol, int(max_iter), p_t, p_wv, x.ctypes.data_as(_D))


def pr_adjoint(ro, ci, weights, x, w, alpha=0.85, tol=1e-14, max_iter=10000, teleport=None):
    """FP64 adjoint; returns (grad_weights[m], grad_teleport[n], lambda[n], iterations)."""
    lib = _load()
    n = len(ro) - 1
    m = len(ci)
    lam = np.empty(n, dtype=np.float64)
    ga = np.zeros(max(m, 1), dtype=np.float64)
    gt = np.empty(n, dtype=np.float64)
    ro_, p_ro = _keep_i(ro)
    ci_, p_ci = _keep_i(ci)
    a_, p_a = _fptr(weights)
    t_, p_t = _dptr(teleport)
    x_, p_x = _dptr(x)
    w_, p_wv = _dptr(w)
    it = lib.mgo_pr_adjoint(n, p_ro, p_ci, p_a, alpha, p_t, p_x, p_wv, tol, int(max_iter), lam.ctypes.data_as(_D),
                            ga.ctypes.data_as(_D), gt.ctypes.data_as(_D))
    return ga[:m], gt, lam, it


# ---------------------------------------------------------------------------
# The reference's own CPU functions (oracle/_ref/libmgref.so)
class Ref:
    """CPUBFS / CPUSSSP / CPUCC / CPUPR and the reference's .mtx ingest.

    Each call returns (result, seconds) where seconds is the wall time of the
    reference function alone (std::chrono around the call)."""

    @staticmethod
    def _csc(ro, ci, csc):
        return csc if csc is not None else csc_of(ro, ci)

    @staticmethod
    def bfs(ro, ci, src, directed=1, csc=None):
        lib = _ref_lib()
        n, m = len(ro) - 1, len(ci)
        co, ri, _ = Ref._csc(ro, ci, csc)
        out = np.empty(n, dtype=np.int32)
        keep = [_keep_i(a) for a in (ro, ci, co, ri)]
        t = lib.mgref_bfs(n, m, keep[0][1], keep[1][1], keep[2][1], keep[3][1], int(directed), int(src),
                          out.ctypes.data_as(_I))
        return out, t

    @staticmethod
    def sssp(ro, ci, w, src, directed=1, csc=None):
        lib = _ref_lib()
        n, m = len(ro) - 1, len(ci)
        co, ri, _ = Ref._csc(ro, ci, csc)
        out = np.empty(n, dtype=np.int32)
        keep = [_keep_i(a) for a in (ro, ci, co, ri, w)]
        t = lib.mgref_sssp(n, m, keep[0][1], keep[1][1], keep[2][1], keep[3][1], keep[4][1], int(directed),
                           int(src), out.ctypes.data_as(_I))
        return out, t

    @staticmethod
    def cc(ro, ci, csc=None):
        lib = _ref_lib()
        n, m = len(ro) - 1, len(ci)
        co, ri, _ = Ref._csc(ro, ci, csc)
        out = np.empty(n, dtype=np.int32)
        keep = [_keep_i(a) for a in (ro, ci, co, ri)]
        t = lib.mgref_cc(n, m, keep[0][1], keep[1][1], keep[2][1], keep[3][1], out.ctypes.data_as(_I))
        return out, t

    @staticmethod
    def pr(ro, ci, csc=None, with_sweeps=False):
        lib = _ref_lib()
        n, m = len(ro) - 1, len(ci)
        co, ri, _ = Ref._csc(ro, ci, csc)
        out = np.empty(n, dtype=np.float32)
        sweeps = C.c_int32(-1)
        keep = [_keep_i(a) for a in (ro, ci, co, ri)]
        t = lib.mgref_pr(n, m, keep[0][1], keep[1][1], keep[2][1], keep[3][1], out.ctypes.data_as(_F),
                         C.byref(sweeps))
        return (out, t, sweeps.value) if with_sweeps else (out, t)

    @staticmethod
    def load_market(path):
        """(row_offsets, col_idx, values_int, col_offsets, row_idx) as the reference ingests the file."""
        lib = _ref_lib()
        n, m = C.c_int32(), C.c_int32()
        h = lib.mgref_load_market(path.encode(), C.byref(n), C.byref(m))
        if not h:
            raise RuntimeError(f"reference failed to load {path}")
        try:
            ro = np.empty(n.value + 1, dtype=np.int32)
            ci = np.empty(m.value, dtype=np.int32)
            vals = np.empty(m.value, dtype=np.int32)
            co = np.empty(n.value + 1, dtype=np.int32)
            ri = np.empty(m.value, dtype=np.int32)
            lib.mgref_graph_get(h, ro.ctypes.data_as(_I), ci.ctypes.data_as(_I), vals.ctypes.data_as(_I),
                                co.ctypes.data_as(_I), ri.ctypes.data_as(_I))
        finally:
            lib.mgref_graph_free(h)
        return ro, ci, vals, co, ri


def bfs_pred(ro, ci, depth, csc=None):
    """BFS predecessors as the reference's pred_extract computes them
    (Algorithms/BFS/predextract.cuh:246-373): over every in-edge (u, v) the
    candidate is u when depth[v] - depth[u] == 1, else -1 (gather_edge, :143-155),
    reduced by max (ReduceFunctor, :211-219); -1 for vertices without in-edges."""
    co, ri, _ = csc if csc is not None else csc_of(ro, ci)
    n = len(ro) - 1
    depth = np.asarray(depth, dtype=np.int64)
    ri = np.asarray(ri, dtype=np.int64)
    dst = np.repeat(np.arange(n), np.diff(np.asarray(co, dtype=np.int64)))
    cand = np.where(depth[dst] - depth[ri] == 1, ri, -1)
    pred = np.full(n, -1, dtype=np.int64)
    np.maximum.at(pred, dst, cand)
    return pred.astype(np.int32)
