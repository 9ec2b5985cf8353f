"""Seeded synthetic graphs and Matrix Market ingest (host side, C++/OpenMP in the library).

All generators are counter-based (splitmix64 of seed, stream and index): the same
arguments give the same CSR on every machine and thread count. See
include/mapgraph_b200_io.h for the exact definitions.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class HostCsr:
    """A host CSR: int32 row offsets (n+1) and column indices (m), optional weights."""
    row_offsets: np.ndarray
    col_idx: np.ndarray
    weights_i32: np.ndarray | None = None
    weights_f32: np.ndarray | None = None

    @property
    def n(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def m(self) -> int:
        return int(self.col_idx.shape[0])

    def out_degree(self) -> np.ndarray:
        return np.diff(self.row_offsets).astype(np.int64)


def _check(st: int, what: str) -> None:
    if st != L.MG_OK:
        lib = L.load()
        raise RuntimeError(f"{what}: {lib.mg_status_string(st).decode()} ({lib.mg_last_error().decode()})")


def _take(h: L.MgHostCsr) -> HostCsr:
    lib = L.load()
    n, m = int(h.n), int(h.m)

    def arr(ptr, count, dt):
        if not ptr or count == 0:
            return np.zeros(count, dtype=dt) if ptr else None
        return np.ctypeslib.as_array(ptr, shape=(count,)).copy()

    try:
        ro = arr(h.row_offsets, n + 1, np.int32)
        ci = arr(h.col_idx, m, np.int32)
        if ci is None:
            ci = np.zeros(0, dtype=np.int32)
        wi = arr(h.weights_i32, m, np.int32)
        wf = arr(h.weights_f32, m, np.float32)
    finally:
        lib.mg_host_csr_free(C.byref(h))
    return HostCsr(ro, ci, wi, wf)


def _wkind(weights: str | None) -> int:
    return {None: L.MG_W_NONE, "none": L.MG_W_NONE, "int": L.MG_W_UNIFORM_INT,
            "lognormal": L.MG_W_LOGNORMAL}[weights]


def gen_er(n: int, m: int, seed: int, weights: str | None = None, p0: float = 1, p1: float = 64) -> HostCsr:
    """Directed Erdos-Renyi multigraph with exactly m edges, self-loops redrawn, duplicates kept."""
    lib = L.load()
    h = L.MgHostCsr()
    _check(lib.mg_gen_er(n, m, seed & (2**64 - 1), _wkind(weights), p0, p1, C.byref(h)), "mg_gen_er")
    return _take(h)


def gen_rmat(scale: int, edge_factor: int, seed: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             symmetrize: bool = True, weights: str | None = None, p0: float = 1, p1: float = 255) -> HostCsr:
    """R-MAT graph (no noise, no id permutation); self-loops dropped, duplicates kept."""
    lib = L.load()
    h = L.MgHostCsr()
    _check(lib.mg_gen_rmat(scale, edge_factor, a, b, c, seed & (2**64 - 1), int(symmetrize), _wkind(weights),
                           p0, p1, C.byref(h)), "mg_gen_rmat")
    return _take(h)


def gen_lattice(rows: int, cols: int, longrange_frac: float, seed: int, weights: str | None = None,
                p0: float = 1, p1: float = 1000) -> HostCsr:
    """2-D 4-neighbour lattice plus uniform long-range pairs, every edge in both directions."""
    lib = L.load()
    h = L.MgHostCsr()
    _check(lib.mg_gen_lattice(rows, cols, longrange_frac, seed & (2**64 - 1), _wkind(weights), p0, p1,
                              C.byref(h)), "mg_gen_lattice")
    return _take(h)


def read_market(path: str, undirected: bool = False) -> HostCsr:
    """Matrix Market file -> CSR with the reference reader's semantics (1-based, rows in file order)."""
    lib = L.load()
    h = L.MgHostCsr()
    _check(lib.mg_read_market(path.encode(), int(undirected), C.byref(h)), "mg_read_market")
    return _take(h)


def _view(g: HostCsr):
    """An MgHostCsr over the arrays of g (kept alive by the returned tuple)."""
    keep = [np.ascontiguousarray(g.row_offsets, dtype=np.int32), np.ascontiguousarray(g.col_idx, dtype=np.int32)]
    h = L.MgHostCsr()
    h.n, h.m = g.n, g.m
    h.row_offsets = keep[0].ctypes.data_as(C.POINTER(C.c_int32))
    h.col_idx = keep[1].ctypes.data_as(C.POINTER(C.c_int32))
    if g.weights_i32 is not None:
        keep.append(np.ascontiguousarray(g.weights_i32, dtype=np.int32))
        h.weights_i32 = keep[-1].ctypes.data_as(C.POINTER(C.c_int32))
    if g.weights_f32 is not None:
        keep.append(np.ascontiguousarray(g.weights_f32, dtype=np.float32))
        h.weights_f32 = keep[-1].ctypes.data_as(C.POINTER(C.c_float))
    return h, keep


def write_market(path: str, g: HostCsr, values: str | None = None) -> None:
    """Writes g as a Matrix Market file (values None, "int" or "float")."""
    h, keep = _view(g)
    kind = {None: 0, "int": 1, "float": 2}[values]
    _check(L.load().mg_write_market(path.encode(), C.byref(h), kind), "mg_write_market")


def save_csr(path: str, g: HostCsr) -> None:
    """Binary CSR cache of g (mg_save_csr)."""
    h, keep = _view(g)
    _check(L.load().mg_save_csr(path.encode(), C.byref(h)), "mg_save_csr")


def load_csr(path: str) -> HostCsr:
    """Reads a binary CSR cache written by save_csr (mg_load_csr)."""
    h = L.MgHostCsr()
    _check(L.load().mg_load_csr(path.encode(), C.byref(h)), "mg_load_csr")
    return _take(h)


def csr_to_csc(g: HostCsr):
    """Stable host transpose: (col_offsets, row_idx, perm) with perm[k] the CSR edge of CSC slot k."""
    lib = L.load()
    co = np.empty(g.n + 1, dtype=np.int32)
    ri = np.empty(max(g.m, 1), dtype=np.int32)
    perm = np.empty(max(g.m, 1), dtype=np.int32)
    ro = np.ascontiguousarray(g.row_offsets, dtype=np.int32)
    ci = np.ascontiguousarray(g.col_idx, dtype=np.int32)
    _check(lib.mg_host_csr_to_csc(g.n, g.m, ro.ctypes.data, ci.ctypes.data, co.ctypes.data, ri.ctypes.data,
                                  perm.ctypes.data), "mg_host_csr_to_csc")
    return co, ri[:g.m], perm[:g.m]


def mixed_degree_sources(row_offsets, k: int, seed: int) -> np.ndarray:
    """k seeded sources: half drawn from the top-1% out-degree vertices, half from
    the vertices of median (non-zero) out-degree -- the batched workload's mix."""
    deg = np.diff(np.asarray(row_offsets, dtype=np.int64))
    rng = np.random.default_rng(seed)
    order = np.argsort(-deg, kind="stable")
    top = order[: max(1, len(order) // 100)]
    med = np.flatnonzero(deg == np.median(deg[deg > 0]))
    if med.size == 0:
        med = np.flatnonzero(deg > 0)
    return np.concatenate([rng.choice(top, k // 2), rng.choice(med, k - k // 2)]).astype(np.int32)


def sparse_teleports(n: int, nvec: int, seed: int) -> np.ndarray:
    """nvec personalised teleport vectors (nvec x n float32): each has a seeded
    support of U{1..32} vertices with uniform mass on it."""
    rng = np.random.default_rng(seed)
    tele = np.zeros((nvec, n), dtype=np.float32)
    for k in range(nvec):
        sup = rng.choice(n, size=rng.integers(1, 33), replace=False)
        tele[k, sup] = 1.0 / sup.size
    return tele
