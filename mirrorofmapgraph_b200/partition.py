"""BFS and PageRank over a 1-D vertex partition: one GraphSlice per rank, one
all-gather per level / iteration.

The reference lays out per-GPU vertex ranges (``GraphSlice`` per GPU,
GASengine/csr_problem.cuh:339-365) but its enactor only ever runs GPU 0
(GASengine/enactor_vertex_centric.cuh:2398-2966). Here the ranges are real:
rank r holds the out-edges and in-edges of its vertices [lo, hi) (global ids)
and the global out-degrees; the visited bitmap, the frontier bitmap and the
depths of all n vertices are replicated. Every level each rank marks its
discoveries in an n-bit bitmap (push from its frontier vertices, or pull into
its unvisited vertices), the ranks all-gather those bitmaps, and every rank folds
the same world x words array into the same next frontier, so levels, directions
(Beamer's rule) and depths agree everywhere without a second exchange. Depths
equal the single-GPU BFS's. PageRank (normalised, uniform teleport) keeps the
whole iterate on every rank: a step computes the rank's own rows with the
degree-binned gather over its in-edges, the slices are all-gathered, and the
merge forms the next gather vector, the L1 change and the dangling mass with
fixed-order sums, so every rank stops at the same iteration.

Exchanges: :class:`CollectiveExchange` all-gathers over a torch.distributed
group (NCCL on the slice's own CUDA stream, one GPU per rank; gloo for host
tensors); :func:`bfs_partitioned_local` runs several slices on one GPU with a
shared buffer in place of the collective.
"""
from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np

from . import _lib as L
from .graph import _check, _is_torch, _ptr


def partition_cuts(row_offsets, world: int, align: int = 32) -> np.ndarray:
    """Cut points c[0] = 0 <= ... <= c[world] = n: rank r owns [c[r], c[r+1]).

    Cuts balance vertices + out-edges per rank and fall on multiples of `align`
    (32: each rank then owns whole words of the exchanged bitmaps)."""
    ro = np.asarray(row_offsets, dtype=np.int64)
    n = ro.size - 1
    if world <= 0:
        raise ValueError("world must be positive")
    work = ro + np.arange(n + 1, dtype=np.int64)
    targets = work[-1] * np.arange(1, world, dtype=np.float64) / world
    cuts = np.searchsorted(work, targets, side="left").astype(np.int64)
    cuts = (cuts // align) * align
    cuts = np.minimum(np.maximum.accumulate(np.clip(cuts, 0, n)), n)
    return np.concatenate([[0], cuts, [n]]).astype(np.int64)


def slice_rows(row_offsets, col_idx, lo: int, hi: int, symmetric: bool = False):
    """Out-edges and in-edges of vertices [lo, hi) as local CSR rows with global
    ids: (out_offsets, out_idx, in_offsets, in_idx); the in-edges are None for a
    symmetric graph. In-edges of a vertex keep CSR order (stable by source)."""
    ro = np.asarray(row_offsets, dtype=np.int64)
    ci = np.asarray(col_idx, dtype=np.int32)
    n = ro.size - 1
    out_off = (ro[lo:hi + 1] - ro[lo]).astype(np.int32)
    out_idx = np.ascontiguousarray(ci[ro[lo]:ro[hi]])
    if symmetric:
        return out_off, out_idx, None, None
    mask = (ci >= lo) & (ci < hi)
    src = np.repeat(np.arange(n, dtype=np.int32), np.diff(ro))[mask]
    tgt = ci[mask].astype(np.int64) - lo
    order = np.argsort(tgt, kind="stable")
    in_idx = np.ascontiguousarray(src[order])
    counts = np.bincount(tgt, minlength=hi - lo)
    in_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return out_off, out_idx, in_off, in_idx


def _level(lv: "L.MgPartLevel") -> dict:
    return {"frontier": lv.frontier, "frontier_edges": lv.frontier_edges, "level": lv.level,
            "done": bool(lv.done), "direction": "pull" if lv.direction == L.MG_DIR_PULL else "push"}


def _pr_level(lv: "L.MgPartLevel") -> dict:
    return {"level": lv.level, "done": bool(lv.done), "residual": lv.residual}


class GraphSlice:
    """One rank's share of a 1-D partition (an ``mg_part`` on the current CUDA
    device): rows [lo, hi) of the graph, both directions, global vertex ids."""

    def __init__(self, n: int, lo: int, hi: int, out_offsets, out_idx, in_offsets=None, in_idx=None,
                 out_degree=None, symmetric: bool = False):
        self._lib = L.load()
        self.n, self.lo, self.hi = int(n), int(lo), int(hi)
        self.symmetric = bool(symmetric)
        keep = []
        ptrs = []
        dev = None
        for a in (out_offsets, out_idx, in_offsets, in_idx, out_degree):
            p, d, k = _ptr(a, np.int32) if a is not None else (None, None, None)
            if a is not None and _is_torch(a) and a.dtype.itemsize != 4:
                raise ValueError("slice arrays must be int32")
            if p is not None:
                dev = d if dev is None else dev
                if d != dev:
                    raise ValueError("slice arrays must all be host or all be device")
            keep.append(k)
            ptrs.append(p)
        flags = (L.MG_GRAPH_SYMMETRIC if symmetric else 0) | (L.MG_GRAPH_DEVICE_INPUT if dev else 0)
        h = C.c_void_p()
        _check(self._lib.mg_part_create(self.n, self.lo, self.hi, *ptrs, flags, C.byref(h)), "mg_part_create")
        self._h = h
        w = C.c_int64()
        _check(self._lib.mg_part_words(h, C.byref(w)), "mg_part_words")
        self.words = int(w.value)
        s = C.c_void_p()
        _check(self._lib.mg_part_stream(h, C.byref(s)), "mg_part_stream")
        self._stream_ptr = s.value or 0
        self._torch_stream = None

    @classmethod
    def from_csr(cls, row_offsets, col_idx, lo: int, hi: int, symmetric: bool = False, out_degree=None):
        """Slice [lo, hi) of a host CSR (the whole graph is read on the host)."""
        ro = np.asarray(row_offsets)
        oo, oi, io, ii = slice_rows(ro, col_idx, lo, hi, symmetric)
        deg = np.diff(ro.astype(np.int64)).astype(np.int32) if out_degree is None else out_degree
        return cls(ro.size - 1, lo, hi, oo, oi, io, ii, deg, symmetric)

    # -- streams ------------------------------------------------------------------
    def stream_context(self):
        """Context that makes the slice's CUDA stream torch's current stream (for
        the collective that follows a step on that stream)."""
        import torch

        if self._torch_stream is None:
            self._torch_stream = torch.cuda.ExternalStream(self._stream_ptr)
        return torch.cuda.stream(self._torch_stream)

    def synchronize(self) -> None:
        import torch

        with self.stream_context():
            torch.cuda.current_stream().synchronize()

    # -- the level protocol --------------------------------------------------------
    def begin(self, srcs, direction: str = "auto", iter_num: int = 0) -> dict:
        s = np.ascontiguousarray(np.atleast_1d(np.asarray(srcs)), dtype=np.int32)
        o = L.MgOpts()
        o.directed = 1
        o.iter_num = int(iter_num)
        o.direction = {"auto": L.MG_DIR_AUTO, "push": L.MG_DIR_PUSH, "pull": L.MG_DIR_PULL}[direction]
        lv = L.MgPartLevel()
        _check(self._lib.mg_part_bfs_begin(self._h, s.ctypes.data, int(s.size), C.byref(o), C.byref(lv)),
               "mg_part_bfs_begin")
        return _level(lv)

    def step(self, bits) -> None:
        """This rank's discoveries of the pending level into `bits` (int32 CUDA
        tensor of `words` entries), on the slice's stream."""
        if not (_is_torch(bits) and bits.is_cuda and bits.numel() == self.words and bits.is_contiguous()):
            raise ValueError(f"bits must be a contiguous CUDA tensor of {self.words} words")
        _check(self._lib.mg_part_bfs_step(self._h, C.c_void_p(bits.data_ptr())), "mg_part_bfs_step")

    def merge(self, gathered, world: int) -> dict:
        if not (_is_torch(gathered) and gathered.is_cuda and gathered.numel() == world * self.words):
            raise ValueError(f"gathered must be a CUDA tensor of {world} x {self.words} words")
        lv = L.MgPartLevel()
        _check(self._lib.mg_part_bfs_merge(self._h, C.c_void_p(gathered.data_ptr()), int(world), C.byref(lv)),
               "mg_part_bfs_merge")
        return _level(lv)

    def result(self, out=None):
        """(depth of all n vertices, stats) of the last run."""
        if out is None:
            res = np.empty(self.n, dtype=np.int32)
            ptr, dev = res.ctypes.data, False
        else:
            res = out
            ptr, dev = (out.data_ptr(), bool(out.is_cuda)) if _is_torch(out) else (out.ctypes.data, False)
        st = L.MgStats()
        _check(self._lib.mg_part_bfs_result(self._h, C.c_void_p(ptr), int(dev), C.byref(st)), "mg_part_bfs_result")
        return res, st.as_dict()

    # -- PageRank (normalised, uniform teleport, unweighted) -------------------------
    def pr_begin(self, alpha: float = 0.85, tol: float = 1e-6, max_iter: int = 50) -> dict:
        o = L.MgPrOpts()
        o.mode = L.MG_PR_NORMALIZED
        o.alpha, o.tol, o.max_iter = float(alpha), float(tol), int(max_iter)
        lv = L.MgPartLevel()
        _check(self._lib.mg_part_pr_begin(self._h, C.byref(o), C.byref(lv)), "mg_part_pr_begin")
        return _pr_level(lv)

    def pr_step(self, slice_) -> None:
        """This rank's new ranks of [lo, hi) into the first hi - lo entries of
        `slice_` (float32 CUDA tensor), on the slice's stream."""
        if not (_is_torch(slice_) and slice_.is_cuda and slice_.numel() >= self.hi - self.lo):
            raise ValueError(f"slice must be a CUDA tensor of at least {self.hi - self.lo} floats")
        _check(self._lib.mg_part_pr_step(self._h, C.c_void_p(slice_.data_ptr())), "mg_part_pr_step")

    def pr_merge(self, gathered, world: int, stride: int, cuts) -> dict:
        if not (_is_torch(gathered) and gathered.is_cuda and gathered.numel() >= world * stride):
            raise ValueError(f"gathered must be a CUDA tensor of {world} x {stride} floats")
        c = np.ascontiguousarray(cuts, dtype=np.int64)
        lv = L.MgPartLevel()
        _check(self._lib.mg_part_pr_merge(self._h, C.c_void_p(gathered.data_ptr()), int(world), int(stride),
                                          c.ctypes.data, C.byref(lv)), "mg_part_pr_merge")
        return _pr_level(lv)

    def pr_result(self, out=None):
        """(ranks of all n vertices, stats) of the last PageRank run."""
        if out is None:
            res = np.empty(self.n, dtype=np.float32)
            ptr, dev = res.ctypes.data, False
        else:
            res = out
            ptr, dev = (out.data_ptr(), bool(out.is_cuda)) if _is_torch(out) else (out.ctypes.data, False)
        st = L.MgStats()
        _check(self._lib.mg_part_pr_result(self._h, C.c_void_p(ptr), int(dev), C.byref(st)), "mg_part_pr_result")
        return res, st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mg_part_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class CollectiveExchange:
    """All-gather of the per-level bitmaps over a torch.distributed group.

    With NCCL the collective is issued on the slice's stream (it follows the
    step's kernels there without a host wait); with gloo the bitmaps are host
    tensors."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self._buf = None

    def gather(self, part, bits):
        import torch
        import torch.distributed as dist

        if self._buf is None or self._buf.numel() != self.world * bits.numel() or self._buf.device != bits.device:
            self._buf = torch.empty(self.world * bits.numel(), dtype=bits.dtype, device=bits.device)
        ctx = part.stream_context() if hasattr(part, "stream_context") and bits.is_cuda else contextlib.nullcontext()
        with ctx:
            dist.all_gather_into_tensor(self._buf, bits, group=self.group)
        return self._buf


def bfs_partitioned(part, srcs, exchange, direction: str = "auto", iter_num: int = 0, out=None):
    """BFS from `srcs` over the ranks of `exchange`; every rank calls it with its
    own slice and the same sources. Returns (depth of all n vertices, stats) on
    every rank."""
    import torch

    lv = part.begin(srcs, direction, iter_num)
    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
    bits = torch.empty(part.words, dtype=torch.int32, device=getattr(part, "device", device))
    levels = []
    while not lv["done"]:
        levels.append(lv["direction"])
        part.step(bits)
        gathered = exchange.gather(part, bits)
        lv = part.merge(gathered, exchange.world)
    depth, st = part.result(out)
    st["directions"] = levels
    return depth, st


def bfs_partitioned_local(parts, srcs, direction: str = "auto", iter_num: int = 0, out=None):
    """The same BFS with every slice on the current GPU: each slice's step writes
    its row of one shared world x words buffer, which stands in for the
    all-gather; every slice then merges that buffer. Returns the depths (they
    agree on every slice; the first slice's are returned) and its stats."""
    import torch

    world = len(parts)
    words = parts[0].words
    buf = torch.empty(world * words, dtype=torch.int32, device="cuda")
    lvs = [p.begin(srcs, direction, iter_num) for p in parts]
    levels = []
    while not lvs[0]["done"]:
        levels.append(lvs[0]["direction"])
        for r, p in enumerate(parts):
            p.step(buf[r * words:(r + 1) * words])
        for p in parts:
            p.synchronize()
        lvs = [p.merge(buf, world) for p in parts]
        if any(lv != lvs[0] for lv in lvs[1:]):
            raise RuntimeError(f"partitions disagree on the level state: {lvs}")
    depth, st = parts[0].result(out)
    st["directions"] = levels
    return depth, st


def pagerank_partitioned(part, cuts, exchange, alpha: float = 0.85, tol: float = 1e-6, max_iter: int = 50,
                         out=None):
    """Normalised PageRank (uniform teleport) over the ranks of `exchange`; every
    rank calls it with its slice and the same cuts. Each iteration all-gathers
    the ranks' new values of their own vertices (slices padded to the largest).
    Returns (ranks of all n vertices, stats) on every rank."""
    import torch

    cuts = np.asarray(cuts, dtype=np.int64)
    stride = int(np.diff(cuts).max()) if cuts.size > 1 else 0
    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
    buf = torch.zeros(max(stride, 1), dtype=torch.float32, device=getattr(part, "device", device))
    lv = part.pr_begin(alpha, tol, max_iter)
    while not lv["done"]:
        part.pr_step(buf)
        gathered = exchange.gather(part, buf)
        lv = part.pr_merge(gathered, exchange.world, max(stride, 1), cuts)
    return part.pr_result(out)


def pagerank_partitioned_local(parts, cuts, alpha: float = 0.85, tol: float = 1e-6, max_iter: int = 50,
                               out=None):
    """The same PageRank with every slice on the current GPU (one shared buffer
    stands in for the all-gather). Returns the first slice's ranks and stats."""
    import torch

    cuts = np.asarray(cuts, dtype=np.int64)
    world = len(parts)
    stride = max(int(np.diff(cuts).max()), 1)
    buf = torch.zeros(world * stride, dtype=torch.float32, device="cuda")
    lvs = [p.pr_begin(alpha, tol, max_iter) for p in parts]
    while not lvs[0]["done"]:
        for r, p in enumerate(parts):
            p.pr_step(buf[r * stride:(r + 1) * stride])
        for p in parts:
            p.synchronize()
        lvs = [p.pr_merge(buf, world, stride, cuts) for p in parts]
        if any(lv != lvs[0] for lv in lvs[1:]):
            raise RuntimeError(f"partitions disagree on the iteration state: {lvs}")
    return parts[0].pr_result(out)
