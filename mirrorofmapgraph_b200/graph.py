"""Device-resident graphs and the vertex programs, over the engine's C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class MapGraphError(RuntimeError):
    """A non-OK mg_status from the engine."""

    def __init__(self, status: int, where: str, detail: str):
        self.status = status
        super().__init__(f"{where}: {status_name(status)} ({detail})")


def status_name(st: int) -> str:
    return L.load().mg_status_string(st).decode()


def _check(st: int, where: str) -> None:
    if st != L.MG_OK:
        raise MapGraphError(st, where, L.load().mg_last_error().decode())


def device_count() -> int:
    return int(L.load().mg_device_count())


def version() -> str:
    return L.load().mg_version().decode()


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, dtype=None):
    """(address, is_device, keepalive) of a NumPy array or a torch tensor."""
    if x is None:
        return None, False, None
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr(), bool(x.is_cuda), x
    a = np.ascontiguousarray(x, dtype=dtype) if dtype is not None else np.ascontiguousarray(x)
    return a.ctypes.data, False, a


def _len(x) -> int:
    return int(x.numel()) if _is_torch(x) else int(np.asarray(x).size)


def _opts(directed=1, iter_num=0, direction="auto", device_output=False, queue_sizing=0.0, threshold=0,
          use_graph=True, delta=0) -> L.MgOpts:
    o = L.MgOpts()
    o.directed = int(directed)
    o.iter_num = int(iter_num) if iter_num else 0
    o.direction = {"auto": L.MG_DIR_AUTO, "push": L.MG_DIR_PUSH, "pull": L.MG_DIR_PULL}[direction]
    o.device_output = int(device_output)
    o.queue_sizing = float(queue_sizing)
    o.threshold = int(threshold)
    o.use_graph = 0 if use_graph else -1
    o.delta = int(delta)
    return o


class Graph:
    """A CSR graph (and its transpose) resident on the current CUDA device.

    Arguments are int32 row offsets (n+1) and column indices (m), optionally int32
    or float32 edge values, as NumPy arrays / host tensors (copied to the device)
    or CUDA tensors (copied device to device). ``symmetric=True`` promises the CSR
    is its own transpose, so no CSC is built. Mirrors CsrProblem::FromHostProblem
    (GASengine/csr_problem.cuh:401-621).
    """

    def __init__(self, row_offsets, col_idx, values=None, symmetric: bool = False, build_csc: bool = True,
                 async_upload: bool = False, _handle=None):
        """async_upload (symmetric graphs, or build_csc=False): return as soon as the
        upload is enqueued, so it overlaps work on other graphs; the input arrays are
        kept referenced by the graph until it is closed, and an invalid CSR is
        reported by the first call on the graph (or by sync())."""
        self._lib = L.load()
        self._h = C.c_void_p()
        self._keep = None
        if _handle is not None:
            self._h = _handle
        else:
            n = _len(row_offsets) - 1
            m = _len(col_idx)
            ro_p, ro_dev, k1 = _ptr(row_offsets, np.int32)
            ci_p, ci_dev, k2 = _ptr(col_idx, np.int32)
            vt = L.MG_DTYPE_NONE
            v_p, v_dev, k3 = None, False, None
            if values is not None:
                dt = str(values.dtype)
                if "int32" in dt:
                    vt = L.MG_DTYPE_I32
                elif "float32" in dt:
                    vt = L.MG_DTYPE_F32
                else:
                    raise ValueError("edge values must be int32 or float32")
                v_p, v_dev, k3 = _ptr(values)
            if len({ro_dev, ci_dev} | ({v_dev} if values is not None else set())) != 1:
                raise ValueError("graph arrays must all be on the host or all on the device")
            flags = (L.MG_GRAPH_SYMMETRIC if symmetric else 0) | (0 if build_csc else L.MG_GRAPH_NO_CSC)
            if ro_dev:
                flags |= L.MG_GRAPH_DEVICE_INPUT
            if async_upload:
                flags |= L.MG_GRAPH_ASYNC_UPLOAD
            _check(self._lib.mg_graph_create(ro_p, ci_p, v_p, vt, n, m, flags, C.byref(self._h)),
                   "mg_graph_create")
            if async_upload:
                self._keep = (k1, k2, k3)  # the copy may still be reading them
            del k1, k2, k3
        n, m, fl, dev = C.c_int64(), C.c_int64(), C.c_uint32(), C.c_int32()
        _check(self._lib.mg_graph_info(self._h, C.byref(n), C.byref(m), C.byref(fl), C.byref(dev)), "mg_graph_info")
        self.n, self.m, self.flags, self.device = n.value, m.value, fl.value, dev.value

    @classmethod
    def from_host_csr(cls, g, values: str | None = None, symmetric: bool = False, build_csc: bool = True):
        vals = {None: None, "i32": g.weights_i32, "f32": g.weights_f32}[values]
        if values is not None and vals is None:
            raise ValueError(f"host graph has no {values} weights")
        return cls(g.row_offsets, g.col_idx, vals, symmetric=symmetric, build_csc=build_csc)

    @classmethod
    def ragged(cls, graphs, symmetric: bool = False):
        """Disjoint union of independent host graphs (mg_graph_create_ragged)."""
        lib = L.load()
        k = len(graphs)
        ros = [np.ascontiguousarray(g.row_offsets, dtype=np.int32) for g in graphs]
        cis = [np.ascontiguousarray(g.col_idx, dtype=np.int32) for g in graphs]
        ro_arr = (C.c_void_p * k)(*[r.ctypes.data for r in ros])
        ci_arr = (C.c_void_p * k)(*[c.ctypes.data for c in cis])
        ns = np.array([r.size - 1 for r in ros], dtype=np.int64)
        ms = np.array([c.size for c in cis], dtype=np.int64)
        h = C.c_void_p()
        _check(lib.mg_graph_create_ragged(k, ro_arr, ci_arr, ns.ctypes.data, ms.ctypes.data,
                                          L.MG_GRAPH_SYMMETRIC if symmetric else 0, C.byref(h)),
               "mg_graph_create_ragged")
        obj = cls(None, None, _handle=h)
        obj.ngraphs = k
        return obj

    def ragged_bases(self) -> np.ndarray:
        out = np.empty(self.ngraphs + 1, dtype=np.int64)
        _check(self._lib.mg_graph_ragged_bases(self._h, out.ctypes.data), "mg_graph_ragged_bases")
        return out

    # -- lifetime ---------------------------------------------------------------
    def sync(self) -> None:
        """Waits for an asynchronous upload and checks it (mg_graph_sync)."""
        _check(self._lib.mg_graph_sync(self._h), "mg_graph_sync")

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.mg_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream_ptr(self) -> int:
        """cudaStream_t of the graph as an integer (for torch.cuda.ExternalStream)."""
        p = C.c_void_p()
        _check(self._lib.mg_graph_stream(self._h, C.byref(p)), "mg_graph_stream")
        return p.value or 0

    def device_arrays(self) -> dict:
        ptrs = [C.c_void_p() for _ in range(6)]
        _check(self._lib.mg_graph_device_arrays(self._h, *[C.byref(p) for p in ptrs]), "mg_graph_device_arrays")
        names = ["row_offsets", "col_idx", "edge_vals", "col_offsets", "row_idx", "csc_perm"]
        return {k: p.value for k, p in zip(names, ptrs)}

    def trace(self) -> list[dict]:
        """Per-level records of the last mg_bfs / mg_sssp / single-vector normalised
        PageRank run on this graph (the reference's verbose per-iteration print):
        level, direction, frontier size, frontier out-edges, value (PageRank: the
        iteration's L1 change)."""
        recs = (L.MgLevelRecord * L.MG_TRACE_LEVELS)()
        cnt = C.c_int32()
        _check(self._lib.mg_graph_trace(self._h, recs, L.MG_TRACE_LEVELS, C.byref(cnt)), "mg_graph_trace")
        names = {L.MG_DIR_PUSH: "push", L.MG_DIR_PULL: "pull"}
        out = [{"level": r.level, "direction": names.get(r.direction, "push"), "frontier": r.frontier,
                "frontier_edges": r.frontier_edges, "value": r.value, "time_ns": r.time_ns}
               for r in recs[: cnt.value]]
        # duration of each level: from the previous level's end (the first has none)
        for a, b in zip(out, out[1:]):
            b["ns"] = b["time_ns"] - a["time_ns"]
        return out

    @staticmethod
    def default_tuning() -> dict:
        """The default traversal tuning (mg_tuning_defaults); needs no device."""
        t = L.MgTuning()
        L.load().mg_tuning_defaults(C.byref(t))
        return t.as_dict()

    def tuning(self) -> dict:
        """The graph's traversal tuning (mg_graph_get_tuning): thresholds and launch
        shapes the traversal kernels read at every call."""
        t = L.MgTuning()
        _check(self._lib.mg_graph_get_tuning(self._h, C.byref(t)), "mg_graph_get_tuning")
        return t.as_dict()

    def set_tuning(self, **fields) -> dict:
        """Changes tuning fields by name (the others keep their values); returns the
        new tuning. A value outside a field's range raises MapGraphError and
        changes nothing."""
        t = L.MgTuning()
        _check(self._lib.mg_graph_get_tuning(self._h, C.byref(t)), "mg_graph_get_tuning")
        for k, v in fields.items():
            if k == "reserved" or k not in dict(L.MgTuning._fields_):
                raise KeyError(f"unknown tuning field {k!r}")
            setattr(t, k, int(v))
        _check(self._lib.mg_graph_set_tuning(self._h, C.byref(t)), "mg_graph_set_tuning")
        return t.as_dict()

    # -- helpers ----------------------------------------------------------------
    def _out(self, out, count, dtype):
        if out is None:
            a = np.empty(count, dtype=dtype)
            return a, a.ctypes.data, False
        if _is_torch(out):
            if out.numel() != count:
                raise ValueError(f"output must have {count} elements")
            return out, out.data_ptr(), bool(out.is_cuda)
        if out.size != count:
            raise ValueError(f"output must have {count} elements")
        return out, out.ctypes.data, False

    @staticmethod
    def _srcs(srcs):
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(srcs)), dtype=np.int32)
        return a, a.ctypes.data, int(a.size)

    # -- vertex programs ------------------------------------------------------------
    def bfs(self, srcs, out=None, **kw):
        """struct bfs: depth from the nearest source (-1 unreached). Returns (depth, stats)."""
        s, sp, ns = self._srcs(srcs)
        res, rp, dev = self._out(out, self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_bfs(self._h, sp, ns, rp, C.byref(o), C.byref(st)), "mg_bfs")
        return res, st.as_dict()

    def bfs_predecessors(self, depth, out=None):
        """Predecessors from a depth array (the reference's pred_extract): the largest
        in-neighbour one level closer, -1 where none."""
        d_p, d_dev, keep = _ptr(depth, np.int32)
        res, rp, dev = self._out(out, self.n, np.int32)
        if d_dev != dev:
            raise ValueError("depth and out must both be host or both be device arrays")
        o = _opts(device_output=dev)
        _check(self._lib.mg_bfs_predecessors(self._h, d_p, rp, C.byref(o)), "mg_bfs_predecessors")
        return res

    def sssp(self, srcs, out=None, **kw):
        """struct sssp: shortest distance from the nearest source (INT_MAX unreached)."""
        s, sp, ns = self._srcs(srcs)
        res, rp, dev = self._out(out, self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_sssp(self._h, sp, ns, rp, C.byref(o), C.byref(st)), "mg_sssp")
        return res, st.as_dict()

    def cc(self, out=None, **kw):
        """struct cc: smallest vertex id of each weakly connected component."""
        res, rp, dev = self._out(out, self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_cc(self._h, rp, C.byref(o), C.byref(st)), "mg_cc")
        return res, st.as_dict()

    def bfs_batch(self, srcs, out=None, **kw):
        s, sp, ns = self._srcs(srcs)
        res, rp, dev = self._out(out, ns * self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_bfs_batch(self._h, sp, ns, rp, C.byref(o), C.byref(st)), "mg_bfs_batch")
        return (res.reshape(ns, self.n) if not _is_torch(res) else res), st.as_dict()

    def sssp_batch(self, srcs, out=None, **kw):
        s, sp, ns = self._srcs(srcs)
        res, rp, dev = self._out(out, ns * self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_sssp_batch(self._h, sp, ns, rp, C.byref(o), C.byref(st)), "mg_sssp_batch")
        return (res.reshape(ns, self.n) if not _is_torch(res) else res), st.as_dict()

    def bfs_ragged(self, srcs, out=None, **kw):
        s, sp, ns = self._srcs(srcs)
        if ns != self.ngraphs:
            raise ValueError("one source per member graph")
        res, rp, dev = self._out(out, self.n, np.int32)
        st = L.MgStats()
        o = _opts(device_output=dev, **kw)
        _check(self._lib.mg_bfs_ragged(self._h, sp, rp, C.byref(o), C.byref(st)), "mg_bfs_ragged")
        return res, st.as_dict()

    @staticmethod
    def _pr_opts(mode="refcompat", directed=1, max_iter=0, weighted=False, alpha=0.85, tol=None,
                 compensated=True, device_output=False, use_graph=True, gather="binned",
                 autotune=False, group_width=0, seg_hub_edges=0, seg_block_cols=0) -> L.MgPrOpts:
        o = L.MgPrOpts()
        o.seg_hub_edges = int(seg_hub_edges)
        o.seg_block_cols = int(seg_block_cols)
        o.autotune = 1 if autotune else 0
        o.group_width = int(group_width)
        o.gather_kernel = {"binned": 0, "tma": 1, "cached": 2, "segmented": 3}[gather]
        o.mode = {"refcompat": L.MG_PR_REFCOMPAT, "normalized": L.MG_PR_NORMALIZED}[mode]
        o.directed = int(directed)
        o.max_iter = int(max_iter)
        o.weighted = int(weighted)
        o.alpha = float(alpha)
        o.tol = 0.0 if tol is None else float(tol)
        o.compensated = 1 if compensated else -1
        o.device_output = int(device_output)
        o.use_graph = 0 if use_graph else -1
        return o

    def pagerank(self, teleport=None, nvec: int = 1, out=None, **kw):
        """struct pagerank (refcompat) or the normalised / personalised power iteration.

        Keywords (mg_pr_opts): mode "refcompat" | "normalized", alpha, tol, max_iter,
        weighted, directed (refcompat), gather "binned" | "cached" | "tma" | "segmented",
        autotune (time the gathers, or with nvec > 1 the group width, once per
        graph), group_width (nvec > 1: vectors per pass, a multiple of 32 <= 256),
        compensated, use_graph. Returns (ranks, stats); with nvec > 1 the ranks are
        nvec x n and stats["status_detail"] is the group width used."""
        t_p, t_dev, keep = _ptr(teleport, np.float32) if teleport is not None else (None, False, None)
        res, rp, dev = self._out(out, nvec * self.n, np.float32)
        st = L.MgStats()
        o = self._pr_opts(device_output=dev, **kw)
        _check(self._lib.mg_pagerank(self._h, t_p, nvec, rp, C.byref(o), C.byref(st)), "mg_pagerank")
        if nvec > 1 and not _is_torch(res):
            res = res.reshape(nvec, self.n)
        return res, st.as_dict()

    def pagerank_backward(self, ranks, dL_dranks, teleport=None, want_weights=True, want_teleport=True,
                          out_weights=None, out_teleport=None, **kw):
        """Adjoint of the normalised PageRank fixed point: (dL/dweights[m], dL/dteleport[n], stats)."""
        r_p, r_dev, k1 = _ptr(ranks, np.float32)
        w_p, w_dev, k2 = _ptr(dL_dranks, np.float32)
        t_p, t_dev, k3 = _ptr(teleport, np.float32) if teleport is not None else (None, False, None)
        gw, gw_p, dev1 = self._out(out_weights, self.m, np.float32) if want_weights else (None, None, r_dev)
        gt, gt_p, dev2 = self._out(out_teleport, self.n, np.float32) if want_teleport else (None, None, r_dev)
        st = L.MgStats()
        kw.setdefault("mode", "normalized")
        o = self._pr_opts(device_output=r_dev, **kw)
        _check(self._lib.mg_pagerank_backward(self._h, t_p, r_p, w_p, gw_p, gt_p, C.byref(o), C.byref(st)),
               "mg_pagerank_backward")
        return gw, gt, st.as_dict()
