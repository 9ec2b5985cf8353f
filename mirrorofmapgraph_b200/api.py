"""The reference's hot-path interface, on top of the engine.

MapGraph drives a vertex program through three objects (all C++ templates in the
reference): a ``Config`` parameter registry (Algorithms/BFS/config.h:70-175,
config.cpp:30-113, per-program defaults in Algorithms/*/register.h), a
``CsrProblem`` holding the device graph (GASengine/csr_problem.cuh:112-828) and an
``EnactorVertexCentric`` running ``EnactIterativeSearch``
(GASengine/enactor_vertex_centric.cuh:2398-2966). The four bundled programs are
the structs ``bfs``, ``sssp``, ``cc`` and ``pagerank`` (Algorithms/*/*.h).

This module keeps those names, argument meanings and call order::

    cfg = Config(bfs); cfg.parseParameterString("src=1 origin=1")
    csr_problem = CsrProblem(bfs, cfg)
    csr_problem.FromHostProblem(False, nodes, edges, column_indices, row_offsets,
                                edge_values, row_indices, column_offsets, 1, directed)
    enactor = EnactorVertexCentric(csr_problem, bfs, cfg)
    enactor.EnactIterativeSearch(csr_problem, row_offsets, directed, 1, [src],
                                 cfg.getParameter("iter_num"), cfg.getParameter("threshold"))
    h_values = csr_problem.ExtractResults()

Each program tag dispatches to the engine's tuned entry point (mg_bfs, mg_sssp,
mg_cc, mg_pagerank). Errors raise :class:`MapGraphError` / ``KeyError`` where the
reference printed and returned a cudaError_t or threw ``std::exception``.
"""
from __future__ import annotations

import numpy as np

from .graph import Graph, MapGraphError  # noqa: F401

INT_MAX = 2**31 - 1


# ---------------------------------------------------------------------------
# Vertex-program tags (types, INIT_VALUE, allow_duplicates and the five phase
# selectors of each struct).
class _Program:
    name = ""
    DataType = np.int32
    INIT_VALUE = 0
    allow_duplicates = True
    SRC_VERTEX = "SINGLE"
    GATHER = "NO_GATHER_EDGES"
    APPLY = "NO_APPLY_VERTICES"
    POST_APPLY = "NO_POST_APPLY_VERTICES"
    EXPAND = "EXPAND_OUT_EDGES"
    PARAMS: dict = {}

    @classmethod
    def srcVertex(cls):
        return cls.SRC_VERTEX

    @classmethod
    def gatherOverEdges(cls):
        return cls.GATHER

    @classmethod
    def applyOverEdges(cls):
        return cls.APPLY

    @classmethod
    def postApplyOverEdges(cls):
        return cls.POST_APPLY

    @classmethod
    def expandOverEdges(cls):
        return cls.EXPAND


# Parameters registered by every driver (Algorithms/BFS/register.h:27-41).
_COMMON = {
    "verbose": (int, 0, "Print out frontier size in each iteration (default 0)"),
    "device": (int, 0, "The device to use (default 0)"),
    "iter_num": (int, INT_MAX, "The number of iterations to perform (default INT_MAX)"),
    "run_CPU": (int, 0, "Run CPU implementation for testing (default 0)"),
    "max_queue_sizing": (float, 1.5, "The frontier queue size is this value times the number of vertices "
                                     "in the graph (default 1.5)"),
    "threshold": (int, 10000, "When frontier size is larger than threshold, two-phase strategy is used "
                              "otherwise dynamic scheduling it used (default 10000)"),
    "stats": (int, 0, "Print out degree histogram (default 0)"),
}
_SOURCES = {
    "src": (int, 1, "Starting vertex (default 1)"),
    "origin": (int, 1, "The origin (0 or 1) for the starting vertices (default 1)"),
    "directed": (int, 1, "The graph is directed (default 1)"),
    "num_src": (int, 1, "The number of starting vertices when random sources is specified (default 1)"),
}


class bfs(_Program):  # Algorithms/BFS/bfs.h:28-262
    name = "bfs"
    INIT_VALUE = -1
    PARAMS = {**_COMMON, **_SOURCES, "with_value": (int, 0, "Whether to load edge values from market file "
                                                               "(default 0)")}


class sssp(_Program):  # Algorithms/SSSP/sssp.h:33-409
    name = "sssp"
    INIT_VALUE = INT_MAX
    APPLY = "APPLY_FRONTIER"
    POST_APPLY = "POST_APPLY_FRONTIER"
    PARAMS = {**_COMMON, **_SOURCES, "with_value": (int, 1, "Whether to load edge values from market file "
                                                               "(default 1)")}


class cc(_Program):  # Algorithms/CC/cc.h:32-349
    name = "cc"
    INIT_VALUE = INT_MAX
    SRC_VERTEX = "ALL"
    APPLY = "APPLY_FRONTIER"
    POST_APPLY = "POST_APPLY_FRONTIER"
    PARAMS = dict(_COMMON)


class pagerank(_Program):  # Algorithms/PageRank/PageRank.h:33-409
    name = "pagerank"
    DataType = np.float32
    INIT_VALUE = 0.0
    allow_duplicates = False
    SRC_VERTEX = "ALL"
    GATHER = "GATHER_IN_EDGES"
    APPLY = "APPLY_FRONTIER"
    POST_APPLY = "POST_APPLY_FRONTIER"
    PARAMS = {**_COMMON,
              "directed": (int, 1, "The graph is directed (default 1)"),
              "tol": (float, 0.1, "The tolerance for correctness check (default 0.1)"),
              "threshold": (int, 1000, "When frontier size is larger than threshold, two-phase strategy is used "
                                       "otherwise dynamic scheduling it used (default 1000)")}


# ---------------------------------------------------------------------------
class Config:
    """Typed parameter registry with the program's registered defaults.

    Unlike the reference (which dereferences ``end()`` on an unregistered name,
    Algorithms/BFS/config.cpp:88-94, and inverts ``getValue<bool>``,
    getvalue.h:35-46), unknown names raise ``KeyError``."""

    def __init__(self, program=bfs):
        self.program = program
        self._desc = dict(program.PARAMS)
        self._vals: dict = {}

    def getParameter(self, name: str):
        if name not in self._desc:
            raise KeyError(f"getParameter error: '{name}' not found")
        typ, default, _ = self._desc[name]
        return self._vals.get(name, default)

    def setParameter(self, name: str, value) -> None:
        if name not in self._desc:
            raise KeyError(f"setParameter error: '{name}' not found")
        typ = self._desc[name][0]
        self._vals[name] = typ(value) if typ is not int else int(float(value)) if isinstance(value, str) and \
            "." in value else int(value)

    def parseParameterString(self, s: str) -> None:
        """``name=value name=value ...`` (config.cpp:30-42: split on spaces/commas)."""
        for tok in s.replace(",", " ").split():
            if "=" not in tok:
                raise KeyError(f"Variable '{tok}' not registered")
            k, v = tok.split("=", 1)
            self.setParameter(k, v)

    def parseFile(self, path: str) -> None:
        """One or more ``name=value`` per line (config.cpp:45-62)."""
        with open(path) as f:
            for line in f:
                if line.strip():
                    self.parseParameterString(line.strip())

    def printOptions(self) -> str:
        return "\n".join(f"           {k}: {d[2]}" for k, d in sorted(self._desc.items()))


class CsrProblem:
    """Device graph of one vertex program (GASengine/csr_problem.cuh:112-828)."""

    def __init__(self, program, cfg: Config | None = None):
        self.program = program
        self.cfg = cfg or Config(program)
        self.graph: Graph | None = None
        self.nodes = 0
        self.edges = 0
        self._result = None
        self.stats: dict = {}

    def FromHostProblem(self, stream_from_host, nodes, edges, h_column_indices, h_row_offsets, h_edge_values=None,
                        h_row_indices=None, h_column_offsets=None, num_gpus: int = 1, directed: int = 1):
        """Uploads the host CSR; the CSC is rebuilt on the device (h_row_indices and
        h_column_offsets are accepted and, as in the reference, not used)."""
        if num_gpus > 1:
            raise MapGraphError(7, "CsrProblem.FromHostProblem", "Multi GPU is not supported yet!")
        ro = np.asarray(h_row_offsets, dtype=np.int32)[: nodes + 1]
        ci = np.asarray(h_column_indices, dtype=np.int32)[:edges]
        vals = None
        if h_edge_values is not None:
            dt = np.float32 if self.program.DataType == np.float32 else np.int32
            vals = np.asarray(h_edge_values)[:edges].astype(dt)
        if self.graph is not None:
            self.graph.close()
        self.graph = Graph(ro, ci, vals)
        self.nodes, self.edges = int(nodes), int(edges)
        return 0

    def ExtractResults(self):
        """The program's per-vertex result (labels / dists / ranks), csr_problem.cuh:371-396."""
        if self._result is None:
            raise MapGraphError(1, "CsrProblem.ExtractResults", "no search has run")
        return self._result.copy()


class EnactorVertexCentric:
    """Runs a vertex program on a CsrProblem (GASengine/enactor_vertex_centric.cuh:91-2968)."""

    def __init__(self, csr_problem_or_cfg=None, program=None, cfg: Config | None = None, DEBUG: bool = False):
        if isinstance(csr_problem_or_cfg, Config):
            cfg = csr_problem_or_cfg
        self.program = program
        self.cfg = cfg
        self.DEBUG = DEBUG

    def EnactIterativeSearch(self, csr_problem: CsrProblem, h_row_offsets=None, directed: int = 1,
                             num_srcs: int = 1, srcs=None, iter_num: int = INT_MAX, threshold: int = 10000):
        prog = self.program or csr_problem.program
        cfg = self.cfg or csr_problem.cfg
        g = csr_problem.graph
        if g is None:
            raise MapGraphError(1, "EnactIterativeSearch", "CsrProblem has no graph")
        it = 0 if iter_num is None or iter_num >= INT_MAX else int(iter_num)
        qs = float(cfg.getParameter("max_queue_sizing")) if "max_queue_sizing" in cfg._desc else 0.0
        # The reference sizes O(m) edge queues; the engine's are vertex-sized, so
        # only factors below 1 constrain them.
        qs = qs if 0 < qs < 1 else 0.0
        if prog is bfs or prog is sssp:
            if srcs is None:
                raise MapGraphError(1, "EnactIterativeSearch", "sources required")
            s = np.asarray(srcs, dtype=np.int32)[:num_srcs]
            fn = g.bfs if prog is bfs else g.sssp
            res, st = fn(s, directed=directed, iter_num=it, queue_sizing=qs, threshold=threshold)
        elif prog is cc:
            # Algorithms/CC/cc.cu:289: CC always runs undirected.
            res, st = g.cc(directed=0, iter_num=it)
        elif prog is pagerank:
            res, st = g.pagerank(mode="refcompat", directed=directed, max_iter=it)
        else:
            raise MapGraphError(7, "EnactIterativeSearch", f"unsupported program {prog!r}")
        csr_problem._result = res
        csr_problem.stats = st
        return 0
