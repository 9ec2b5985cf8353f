"""mirrorofmapgraph_b200 -- a B200-native (sm_100a) Gather-Apply-Scatter graph engine.

The engine is the CUDA library ``lib/libmapgraph_b200.so`` behind the C ABI of
``include/mapgraph_b200.h``. This package is its Python host side:

* :class:`Graph` -- a device-resident CSR/CSC graph with one method per vertex
  program (``bfs``, ``sssp``, ``cc``, ``pagerank``, batched and adjoint forms);
* :mod:`.api` -- the reference's own interface for the hot path
  (``Config``, ``CsrProblem``, ``EnactorVertexCentric`` and the program tags
  ``bfs``, ``sssp``, ``cc``, ``pagerank``), so code written against MapGraph's
  template API reads the same;
* :mod:`.generators` -- seeded synthetic graphs and Matrix Market ingest.

Results are NumPy arrays (host) unless device output is requested with a torch
CUDA tensor. There is no CPU fallback: without the library or a GPU every compute
call raises :class:`MapGraphError`.
"""
from __future__ import annotations

from .graph import Graph, MapGraphError, device_count, version  # noqa: F401
from .generators import (HostCsr, gen_er, gen_lattice, gen_rmat, read_market, csr_to_csc,  # noqa: F401
                         mixed_degree_sources, sparse_teleports, write_market, save_csr, load_csr)
from .api import Config, CsrProblem, EnactorVertexCentric, bfs, sssp, cc, pagerank  # noqa: F401

__all__ = [
    "Graph", "MapGraphError", "device_count", "version", "HostCsr", "gen_er", "gen_rmat", "gen_lattice",
    "read_market", "csr_to_csc", "mixed_degree_sources", "sparse_teleports", "write_market", "save_csr", "load_csr", "Config", "CsrProblem", "EnactorVertexCentric", "bfs", "sssp", "cc", "pagerank",
]
