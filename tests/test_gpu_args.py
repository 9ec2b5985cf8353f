"""Host pointers passed where an entry point needs device memory.

With device_output set, every entry point writes (and reads) the caller's arrays
from its kernels. A host array passed by mistake must come back as MG_ERR_ARG,
checked on the host before any launch, and leave the graph usable; the host
buffer is never touched.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import mirrorofmapgraph_b200 as mg
import oracle
from mirrorofmapgraph_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    h = mg.gen_er(4096, 65536, 17, weights="int", p0=1, p1=64)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        yield h, g


def _opts(**kw):
    o = L.MgOpts()
    o.directed = 1
    o.device_output = 1
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _pr_opts():
    o = L.MgPrOpts()
    o.mode = L.MG_PR_NORMALIZED
    o.directed = 1
    o.max_iter = 20
    o.alpha = 0.85
    o.tol = 1e-6
    o.compensated = 1
    o.device_output = 1
    return o


def _rejected(rc, host):
    lib = L.load()
    assert rc == L.MG_ERR_ARG, rc
    assert "device memory" in lib.mg_last_error().decode()
    assert (host == -7).all()


def test_traversals_reject_host_outputs(graph):
    h, g = graph
    lib = L.load()
    src = np.zeros(1, dtype=np.int32)
    pageable = np.full(g.n, -7, dtype=np.int32)
    pinned = torch.full((g.n,), -7, dtype=torch.int32).pin_memory()
    for buf, ptr in ((pageable, pageable.ctypes.data), (pinned.numpy(), pinned.data_ptr())):
        _rejected(lib.mg_bfs(g._h, src.ctypes.data, 1, ptr, C.byref(_opts()), None), buf)
        _rejected(lib.mg_bfs_batch(g._h, src.ctypes.data, 1, ptr, C.byref(_opts()), None), buf)
        _rejected(lib.mg_sssp(g._h, src.ctypes.data, 1, ptr, C.byref(_opts()), None), buf)
        _rejected(lib.mg_sssp_batch(g._h, src.ctypes.data, 1, ptr, C.byref(_opts()), None), buf)
        _rejected(lib.mg_cc(g._h, ptr, C.byref(_opts(directed=0)), None), buf)
    # the graph still answers, exact against the oracle
    depth, _ = g.bfs([0])
    np.testing.assert_array_equal(depth, oracle.bfs(h.row_offsets, h.col_idx, [0]))


def test_pagerank_and_adjoint_reject_host_arrays(graph):
    h, g = graph
    lib = L.load()
    host = np.full(g.n, -7, dtype=np.float32)
    _rejected(lib.mg_pagerank(g._h, None, 1, host.ctypes.data, C.byref(_pr_opts()), None), host)
    dev = torch.zeros(g.n, dtype=torch.float32, device="cuda")
    w = torch.ones(g.n, dtype=torch.float32, device="cuda")
    # a host gradient output next to device inputs
    rc = lib.mg_pagerank_backward(g._h, None, dev.data_ptr(), w.data_ptr(), None, host.ctypes.data,
                                  C.byref(_pr_opts()), None)
    _rejected(rc, host)
    x, st = g.pagerank(mode="normalized", max_iter=50, tol=1e-6)
    xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 1e-6, st["iterations"])
    assert float(np.abs(x.astype(np.float64) - xr).sum()) <= 1e-6


def test_predecessors_reject_host_arrays(graph):
    h, g = graph
    lib = L.load()
    depth = torch.empty(g.n, dtype=torch.int32, device="cuda")
    host = np.full(g.n, -7, dtype=np.int32)
    o = _opts()
    rc = lib.mg_bfs_predecessors(g._h, depth.data_ptr(), host.ctypes.data, C.byref(o))
    _rejected(rc, host)
