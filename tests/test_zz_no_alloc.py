"""mg_bfs_noalloc (BFS over the fixed static scratch array) against mg_bfs.

The file name sorts last, so in a full run these tests execute after every other
GPU test in the same process; they also pass alone in a fresh process. BFS depths
are integers: the comparison is exact (tolerance 0). Besides matching mg_bfs,
the tests check the property the entry point exists for: with every device
allocation of the library made to fail (mg_debug_fail_alloc), calls still
succeed, and the device's free memory does not move across a warm call.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import mirrorofmapgraph_b200 as mg
import oracle
from mirrorofmapgraph_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _noalloc(g, srcs, out, directed=1, direction=L.MG_DIR_AUTO, queue_sizing=0.0):
    lib = L.load()
    s = np.ascontiguousarray(srcs, dtype=np.int32)
    o = L.MgOpts()
    o.directed = directed
    o.direction = direction
    o.queue_sizing = queue_sizing
    st = L.MgStats()
    rc = lib.mg_bfs_noalloc(g._h, s.ctypes.data, int(s.size), C.c_void_p(out.data_ptr()), C.byref(o),
                            C.byref(st))
    return rc, st


def _reference(g, srcs, **kw):
    depth, st = g.bfs(srcs, **kw)
    return depth, st


def _two_calls_match(g, srcs, directed=1, direction="auto"):
    code = {"auto": L.MG_DIR_AUTO, "push": L.MG_DIR_PUSH, "pull": L.MG_DIR_PULL}[direction]
    ref, rst = _reference(g, srcs, directed=directed, direction=direction)
    for _ in range(2):
        out = torch.full((g.n,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc, st = _noalloc(g, srcs, out, directed=directed, direction=code)
        assert rc == L.MG_OK, L.load().mg_last_error().decode()
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        assert st.iterations == rst["iterations"]
        assert st.edges_traversed == rst["edges_traversed"]


@pytest.mark.parametrize("direction", ["auto", "push", "pull"])
def test_rmat_symmetric_matches_mg_bfs(direction):
    h = mg.gen_rmat(18, 16, 7, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        deg = np.diff(h.row_offsets)
        _two_calls_match(g, [int(np.argmax(deg))], direction=direction)
        _two_calls_match(g, [0, 5, 77, int(h.n - 1)], direction=direction)


@pytest.mark.parametrize("directed", [1, 0])
def test_directed_graph_both_modes(directed):
    h = mg.gen_er(1 << 16, 1 << 19, 11)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        _two_calls_match(g, [3], directed=directed)


def test_largest_accepted_graph():
    n = L.MG_BFS_NOALLOC_MAX_VERTICES
    h = mg.gen_er(n, 4 * n, 5)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        _two_calls_match(g, [1])


def test_rejects_sizes_beyond_the_scratch():
    n = L.MG_BFS_NOALLOC_MAX_VERTICES + 1
    h = mg.gen_er(n, 2 * n, 9)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(g, [0], out)
        assert rc == L.MG_ERR_ARG
        assert "fixed scratch" in L.load().mg_last_error().decode()
    h = mg.gen_er(1000, 4000, 9)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        out = torch.empty(h.n, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(g, np.zeros(L.MG_BFS_NOALLOC_MAX_SOURCES + 1, dtype=np.int32), out)
        assert rc == L.MG_ERR_ARG
        rc, _ = _noalloc(g, [1000], out)
        assert rc == L.MG_ERR_ARG


def test_allocates_nothing_on_a_fresh_graph():
    """A graph that never ran mg_bfs has no workspace: with the allocation hook
    failing every library allocation, two calls still succeed and match the oracle."""
    lib = L.load()
    h = mg.gen_rmat(16, 16, 21, symmetrize=True)
    ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        out = torch.full((g.n,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert lib.mg_debug_fail_alloc(1) == L.MG_OK
        try:
            for _ in range(2):
                rc, st = _noalloc(g, [0], out)
                assert rc == L.MG_OK, lib.mg_last_error().decode()
                np.testing.assert_array_equal(out.cpu().numpy(), ref)
        finally:
            lib.mg_debug_fail_alloc(0)
        # the hook was live: an allocating entry point fails under it
        assert lib.mg_debug_fail_alloc(1) == L.MG_OK
        try:
            with pytest.raises(mg.MapGraphError):
                g.bfs([0])
        finally:
            lib.mg_debug_fail_alloc(0)


def test_free_memory_unchanged_across_a_warm_call():
    h = mg.gen_er(1 << 18, 1 << 21, 23)
    ref = oracle.bfs(h.row_offsets, h.col_idx, [5])
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        out = torch.empty(g.n, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(g, [5], out)  # warm-up: module and symbol set-up
        assert rc == L.MG_OK
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, _ = _noalloc(g, [5], out)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == L.MG_OK
        assert free1 == free0
        np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_host_depth_pointer_is_rejected_before_any_launch():
    lib = L.load()
    h = mg.gen_er(4096, 65536, 3)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        host = np.full(g.n, -7, dtype=np.int32)
        s = np.zeros(1, dtype=np.int32)
        o = L.MgOpts()
        o.directed = 1
        rc = lib.mg_bfs_noalloc(g._h, s.ctypes.data, 1, host.ctypes.data, C.byref(o), None)
        assert rc == L.MG_ERR_ARG
        assert "device memory" in lib.mg_last_error().decode()
        assert (host == -7).all()
        # the graph is still usable
        out = torch.empty(g.n, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(g, [0], out)
        assert rc == L.MG_OK
        np.testing.assert_array_equal(out.cpu().numpy(), oracle.bfs(h.row_offsets, h.col_idx, [0]))
