"""1-D vertex partition (host logic, CPU): cut points, row slices, and the level
protocols of bfs_partitioned and pagerank_partitioned over two and three gloo
ranks. Each rank's device step is stood in for by a NumPy slice with the
GraphSlice method signatures (begin / step / merge / result on n-bit bitmaps;
pr_begin / pr_step / pr_merge / pr_result on padded float slices); depths and
ranks are checked against the oracle."""
import os
import socket

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200.partition import partition_cuts, slice_rows


def test_cuts_cover_vertices_on_word_boundaries():
    h = mg.gen_rmat(12, 8, 3)
    for world in (1, 2, 3, 5, 8):
        c = partition_cuts(h.row_offsets, world)
        assert c[0] == 0 and c[-1] == h.n and len(c) == world + 1
        assert (np.diff(c) >= 0).all()
        assert all(x % 32 == 0 for x in c[:-1])
        work = np.asarray(h.row_offsets, np.int64) + np.arange(h.n + 1)
        share = np.diff(work[c])
        assert share.max() <= work[-1] / world + np.diff(work).max() + 32 * (1 + np.diff(h.row_offsets).max())
    tiny = np.array([0, 1, 2, 2], np.int32)
    assert list(partition_cuts(tiny, 4)) == [0, 0, 0, 0, 3]


def test_slices_rebuild_the_graph_and_its_transpose():
    h = mg.gen_er(700, 4000, 11)
    c = partition_cuts(h.row_offsets, 3)
    co, ri, _ = oracle.csc_of(h.row_offsets, h.col_idx)
    outs, ins = [], []
    for r in range(3):
        oo, oi, io, ii = slice_rows(h.row_offsets, h.col_idx, int(c[r]), int(c[r + 1]))
        assert oo[0] == 0 and io[0] == 0
        outs.append((oo, oi))
        ins.append((io, ii))
    np.testing.assert_array_equal(np.concatenate([oi for _, oi in outs]), h.col_idx)
    np.testing.assert_array_equal(np.concatenate([ii for _, ii in ins]), ri)
    deg_in = np.concatenate([np.diff(io) for io, _ in ins])
    np.testing.assert_array_equal(deg_in, np.diff(co))
    oo, oi, io, ii = slice_rows(h.row_offsets, h.col_idx, 64, 128, symmetric=True)
    assert io is None and ii is None and oo.size == 65


class _NumpySlice:
    """Stand-in for GraphSlice on the host: the same level protocol on n-bit
    bitmaps (bit i of word w is vertex 32 w + i), the same Beamer rule."""
    device = "cpu"

    def __init__(self, ro, ci, lo, hi):
        self.ro = np.asarray(ro, np.int64)
        self.ci = np.asarray(ci, np.int32)
        self.n = self.ro.size - 1
        self.lo, self.hi = lo, hi
        self.words = (self.n + 31) // 32
        self.deg = np.diff(self.ro)
        self.m_total = int(self.deg.sum())
        co, ri, _ = oracle.csc_of(ro, ci)
        self.co, self.ri = np.asarray(co, np.int64), np.asarray(ri, np.int32)

    def _pack(self, mask):
        pad = np.zeros(self.words * 32, bool)
        pad[: self.n] = mask
        return np.packbits(pad, bitorder="little").view("<u4").view(np.int32)

    def _unpack(self, words):
        return np.unpackbits(np.asarray(words, np.int32).view(np.uint8), bitorder="little")[: self.n].astype(bool)

    def begin(self, srcs, direction="auto", iter_num=0):
        self.mode = direction
        self.vis = np.zeros(self.n, bool)
        self.depth = np.full(self.n, -1, np.int32)
        s = np.unique(np.asarray(srcs))
        self.vis[s] = True
        self.depth[s] = 0
        self.fr = self.vis.copy()
        self.level, self.dir = 0, "push"
        self.nf, self.mf = int(s.size), int(self.deg[s].sum())
        self.vdeg = self.mf
        self.cap = iter_num if iter_num > 0 else self.n + 1
        self.done = self.nf == 0
        return self._lv()

    def _lv(self):
        return {"frontier": self.nf, "frontier_edges": self.mf, "level": self.level, "done": self.done,
                "direction": self.dir}

    def step(self, bits):
        import torch
        disc = np.zeros(self.n, bool)
        own = np.zeros(self.n, bool)
        own[self.lo:self.hi] = True
        if self.dir == "push":
            for v in np.flatnonzero(self.fr & own):
                t = self.ci[self.ro[v]:self.ro[v + 1]]
                disc[t[~self.vis[t]]] = True
        else:
            for v in np.flatnonzero(own & ~self.vis):
                if self.fr[self.ri[self.co[v]:self.co[v + 1]]].any():
                    disc[v] = True
        bits.copy_(torch.from_numpy(self._pack(disc)))

    def merge(self, gathered, world):
        g = gathered.numpy().reshape(world, self.words)
        new = np.zeros(self.n, bool)
        for r in range(world):
            new |= self._unpack(g[r])
        new &= ~self.vis
        self.vis |= new
        self.depth[new] = self.level + 1
        self.fr = new
        self.level += 1
        self.nf, self.mf = int(new.sum()), int(self.deg[new].sum())
        self.vdeg += self.mf
        self.done = self.nf == 0 or self.level >= self.cap
        if not self.done:
            if self.mode != "auto":
                self.dir = self.mode
            elif self.dir == "push":
                self.dir = "pull" if self.mf > (self.m_total - self.vdeg) // 14 else "push"
            else:
                self.dir = "push" if self.nf * 24 < self.n else "pull"
        return self._lv()

    def result(self, out=None):
        return self.depth.copy(), {"iterations": self.level, "edges_traversed": self.vdeg}

    # PageRank protocol (normalised, uniform teleport): FP64 stand-in.
    def pr_begin(self, alpha=0.85, tol=1e-6, max_iter=50):
        self.alpha, self.tol, self.max_iter = alpha, tol, max_iter
        self.x = np.full(self.n, 1.0 / self.n)
        self.plevel, self.resid = 0, 0.0
        self.pdone = max_iter <= 0
        return {"level": 0, "done": self.pdone, "residual": 0.0}

    def _y(self):
        return np.where(self.deg > 0, self.x / np.maximum(self.deg, 1), 0.0)

    def pr_step(self, slice_):
        import torch
        y, t = self._y(), 1.0 / self.n
        d = self.x[self.deg == 0].sum()
        v = np.arange(self.lo, self.hi)
        acc = np.array([y[self.ri[self.co[u]:self.co[u + 1]]].sum() for u in v])
        slice_[: self.hi - self.lo] = torch.from_numpy((self.alpha * (acc + d * t) + (1 - self.alpha) * t)
                                                       .astype(np.float32))

    def pr_merge(self, gathered, world, stride, cuts):
        g = gathered.numpy().reshape(world, stride).astype(np.float64)
        new = np.concatenate([g[r, : cuts[r + 1] - cuts[r]] for r in range(world)])
        self.resid = float(np.abs(new - self.x).sum())
        self.x = new
        self.plevel += 1
        self.pdone = self.resid < self.tol or self.plevel >= self.max_iter
        return {"level": self.plevel, "done": self.pdone, "residual": self.resid}

    def pr_result(self, out=None):
        return self.x.copy(), {"iterations": self.plevel, "residual": self.resid}


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from mirrorofmapgraph_b200.partition import CollectiveExchange, bfs_partitioned, pagerank_partitioned
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = {}
        for name, h in (("rmat", mg.gen_rmat(11, 8, 5)), ("lattice", mg.gen_lattice(40, 30, 0.0, 2))):
            c = partition_cuts(h.row_offsets, world)
            part = _NumpySlice(h.row_offsets, h.col_idx, int(c[rank]), int(c[rank + 1]))
            ex = CollectiveExchange()
            for mode in ("auto", "push", "pull"):
                d, st = bfs_partitioned(part, [0, 7], ex, direction=mode)
                res[f"{name}_{mode}"] = d
                res[f"{name}_{mode}_levels"] = np.array([st["iterations"], st["edges_traversed"]])
                res[f"{name}_{mode}_dirs"] = np.array([x == "pull" for x in st["directions"]])
            x, st = pagerank_partitioned(part, c, ex)
            res[f"{name}_pr"] = x
            res[f"{name}_pr_iters"] = np.array([st["iterations"]])
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), **res)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_bfs_protocol_over_gloo_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    graphs = {"rmat": mg.gen_rmat(11, 8, 5), "lattice": mg.gen_lattice(40, 30, 0.0, 2)}
    z0 = np.load(tmp_path / "r0.npz")
    for name, h in graphs.items():
        ref = oracle.bfs(h.row_offsets, h.col_idx, [0, 7])
        for mode in ("auto", "push", "pull"):
            for r in range(world):
                z = np.load(tmp_path / f"r{r}.npz")
                np.testing.assert_array_equal(z[f"{name}_{mode}"], ref)
                np.testing.assert_array_equal(z[f"{name}_{mode}_levels"], z0[f"{name}_{mode}_levels"])
                np.testing.assert_array_equal(z[f"{name}_{mode}_dirs"], z0[f"{name}_{mode}_dirs"])
            lv = z0[f"{name}_{mode}_levels"]
            assert lv[0] == ref.max() + 1
            assert lv[1] == int(np.diff(h.row_offsets)[ref >= 0].sum())
            dirs = z0[f"{name}_{mode}_dirs"]
            it = int(z0[f"{name}_pr_iters"][0])
            xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, it)
            for r in range(world):
                z = np.load(tmp_path / f"r{r}.npz")
                assert np.abs(z[f"{name}_pr"] - xr).sum() <= 1e-6
                np.testing.assert_array_equal(z[f"{name}_pr"], z0[f"{name}_pr"])
            if mode == "push":
                assert not dirs.any()
            if mode == "pull":
                assert dirs[1:].all() and not dirs[0]
