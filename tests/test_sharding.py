"""Sharding of batched workloads over ranks (host logic, CPU): two gloo ranks
split sources / teleport vectors, run their slice, and all-gather the rows. The
per-rank compute is a deterministic stand-in with the Graph method signatures,
so the test needs no GPU."""
import os
import socket

import numpy as np
import pytest

from mirrorofmapgraph_b200.sharding import shard_range


def test_shard_range_covers_every_instance_once():
    for total in (0, 1, 5, 64, 100):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and b >= a
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


class _FakeGraph:
    """Deterministic stand-in for mirrorofmapgraph_b200.Graph (same signatures)."""
    n = 11

    def bfs_batch(self, srcs, **kw):
        srcs = np.asarray(srcs, np.int32)
        return (np.add.outer(srcs, np.arange(self.n)) % 7).astype(np.int32), {}

    def sssp_batch(self, srcs, **kw):
        srcs = np.asarray(srcs, np.int32)
        return (np.add.outer(3 * srcs, np.arange(self.n)) % 1000).astype(np.int32), {}

    def pagerank(self, teleport=None, nvec=1, **kw):
        t = np.asarray(teleport, np.float32).reshape(nvec, self.n)
        return (2 * t + 0.5).reshape(-1) if nvec == 1 else 2 * t + 0.5, {}


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from mirrorofmapgraph_b200 import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _FakeGraph()
        srcs = np.arange(9, dtype=np.int32) * 5
        tele = np.random.default_rng(0).random((7, g.n)).astype(np.float32)
        d = sharding.bfs_batch_sharded(g, srcs)
        s = sharding.sssp_batch_sharded(g, srcs)
        p = sharding.pagerank_sharded(g, tele)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), d=d, s=s, p=p)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batches_gather_full_results(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    g = _FakeGraph()
    srcs = np.arange(9, dtype=np.int32) * 5
    tele = np.random.default_rng(0).random((7, g.n)).astype(np.float32)
    for r in range(world):
        z = np.load(tmp_path / f"r{r}.npz")
        np.testing.assert_array_equal(z["d"], g.bfs_batch(srcs)[0])
        np.testing.assert_array_equal(z["s"], g.sssp_batch(srcs)[0])
        np.testing.assert_array_equal(z["p"], g.pagerank(tele, nvec=7)[0])
