"""Batched workloads across ranks (one process per GPU, torch.distributed).

The instances of a batch -- BFS/SSSP sources, personalised PageRank vectors,
member graphs of a ragged batch -- are independent, so they shard without any
exchange during the run: every rank holds the whole graph, runs a contiguous
slice of the instances through the single-GPU batched entry point, and one
all-gather at the end assembles the full result on every rank. No reference
counterpart (the reference drives one GPU; its multi-GPU partitioning scaffolding,
GASengine/csr_problem.cuh:339-365, is unused).

With the NCCL backend the gather runs on device tensors; with gloo (CPU tests) on
host tensors. Slices are padded to the largest one so that every rank sends the
same number of rows, as all-gather needs.
"""
from __future__ import annotations

import numpy as np


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous slice [lo, hi) of `total` instances owned by `rank`: the first
    total % world ranks get one instance more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(int(total), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_rows(local: np.ndarray, total: int, group=None) -> np.ndarray:
    """All-gathers row slices (rank r holds rows shard_range(total, r, world))
    into the full `total x row` array on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_range(total, rank, world)
    local = np.asarray(local)
    if local.shape[0] != hi - lo:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, owns {hi - lo}")
    width = local.shape[1:]
    most = -(-int(total) // world)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    pad = torch.zeros((most,) + tuple(width), dtype=torch.from_numpy(local[:0].copy()).dtype, device=dev)
    pad[: hi - lo] = torch.from_numpy(np.ascontiguousarray(local)).to(dev)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    rows = []
    for r in range(world):
        a, b = shard_range(total, r, world)
        rows.append(parts[r][: b - a].cpu().numpy())
    return np.concatenate(rows, axis=0)


def bfs_batch_sharded(graph, srcs, group=None, **kw) -> np.ndarray:
    """Depth rows (len(srcs) x n) of a multi-source BFS with the sources split
    over the ranks; every rank returns the full array."""
    import torch.distributed as dist

    srcs = np.asarray(srcs, dtype=np.int32)
    lo, hi = shard_range(srcs.size, dist.get_rank(group), dist.get_world_size(group))
    local = graph.bfs_batch(srcs[lo:hi], **kw)[0] if hi > lo else np.zeros((0, graph.n), np.int32)
    return gather_rows(local, srcs.size, group)


def sssp_batch_sharded(graph, srcs, group=None, **kw) -> np.ndarray:
    """Distance rows (len(srcs) x n) with the sources split over the ranks."""
    import torch.distributed as dist

    srcs = np.asarray(srcs, dtype=np.int32)
    lo, hi = shard_range(srcs.size, dist.get_rank(group), dist.get_world_size(group))
    local = graph.sssp_batch(srcs[lo:hi], **kw)[0] if hi > lo else np.zeros((0, graph.n), np.int32)
    return gather_rows(local, srcs.size, group)


def pagerank_sharded(graph, teleport: np.ndarray, group=None, **kw) -> np.ndarray:
    """Personalised PageRank rows (nvec x n) with the teleport vectors split over
    the ranks (each rank runs its slice as one batched solve)."""
    import torch.distributed as dist

    teleport = np.asarray(teleport, dtype=np.float32)
    nvec = teleport.shape[0]
    lo, hi = shard_range(nvec, dist.get_rank(group), dist.get_world_size(group))
    kw.setdefault("mode", "normalized")
    if hi - lo == 0:
        local = np.zeros((0, graph.n), np.float32)
    else:
        x, _ = graph.pagerank(teleport=np.ascontiguousarray(teleport[lo:hi]), nvec=hi - lo, **kw)
        local = np.asarray(x).reshape(hi - lo, graph.n)
    return gather_rows(local, nvec, group)
