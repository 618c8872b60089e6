"""Sharding of a graph database over processes (one per GPU).

A graph database is a union of independent graphs, so every rank can hold a
contiguous range of them and match / mine locally; the only exchange is the
per-level sum of candidate supports and embedding counts when mining (a
pattern's support is the number of graphs holding it, and every graph lives
on exactly one rank).  The reference runs on one GPU only.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np

from .workloads import GraphDB


def graph_range(num_graphs: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced [g0, g1) of graph ids for `rank`."""
    if not 0 <= rank < world:
        raise ValueError("rank outside world")
    base, extra = divmod(num_graphs, world)
    g0 = rank * base + min(rank, extra)
    return g0, g0 + base + (1 if rank < extra else 0)


def shard_database(db: GraphDB, rank: int, world: int) -> GraphDB:
    """The graphs of `rank`, renumbered to vertex ids 1..V_r (edges kept)."""
    G = len(db.first) - 1
    g0, g1 = graph_range(G, rank, world)
    v0, v1 = int(db.first[g0]), int(db.first[g1])  # vertex ids [v0, v1)
    keep = (db.src >= v0) & (db.src < v1)
    shift = v0 - 1
    vl = np.zeros(v1 - v0 + 1, dtype=np.uint32)
    vl[1:] = db.vlabels[v0:v1]
    return GraphDB(f"{db.name}[{rank}/{world}]", vl, (db.src[keep] - shift).astype(np.uint32),
                   (db.dst[keep] - shift).astype(np.uint32), db.elabels[keep].copy(),
                   (db.first[g0:g1 + 1] - shift).astype(np.int64), dict(db.params, shard=(rank, world, g0, g1)))


class SupportReducer:
    """gva_mine reduce hook: sums each level's supports and embedding counts
    over a torch.distributed process group (NCCL tensors on the current CUDA
    device, gloo tensors on the CPU)."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        backend = dist.get_backend(group)
        self.device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        self.calls = 0

    def __call__(self, supports: np.ndarray, embeddings: np.ndarray) -> None:
        import torch
        n = len(supports)
        t = torch.empty(2 * n, dtype=torch.int64)
        t[:n] = torch.from_numpy(supports.astype(np.int64))
        t[n:] = torch.from_numpy(embeddings.astype(np.int64))
        t = t.to(self.device)
        self.dist.all_reduce(t, group=self.group)
        t = t.cpu().numpy()
        supports[:] = t[:n].astype(np.uint32)
        embeddings[:] = t[n:].astype(np.uint64)
        self.calls += 1
