"""Multi-process path on CPU: graph-database sharding and the per-level
support reduction (geneva_b200.shard) over a world-size-2 gloo group.

Each rank counts pattern supports on its own shard (brute force stands in
for the GPU matcher, which these ranks do not have); SupportReducer sums
them; the result must equal the counts on the whole database.
"""
import os
import socket

import numpy as np
import pytest

from geneva_b200 import workloads
from geneva_b200.shard import graph_range, shard_database


def test_graph_range_partitions_exactly():
    for G in (1, 2, 7, 100, 20000):
        for world in (1, 2, 3, 8):
            spans = [graph_range(G, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == G
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def test_shard_database_keeps_every_graph():
    db = workloads.graph_database(50, 5, 12, 2.5, 3, None, 2, seed=9, name="t")
    parts = [shard_database(db, r, 3) for r in range(3)]
    assert sum(len(p.first) - 1 for p in parts) == 50
    assert sum(p.num_edges for p in parts) == db.num_edges
    assert sum(p.num_vertices for p in parts) == db.num_vertices
    for p in parts:
        assert p.first[0] == 1 and p.first[-1] == p.num_vertices + 1
        assert p.src.min() >= 1 and max(p.src.max(), p.dst.max()) <= p.num_vertices
        g = p.graph_of(p.src.astype(np.int64))
        assert np.array_equal(g, p.graph_of(p.dst.astype(np.int64)))  # no edge crosses graphs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    from brute_miner import mine as brute_mine
    from geneva_b200.shard import SupportReducer
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    db = workloads.graph_database(60, 5, 10, 2.5, 3, None, 2, seed=17, name="t")
    whole = brute_mine(db, 2, 1)                       # every pattern with its support
    codes = sorted(whole)
    local = brute_mine(shard_database(db, rank, world), 2, 1)
    sup = np.array([local.get(c, 0) for c in codes], dtype=np.uint32)
    emb = np.arange(len(codes), dtype=np.uint64) * (rank + 1)
    red = SupportReducer()
    red(sup, emb)
    if rank == 0:
        ok = all(int(s) == whole[c] for s, c in zip(sup, codes))
        ok &= bool(np.array_equal(emb, np.arange(len(codes), dtype=np.uint64) * sum(range(1, world + 1))))
        with open(out_path, "w") as f:
            f.write("ok" if ok and red.calls == 1 else "mismatch")
    dist.barrier()
    dist.destroy_process_group()


def test_support_reduction_over_gloo(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    out = tmp_path / "result.txt"
    mp.spawn(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    assert out.read_text() == "ok"
