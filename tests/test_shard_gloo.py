"""Multi-process path on CPU: graph-database sharding and the per-level
support reduction (geneva_b200.shard) over a world-size-2 gloo group.

Each rank counts pattern supports on its own shard (brute force or the oracle
stand in for the GPU matcher, which these ranks do not have); SupportReducer
sums them; the result must equal the counts on the whole database.  The
second test drives the miner's own level loop (gva_mine_host: the loop
gva_mine runs, with its reduce hook) on both ranks: every level's candidates
must be the same on both ranks and the mined patterns those of one process
holding the whole database.
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


def _oracle_eval(oracle, og, db, seen):
    """Evaluator of a rank: supports and embedding counts of the candidates on
    this rank's graphs, by the oracle; records every level's candidates."""
    def ev(texts):
        seen.append(list(texts))
        c, sup, _ = oracle.many_graph_counts(og, texts, db.first, threads=2)
        return sup, c
    return ev


def _level_loop_rank(rank, world, port, out_dir):
    import json
    import torch.distributed as dist
    import geneva_b200 as gv
    from geneva_b200.shard import SupportReducer
    from oracle_lib import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    db = workloads.graph_database(80, 5, 12, 2.8, 3, None, 2, seed=23, name="t")
    part = shard_database(db, rank, world)
    oracle = Oracle.get()
    og = oracle.from_edges(part.vlabels, part.src, part.dst, part.elabels)
    seen = []
    labels = np.unique(db.vlabels[1:])  # every rank mines over the database's labels
    pats, st = gv.mine_host(labels, 2, 4, 6, _oracle_eval(oracle, og, part, seen), reduce=SupportReducer(),
                            host_threads=2)
    oracle.free(og)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"levels": seen, "patterns": [[p.text, p.support, p.embeddings] for p in pats],
                   "candidates": st["candidates"]}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_mining_level_loop_over_gloo(tmp_path):
    import json
    import geneva_b200 as gv
    from brute_miner import mine as brute_mine, pattern_from_text
    from oracle_lib import Oracle
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(_level_loop_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    # both ranks evaluated the same candidates, level by level, and took the same decisions
    assert r0["levels"] == r1["levels"] and len(r0["levels"]) >= 3
    assert r0["patterns"] == r1["patterns"]
    # and those of one process holding every graph
    db = workloads.graph_database(80, 5, 12, 2.8, 3, None, 2, seed=23, name="t")
    oracle = Oracle.get()
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    seen = []
    pats, _ = gv.mine_host(np.unique(db.vlabels[1:]), 2, 4, 6, _oracle_eval(oracle, og, db, seen), host_threads=2)
    oracle.free(og)
    assert seen == r0["levels"]
    assert [[p.text, p.support, p.embeddings] for p in pats] == r0["patterns"]
    # embedding counts summed through the reduce hook (uint64 through int64) equal the whole database's
    want = brute_mine(db, 4, 6)
    assert {pattern_from_text(t): s for t, s, _ in r0["patterns"]} == want
