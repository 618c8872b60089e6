"""Mining layer (gva_mine) against a brute-force miner and the oracle."""
import numpy as np
import pytest

import geneva_b200 as gv
from geneva_b200 import workloads
from brute_miner import mine as brute_mine, pattern_from_text

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("max_edges,minsup,vl,el", [(3, 8, 3, 1), (4, 15, 4, 1), (3, 6, 3, 2)])
def test_mined_patterns_equal_brute_force(native, max_edges, minsup, vl, el):
    db = workloads.graph_database(120, 6, 12, 2.6, vl, None, el, seed=300 + max_edges * 7 + vl, name="tiny")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    pats, stats = gv.mine(gdb, max_edges, minsup)
    got = {pattern_from_text(p.text): p.support for p in pats}
    want = brute_mine(db, max_edges, minsup)
    assert got == want
    assert stats["frequent"] == len(pats) and stats["candidates"] >= len(pats)
    assert max(p.edges for p in pats) <= max_edges
    gdb.close()


def test_mined_supports_match_oracle_rows(native, oracle):
    db = workloads.graph_database(150, 8, 16, 3.0, 3, None, 2, seed=41, name="tiny2")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    pats, _ = gv.mine(gdb, 3, 10)
    assert len(pats) > 10
    for p in pats[:: max(1, len(pats) // 25)]:
        rows, _ = oracle.match(og, p.text)
        graphs = np.unique(db.graph_of(rows[:, 0].astype(np.int64))) if rows.size else []
        assert p.support == len(graphs), p.text
        assert p.embeddings == rows.shape[0], p.text
    oracle.free(og)
    gdb.close()


def test_mining_small_batches_give_same_result(native):
    db = workloads.graph_database(100, 6, 14, 3.0, 3, None, 2, seed=5, name="tiny3")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    a, _ = gv.mine(gdb, 3, 5)
    b, _ = gv.mine(gdb, 3, 5, batch_limit=7, budget_bytes=1 << 16)
    key = lambda ps: sorted((p.text, p.support, p.embeddings) for p in ps)
    assert key(a) == key(b)
    gdb.close()


def test_mining_with_more_than_256_labels(native):
    # canonical codes switch to 2-byte values past 256 vertex labels
    db = workloads.graph_database(200, 6, 12, 2.8, 1000, 1.0, 2, seed=77, name="manylabels")
    assert len(np.unique(db.vlabels)) > 256
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    pats, _ = gv.mine(gdb, 3, 3)
    got = {pattern_from_text(p.text): p.support for p in pats}
    assert got == brute_mine(db, 3, 3) and len(got) > 0
    gdb.close()


def test_mining_cancel_flag(native):
    """A set cancel flag stops a run at its first batch boundary with status 7."""
    import ctypes
    db = workloads.graph_database(100, 6, 14, 3.0, 3, None, 2, seed=5, name="tiny4")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    flag = ctypes.c_int(1)
    with pytest.raises(gv.GenevaError) as e:
        gv.mine(gdb, 3, 5, cancel=flag)
    assert e.value.status == 7
    with pytest.raises(gv.GenevaError) as e:
        gv.mine(gdb, 3, 5, support="mni", cancel=flag)
    assert e.value.status == 7
    flag.value = 0
    pats, _ = gv.mine(gdb, 3, 5, cancel=flag)  # unset: runs to completion
    assert len(pats) > 0
    gdb.close()
