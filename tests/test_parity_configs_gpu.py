"""Parity at the benchmark configurations' full sizes, through the C ABI.

* 4,096 query patterns of 3-8 vertices (connected induced subgraphs of the
  1,000-graph database's graphs) counted in one batched run: the int64
  embedding count of every (query, graph) pair and every query's support
  against the oracle (cpumine restated, rows mapped to graph ids).
* Mining the 1,000-graph database (patterns up to 4 edges, support >= 5 %):
  the frequent-pattern set and supports against a brute-force miner that
  enumerates every connected edge subset of every graph, and every frequent
  pattern's embedding count against the oracle.
* The 20,000-graph database: the seeded pattern list the benchmark matches
  (its first 1,024 patterns) counted in one batched run against the oracle
  (counts and supports), and a seeded sample of the patterns mined from it
  (up to 6 edges, support >= 2 %) against the oracle's supports and counts.

Integer results: compared exactly.
"""
import numpy as np
import pytest

import geneva_b200 as gv
from brute_miner import build_native, mine_native, pattern_from_text
from geneva_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config1(native, oracle):
    db = workloads.config1(seed=1)
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    yield db, gdb, og
    oracle.free(og)
    gdb.close()


@pytest.fixture(scope="module")
def config2(native, oracle):
    db = workloads.config2(seed=2)
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    yield db, gdb, og
    oracle.free(og)
    gdb.close()


def test_config3_all_queries_per_graph_counts(config1, oracle):
    db, gdb, og = config1
    queries = workloads.config3_queries(db, 4096, seed=1000)
    plans = gv.Plan.batch_from_texts(queries)
    counts, (gc, sup), _ = gv.batch_count(gdb, plans, graph_counts=True, support=True)
    want_counts, want_sup, want_gc = oracle.many_graph_counts(og, queries, db.first)
    assert np.array_equal(counts, want_counts)
    assert np.array_equal(sup, want_sup)
    bad = [i for i in range(len(queries)) if not np.array_equal(gc[i], want_gc[i])]
    assert not bad, f"{len(bad)} queries differ per graph, first: {queries[bad[0]]!r}"
    assert (counts > 0).all()  # induced subgraphs of the database: every query occurs


def test_config1_mining_equals_brute_force(config1, oracle, tmp_path):
    db, gdb, og = config1
    minsup = 50  # 5 % of 1,000 graphs
    pats, stats = gv.mine(gdb, 4, minsup)
    got = {pattern_from_text(p.text): p.support for p in pats}
    want = mine_native(db, 4, minsup, build_native(tmp_path), tmp_path)
    assert len(got) == len(pats)  # no pattern mined twice
    assert got == want
    assert stats["frequent"] == len(pats)
    texts = [p.text for p in pats]
    want_counts, want_sup, _ = oracle.many_graph_counts(og, texts, db.first)
    assert np.array_equal(np.array([p.embeddings for p in pats], dtype=np.uint64), want_counts)
    assert np.array_equal(np.array([p.support for p in pats], dtype=np.uint32), want_sup)


def test_config2_pattern_list_counts_and_supports(config2, oracle):
    db, gdb, og = config2
    queries = workloads.config2_patterns(db)[:1024]
    plans = gv.Plan.batch_from_texts(queries)
    counts, sup, _ = gv.batch_count(gdb, plans, support=True)
    want_counts, want_sup, _ = oracle.many_graph_counts(og, queries, db.first)
    assert np.array_equal(counts, want_counts)
    assert np.array_equal(sup, want_sup)
    # the plain per-query path agrees on a slice
    for q, p, c in list(zip(queries, plans, counts))[:64]:
        assert gv.match(gdb, p, count_only=True).num_rows == int(c), q


def test_config2_mined_patterns_against_oracle(config2, oracle):
    db, gdb, og = config2
    minsup = 400  # 2 % of 20,000 graphs
    pats, stats = gv.mine(gdb, 6, minsup)
    assert len(pats) == stats["frequent"] > 1000
    rng = np.random.default_rng(7)
    pick = sorted(rng.choice(len(pats), 400, replace=False).tolist())
    texts = [pats[i].text for i in pick]
    want_counts, want_sup, _ = oracle.many_graph_counts(og, texts, db.first)
    got_counts = np.array([pats[i].embeddings for i in pick], dtype=np.uint64)
    got_sup = np.array([pats[i].support for i in pick], dtype=np.uint32)
    assert np.array_equal(got_counts, want_counts)
    assert np.array_equal(got_sup, want_sup)
    assert (got_sup >= minsup).all()
    # every pattern's text is distinct up to isomorphism (canonical dedupe)
    edges = np.array([p.edges for p in pats])
    small = [pats[i].text for i in np.nonzero(edges <= 3)[0]]
    assert len({pattern_from_text(t) for t in small}) == len(small)
