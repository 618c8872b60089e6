"""Batched engine (gva_batch_count) against the plain path and the oracle."""
import random

import numpy as np
import pytest

import geneva_b200 as gv
from geneva_b200 import workloads
from querygen import random_query

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_db(native, oracle):
    db = workloads.graph_database(300, 10, 30, 3.0, 4, None, 2, seed=77, name="small")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    yield db, gdb, og
    oracle.free(og)
    gdb.close()


def _patterns(db, n, seed):
    pats = workloads.sample_patterns(db, n, 3, 6, seed=seed)
    rng = random.Random(seed)
    pats += [random_query(rng) for _ in range(n // 4)]
    return pats


def test_batch_counts_match_plain_and_oracle(small_db, oracle):
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 80, 5) if oracle.count(og, p, cap_rows=1_000_000) is not None]
    plans = [gv.Plan.from_text(p) for p in pats]
    counts, _, stats = gv.batch_count(gdb, plans)
    assert stats["rounds"] >= 2
    for p, plan, c in zip(pats, plans, counts):
        assert int(c) == oracle.count(og, p), p
        assert int(c) == gv.match(gdb, plan, count_only=True).num_rows, p
    # single-vertex plans give the same counts
    sv = [gv.Plan.from_text(p, gv.MODE_SV) for p in pats]
    counts_sv, _, _ = gv.batch_count(gdb, sv)
    assert np.array_equal(counts, counts_sv)


def test_per_graph_counts_and_support(small_db, oracle):
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 40, 9) if oracle.count(og, p, cap_rows=500_000) is not None]
    plans = [gv.Plan.from_text(p) for p in pats]
    counts, (gc, sup), _ = gv.batch_count(gdb, plans, graph_counts=True, support=True)
    G = len(db.first) - 1
    assert gc.shape == (len(pats), G)
    for i, p in enumerate(pats):
        rows, _ = oracle.match(og, p)
        g = db.graph_of(rows[:, 0].astype(np.int64)) if rows.size else np.zeros(0, dtype=np.int64)
        want = np.bincount(g, minlength=G).astype(np.uint64)
        assert np.array_equal(gc[i], want), p
        assert int(sup[i]) == int((want > 0).sum()), p
        assert int(counts[i]) == int(want.sum())


def test_small_budget_splits_tasks(small_db, oracle):
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 30, 13) if oracle.count(og, p, cap_rows=500_000) is not None]
    plans = [gv.Plan.from_text(p) for p in pats]
    full, _, s_full = gv.batch_count(gdb, plans)
    tiny, _, s_tiny = gv.batch_count(gdb, plans, budget_bytes=2048)
    assert np.array_equal(full, tiny)
    assert s_tiny["splits"] > 0 and s_tiny["rounds"] > s_full["rounds"]


def test_shared_prefixes_and_duplicates(small_db, oracle):
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 20, 21) if oracle.count(og, p, cap_rows=500_000) is not None]
    plans = [gv.Plan.from_text(p) for p in pats] * 3  # every plan three times
    counts, (gc, sup), stats = gv.batch_count(gdb, plans, graph_counts=True, support=True)
    n = len(pats)
    for i in range(n):
        assert counts[i] == counts[i + n] == counts[i + 2 * n] == oracle.count(og, pats[i])
        assert np.array_equal(gc[i], gc[i + 2 * n]) and sup[i] == sup[i + n]
    single, _, s1 = gv.batch_count(gdb, plans[:n])
    assert stats["trie_nodes"] == s1["trie_nodes"]  # duplicates add no work
    assert np.array_equal(single, counts[:n])


def test_enron_batch(native, enron_dir):
    db = gv.loadDataBase(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    q = (enron_dir / "Enron_4_6_0.query").read_text()
    plans = [gv.Plan.from_text(q), gv.Plan.from_text(q, gv.MODE_SV), gv.Plan.from_text("v 0 1\nv 1 9\ne 0 1 1\n")]
    counts, _, _ = gv.batch_count(db, plans)
    assert counts.tolist() == [157502, 157502, 0]
    with pytest.raises(gv.GenevaError):
        gv.batch_count(db, plans, support=True)  # no graph ids declared
    db.close()


@pytest.mark.parametrize("rows_per_item,hub", [(32, 0), (64, 0), (128, 1), (64, 1 << 30), (32, 5), (128, 32)])
def test_launch_shapes_give_the_oracle_counts(small_db, oracle, rows_per_item, hub):
    """Every launch shape of the round kernels counts (and writes the
    intermediate frontiers of) the same rows: hub 0 sends every row's
    candidates through the warp-shared path, 1 << 30 none."""
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 60, 21) if oracle.count(og, p, cap_rows=1_000_000) is not None]
    plans = [gv.Plan.from_text(p) for p in pats]
    keep = gdb.tuning
    try:
        gdb.set_tuning(rows_per_item, hub)
        assert {k: gdb.tuning[k] for k in ("rows_per_item", "hub")} == {"rows_per_item": rows_per_item, "hub": hub}
        counts, (gc, sup), _ = gv.batch_count(gdb, plans, graph_counts=True, support=True)
    finally:
        gdb.set_tuning(keep["rows_per_item"], keep["hub"])
    want_counts, want_sup, want_gc = oracle.many_graph_counts(og, pats, db.first)
    assert np.array_equal(counts, want_counts)
    assert np.array_equal(sup, want_sup)
    for i in range(len(pats)):
        assert np.array_equal(gc[i], want_gc[i]), pats[i]


def test_autotune_keeps_a_valid_shape(small_db, oracle):
    db, gdb, og = small_db
    pats = workloads.sample_patterns(db, 200, 3, 6, seed=31)
    plans = gv.Plan.batch_from_texts(pats)
    t = gdb.autotune(plans)
    assert t["rows_per_item"] in (32, 64, 128) and t["shapes_tried"] == 12
    assert 0 < t["ms"] <= t["default_ms"]
    assert {k: gdb.tuning[k] for k in ("rows_per_item", "hub")} == {"rows_per_item": t["rows_per_item"], "hub": t["hub"]}
    counts, _, _ = gv.batch_count(gdb, plans)
    want, _, _ = oracle.many_graph_counts(og, pats, db.first)
    assert np.array_equal(counts, want)


def test_hub_vertices_of_the_packed_segment_index(native, oracle):
    """Vertices with more than 255 neighbours in a partition take the packed
    index's wide records (a row of cumulative words instead of bytes): a
    graph with a few such hubs, matched through the batched and the plain
    path, against the oracle (counts per graph, supports, rows)."""
    rng = np.random.default_rng(5)
    V = 3000
    vl = np.zeros(V + 1, dtype=np.uint32)
    vl[1:] = rng.integers(1, 6, size=V)
    edges = set()
    for hub in (1, 2, 3):
        for w in rng.choice(np.arange(4, V + 1), size=700, replace=False):
            edges.add((hub, int(w), 1 + (int(w) % 2)))
    while len(edges) < 2100 + 6000:
        a, b = (int(x) for x in rng.integers(1, V + 1, size=2))
        if a != b:
            edges.add((min(a, b), max(a, b), int(rng.integers(1, 3))))
    e = np.array(sorted(edges), dtype=np.uint32)
    first = np.array([1, V + 1], dtype=np.int64)
    gdb = gv.Database.from_edges(vl, e[:, 0], e[:, 1], e[:, 2])
    gdb.set_graphs(first)
    og = oracle.from_edges(vl, e[:, 0], e[:, 1], e[:, 2])
    pats = ["v 0 %d\nv 1 %d\nv 2 %d\ne 0 1 1\ne 0 2 %d\n" % (int(vl[1]), a, b, el)
            for a in (1, 3) for b in (2, 4) for el in (1, 2)]
    pats += ["v 0 %d\nv 1 %d\nv 2 %d\nv 3 %d\ne 0 1 1\ne 1 2 2\ne 0 2 1\ne 2 3 %d\n" % (int(vl[2]), a, b, c, el)
             for a in (1, 2) for b in (3, 5) for c in (1, 4) for el in (1, 2)]
    pats = [p for p in pats if oracle.count(og, p, cap_rows=3_000_000) is not None]
    assert len(pats) >= 10
    plans = [gv.Plan.from_text(p) for p in pats]
    counts, sup, _ = gv.batch_count(gdb, plans, support=True)
    want, want_sup, _ = oracle.many_graph_counts(og, pats, first)
    assert np.array_equal(counts, want) and np.array_equal(sup, want_sup)
    from oracle_lib import rows_digest
    for p, plan in list(zip(pats, plans))[:8]:
        got = gv.match(gdb, plan).rows()
        rows, _ = oracle.match(og, p)
        assert rows_digest(got) == rows_digest(rows), p
    oracle.free(og)
    gdb.close()


def test_batch_count_texts_equals_planned_batch(small_db, oracle):
    """gva_batch_count_texts (texts read and planned inside the call) gives the
    counts of gva_batch_count over planned handles, in DV and SV mode; a text
    the planner rejects fails alone (count 0, its status), after the others
    were counted."""
    import ctypes
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 120, 41) if oracle.count(og, p, cap_rows=1_000_000) is not None]
    for mode in (gv.MODE_DV, gv.MODE_SV):
        plans = [gv.Plan.from_text(p, mode) for p in pats]
        want, (wgc, wsup), _ = gv.batch_count(gdb, plans, graph_counts=True, support=True)
        got, (gc, sup), st = gv.batch_count_texts(gdb, pats, mode=mode, graph_counts=True, support=True)
        assert np.array_equal(got, want) and np.array_equal(gc, wgc) and np.array_equal(sup, wsup)
        assert st["trie_nodes"] > 0
    bad = list(pats[:5]) + ["v 0 1\nv 1 1\ne 0 0 1\n", "v 0 1\nv 2 1\ne 0 2 1\n", "v 0 1\nv 1 2\n"] + list(pats[5:10])
    lib = gv.library()
    n = len(bad)
    arr = (ctypes.c_char_p * n)(*[t.encode() for t in bad])
    counts = np.zeros(n, dtype=np.uint64)
    status = np.zeros(n, dtype=np.int32)
    o = gv._BatchOpts(None, 0, 0, 0)
    rc = lib.gva_batch_count_texts(gdb._h, ctypes.cast(arr, ctypes.c_void_p), n, gv.MODE_DV, ctypes.byref(o),
                                   counts.ctypes.data, None, None, status.ctypes.data, None)
    assert rc != 0 and b"query 5" in lib.gva_last_error()
    assert list(status[5:8]) == [6, 2, 2]  # self-loop, ids not 0..n-1, no edges
    want = [oracle.count(og, t) for t in pats[:10]]
    assert [int(c) for i, c in enumerate(counts) if i not in (5, 6, 7)] == want
    assert int(counts[5]) == int(counts[6]) == int(counts[7]) == 0


def test_device_rounds_match_host_rounds(small_db, oracle):
    """Rounds scheduled on the device (a planning kernel per round, every
    round launched at once) give the counts, per-graph counts and supports of
    rounds scheduled on the host, and the oracle's counts."""
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 160, 31) if oracle.count(og, p, cap_rows=1_000_000) is not None]
    for mode in (gv.MODE_DV, gv.MODE_SV):
        plans = [gv.Plan.from_text(p, mode) for p in pats]
        dc, (dgc, dsup), ds = gv.batch_count(gdb, plans, graph_counts=True, support=True)
        hc, (hgc, hsup), hs = gv.batch_count(gdb, plans, graph_counts=True, support=True, host_rounds=True)
        assert ds["device_rounds"] == ds["rounds"] > 0
        assert hs["device_rounds"] == 0 and hs["rounds"] > 0
        assert np.array_equal(dc, hc) and np.array_equal(dgc, hgc) and np.array_equal(dsup, hsup)
        for p, c in zip(pats, dc):
            assert int(c) == oracle.count(og, p), p


def test_device_rounds_overflow_falls_back_to_host(native, oracle):
    """A round whose output outgrows its frontier region makes the run start
    over with host-scheduled rounds (same results) and doubles the region for
    later runs."""
    rng = np.random.default_rng(5)
    V = 3000
    vl = np.zeros(V + 1, dtype=np.uint32)
    vl[1:] = rng.integers(1, 3, size=V)
    edges = set()
    while len(edges) < 30000:
        a, b = (int(x) for x in rng.integers(1, V + 1, size=2))
        if a != b:
            edges.add((min(a, b), max(a, b), 1))
    e = np.array(sorted(edges), dtype=np.uint32)
    gdb = gv.Database.from_edges(vl, e[:, 0], e[:, 1], e[:, 2])
    og = oracle.from_edges(vl, e[:, 0], e[:, 1], e[:, 2])
    pats = ["v 0 %d\nv 1 %d\nv 2 %d\ne 0 1 1\ne 1 2 1\n" % (a, b, c) for a in (1, 2) for b in (1, 2) for c in (1, 2)]
    pats += ["v 0 1\nv 1 2\nv 2 1\nv 3 2\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 3 0 1\n",  # a 4-cycle
             "v 0 1\nv 1 2\nv 2 1\nv 3 2\ne 0 1 1\ne 1 2 1\ne 2 3 1\n",  # a 3-edge path
             "v 0 1\nv 1 2\nv 2 2\nv 3 1\ne 0 1 1\ne 0 2 1\ne 0 3 1\n"]  # a 3-edge star
    checked = len(pats)
    # a 5-edge path: its written prefixes (up to millions of rows of 5
    # columns) outgrow a 1 MiB region, and fit two of 1 GiB
    pats += ["v 0 1\nv 1 2\nv 2 1\nv 3 2\nv 4 1\nv 5 2\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 3 4 1\ne 4 5 1\n"]
    plans = [gv.Plan.from_text(p) for p in pats]
    want, _, hs = gv.batch_count(gdb, plans, host_rounds=True)
    assert [int(c) for c in want[:checked]] == [oracle.count(og, p) for p in pats[:checked]]
    t = gdb.tuning
    try:
        gdb.set_tuning(t["rows_per_item"], t["hub"], round_region_mb=1)
        got, _, s = gv.batch_count(gdb, plans)
        assert s["device_rounds"] == 0 and s["rounds"] > 0
        assert gdb.tuning["round_region_mb"] == 2
        assert np.array_equal(got, want)
        gdb.set_tuning(t["rows_per_item"], t["hub"], round_region_mb=1024)
        got, _, s = gv.batch_count(gdb, plans)
        assert s["device_rounds"] == s["rounds"] > 0
        assert np.array_equal(got, want)
    finally:
        gdb.set_tuning(t["rows_per_item"], t["hub"], round_region_mb=t["round_region_mb"])
    oracle.free(og)
    gdb.close()


def test_split_runs_schedule_on_the_host_unless_asked(small_db, oracle):
    """A run of 12,288 plans or more runs as two halves, scheduled on the host
    by default; GVA_BATCH_DEVICE_ROUNDS schedules the same halves on the
    device, with the same results; the two flags together are refused."""
    import ctypes
    db, gdb, og = small_db
    pats = [p for p in _patterns(db, 120, 43) if oracle.count(og, p, cap_rows=1_000_000) is not None]
    reps = 12288 // len(pats) + 1
    plans = gv.Plan.batch_from_texts(pats * reps)
    hc, hs, hst = gv.batch_count(gdb, plans, support=True)
    dc, ds, dst = gv.batch_count(gdb, plans, support=True, device_rounds=True)
    assert hst["device_rounds"] == 0 and dst["device_rounds"] > 0
    assert np.array_equal(hc, dc) and np.array_equal(hs, ds)
    assert [int(c) for c in hc[:len(pats)]] == [oracle.count(og, p) for p in pats]
    o = gv._BatchOpts(None, 0, 0, gv.BATCH_HOST_ROUNDS | gv.BATCH_DEVICE_ROUNDS)
    counts = np.zeros(len(plans), dtype=np.uint64)
    arr = gv._plan_handles(plans)
    rc = gv.library().gva_batch_count(gdb._h, arr.ctypes.data, len(plans), ctypes.byref(o), counts.ctypes.data,
                                      None, None, None)
    assert rc != 0 and b"exclude each other" in gv.library().gva_last_error()
