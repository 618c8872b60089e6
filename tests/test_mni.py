"""Single-graph MNI support (gva_mni_support, gva_mine with GVA_SUPPORT_MNI)
against the oracle's cpumine rows and a brute-force image-set miner."""
import random

import numpy as np
import pytest

import geneva_b200 as gv
from geneva_b200 import workloads
from brute_miner import pattern_from_text
from mni_oracle import brute_mni_mine, mni_from_rows


def code_text(code) -> str:
    n = code[0]
    labels = code[1:1 + n]
    adj = code[1 + n:]
    lines = [f"v {i} {labels[i]}" for i in range(n)]
    k = 0
    for i in range(n):
        for j in range(i + 1, n):
            if adj[k]:
                lines.append(f"e {i} {j} {adj[k]}")
            k += 1
    return "\n".join(lines) + "\n"


def tiny_graph(seed=3):
    return workloads.rmat_graph(6, 150, 3, None, seed=seed, name="tiny_rmat")


def small_graph(seed=5):
    return workloads.rmat_graph(9, 2500, 4, 1.0, seed=seed, name="small_rmat")


@pytest.fixture(scope="module")
def tiny_brute():
    db = tiny_graph()
    return db, brute_mni_mine(db, 3)


def test_rmat_generator_shape():
    db = workloads.rmat_graph(10, 5000, 8, 1.0, seed=1)
    assert db.num_vertices == 1024 and db.num_edges == 5000
    assert (db.src != db.dst).all() and db.src.min() >= 1 and max(db.src.max(), db.dst.max()) <= 1024
    keys = np.minimum(db.src, db.dst).astype(np.uint64) << np.uint64(32) | np.maximum(db.src, db.dst)
    assert len(np.unique(keys)) == 5000
    deg = np.bincount(np.concatenate([db.src, db.dst]), minlength=1025)[1:]
    assert deg.max() > 8 * deg.mean()  # skewed
    again = workloads.rmat_graph(10, 5000, 8, 1.0, seed=1)
    assert np.array_equal(again.src, db.src) and np.array_equal(again.vlabels, db.vlabels)


def test_oracle_rows_agree_with_brute_force(oracle, tiny_brute):
    """The two CPU oracles (cpumine rows + orbit union; edge-subset images) agree."""
    db, want = tiny_brute
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    codes = sorted(want)
    assert len(codes) > 30
    for code in codes[:: max(1, len(codes) // 60)]:
        text = code_text(code)
        assert mni_from_rows(oracle, og, text) == want[code], text
    oracle.free(og)


def test_cpu_mni_search_agrees_with_brute_force(oracle, tiny_brute):
    """The oracle's CPU existence search (the CPU baseline of the single-graph
    configuration) against the edge-subset images, exact and capped."""
    db, want = tiny_brute
    mg = oracle.mni_graph(db.vlabels, db.src, db.dst, db.elabels)
    codes = sorted(want)
    for code in codes[:: max(1, len(codes) // 80)]:
        text = code_text(code)
        assert oracle.mni(mg, text)[0] == want[code], text
        assert oracle.mni(mg, text, cap=3)[0] == min(want[code], 3), text
    oracle.mni_graph_free(mg)


@pytest.mark.gpu
@pytest.mark.parametrize("plain", [False, True])
def test_mni_exact_matches_oracle(native, oracle, plain):
    db = small_graph()
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    pats = workloads.sample_patterns(db, 40, 2, 5, seed=11)
    pats = [p for p in pats if oracle.count(og, p, cap_rows=2_000_000) is not None]
    assert len(pats) >= 20
    sup, st = gv.mni_support(gdb, pats, cap=0, plain=plain, profile=True)
    mg = oracle.mni_graph(db.vlabels, db.src, db.dst, db.elabels)
    for p, s in zip(pats, sup):
        assert int(s) == mni_from_rows(oracle, og, p), p
        assert int(s) == oracle.mni(mg, p)[0], p
    oracle.mni_graph_free(mg)
    assert st["tasks"] >= len(pats) and st["kernel"]["launches"] >= 1
    oracle.free(og)
    gdb.close()


@pytest.mark.gpu
def test_mni_capped_and_absent(native, oracle):
    db = small_graph()
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    pats = workloads.sample_patterns(db, 24, 2, 4, seed=12)
    exact = [mni_from_rows(oracle, og, p) for p in pats]
    for cap in (1, 7, 40):
        sup, _ = gv.mni_support(gdb, pats, cap=cap)
        assert [int(x) for x in sup] == [min(e, cap) for e in exact]
        sup_p, _ = gv.mni_support(gdb, pats, cap=cap, plain=True)
        assert np.array_equal(sup, sup_p)
    # a label the graph lacks, an edge label it lacks, a single vertex
    odd = ["v 0 1\nv 1 99\ne 0 1 1\n", "v 0 1\nv 1 2\ne 0 1 7\n", "v 0 2\n"]
    sup, _ = gv.mni_support(gdb, odd)
    assert int(sup[0]) == 0 and int(sup[1]) == 0
    assert int(sup[2]) == int((db.vlabels[1:] == 2).sum())
    with pytest.raises(gv.GenevaError):
        gv.mni_support(gdb, ["v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n"])  # not connected
    nine = "".join(f"v {i} 1\n" for i in range(9)) + "".join(f"e {i} {i + 1} 1\n" for i in range(8))
    with pytest.raises(gv.GenevaError):
        gv.mni_support(gdb, [nine])
    oracle.free(og)
    gdb.close()


@pytest.mark.gpu
def test_mni_mining_equals_brute_force(native, tiny_brute):
    db, want_all = tiny_brute
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    for minsup in (2, 4):
        want = {c: m for c, m in want_all.items() if m >= minsup}
        pats, stats = gv.mine(gdb, 3, minsup, support="mni", mni_cap=1 << 30)
        got = {pattern_from_text(p.text): p.support for p in pats}
        assert got == want
        # default cap = min_support: frequency decided, supports reported as min(MNI, minsup)
        pats2, _ = gv.mine(gdb, 3, minsup, support="mni")
        got2 = {pattern_from_text(p.text): p.support for p in pats2}
        assert got2 == {c: min(m, minsup) for c, m in want.items()}
        assert stats["mni_tasks"] > 0 and stats["frequent"] == len(pats)
    gdb.close()


@pytest.mark.gpu
def test_mni_eight_vertex_path_and_hub_star(native, oracle):
    db = small_graph(seed=8)
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    rng = random.Random(3)
    pats = workloads.sample_patterns(db, 6, 8, 8, seed=21, p_extra=0.0)  # 8-vertex trees
    hub = int(np.argmax(np.bincount(np.concatenate([db.src, db.dst]))))
    lab = int(db.vlabels[hub])
    star = f"v 0 {lab}\n" + "".join(f"v {i} {rng.choice([1, 2])}\n" for i in range(1, 6)) + \
        "".join(f"e 0 {i} 1\n" for i in range(1, 6))
    pats.append(star)
    pats = [p for p in pats if oracle.count(og, p, cap_rows=5_000_000) is not None]
    sup, _ = gv.mni_support(gdb, pats, cap=0)
    for p, s in zip(pats, sup):
        assert int(s) == mni_from_rows(oracle, og, p), p
    oracle.free(og)
    gdb.close()


@pytest.mark.gpu
def test_mni_on_a_config4_shaped_rmat(native, oracle):
    """R-MAT with the single-graph configuration's shape at 1/64 of its size
    (a = 0.57, b = c = 0.19, average degree 32, 32 vertex labels Zipf(1.0)):
    300 sampled patterns of 2-4 vertices, exact and capped at 1,000 (the
    configuration's minimum support), batched and plain, against the oracle's
    existence search; 120 of those with at most 200,000 oracle rows also
    against the cpumine rows with automorphism orbits unioned."""
    db = workloads.rmat_graph(16, 1 << 20, 32, 1.0, seed=44, name="c4_shape")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    mg = oracle.mni_graph(db.vlabels, db.src, db.dst, db.elabels)
    og = oracle.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    pats = workloads.sample_patterns(db, 300, 2, 4, seed=45)
    exact = [oracle.mni(mg, p)[0] for p in pats]
    sup, _ = gv.mni_support(gdb, pats, cap=0)
    assert [int(x) for x in sup] == exact
    for plain in (False, True):
        capped, _ = gv.mni_support(gdb, pats, cap=1000, plain=plain)
        assert [int(x) for x in capped] == [min(e, 1000) for e in exact]
    rows_checked = 0
    for p, e in zip(pats, exact):
        if rows_checked == 120 or oracle.count(og, p, cap_rows=200_000) is None:
            continue
        assert mni_from_rows(oracle, og, p) == e, p
        rows_checked += 1
    assert rows_checked >= 100
    oracle.mni_graph_free(mg)
    oracle.free(og)
    gdb.close()
