"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Row sets are compared as (distinct count, sha256 of sorted distinct rows);
integer work, so the bar is bit-exact.  Golden hashes come from the reference
`cpumine` (tests/golden/make_golden.py); fresh random cases are checked
against the oracle, including per-phase row counts.
"""
import json
import os
import random
import subprocess

import numpy as np
import pytest

import geneva_b200 as gv
from conftest import GOLDEN
from oracle_lib import rows_digest
from querygen import make_graph, random_query, sample_query, query_text

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden_dbs(native):
    dbs = {}
    for p in sorted((GOLDEN / "graphs").glob("*.mygraph")):
        dbs[p.stem] = gv.loadDataBase(p, p.with_suffix(".metadata"))
    yield dbs
    for d in dbs.values():
        d.close()


@pytest.mark.parametrize("mode", [gv.MODE_DV, gv.MODE_SV])
def test_golden_graphs_match_reference_cpumine(golden_dbs, golden_matches, mode):
    for m in golden_matches:
        plan = gv.Plan.from_text(m["q"], mode)
        res = gv.match(golden_dbs[m["graph"]], plan)
        rows = res.rows()
        assert rows.shape[0] == res.num_rows
        assert res.num_rows == m["rows"], (m["graph"], m["q"])
        assert rows_digest(rows) == (m["rows"], m["sha256"]), (m["graph"], m["q"])


def test_enron_known_answer(native, oracle, enron_dir):
    kat = json.loads((GOLDEN / "enron" / "enron.json").read_text())
    db = gv.loadDataBase(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    assert "declares 4 partitions" in db.warnings
    q = (enron_dir / "Enron_4_6_0.query").read_text()
    og = oracle.load(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    _, ophases = oracle.match(og, q)
    oracle.free(og)
    for mode in (gv.MODE_DV, gv.MODE_SV):
        res = gv.match(db, gv.Plan.from_text(q, mode))
        assert rows_digest(res.rows()) == (kat["rows"], kat["sha256"])
        if mode == gv.MODE_DV:
            assert res.phase_rows == ophases == [13891, 194892, 6123, 157502]
    # deterministic output order
    a = gv.match(db, gv.Plan.from_text(q)).rows()
    b = gv.match(db, gv.Plan.from_text(q)).rows()
    assert np.array_equal(a, b)
    db.close()


def _edge_arrays(labels, edges):
    vl = np.array([0] + list(labels), dtype=np.uint32)  # ids shift by one: data ids are 1-based
    src = np.array([a + 1 for a, _, _ in edges], dtype=np.uint32)
    dst = np.array([b + 1 for _, b, _ in edges], dtype=np.uint32)
    el = np.array([l for _, _, l in edges], dtype=np.uint32)
    return vl, src, dst, el


SPECS = [
    dict(n=300, avg_deg=6.0, vlabels=2, elabels=1, seed=11, hub=0),
    dict(n=2000, avg_deg=4.0, vlabels=3, elabels=2, seed=12, hub=300),
    dict(n=500, avg_deg=8.0, vlabels=1, elabels=1, seed=13, hub=0),
    dict(n=3000, avg_deg=3.0, vlabels=5, elabels=3, seed=14, hub=4500 - 1600),
]


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"n{s['n']}_l{s['vlabels']}_e{s['elabels']}")
def test_random_queries_match_oracle(native, oracle, spec):
    labels, edges = make_graph(spec)
    arrs = _edge_arrays(labels, edges)
    db = gv.Database.from_edges(*arrs)
    og = oracle.from_edges(*arrs)
    rng = random.Random(spec["seed"] * 31)
    checked = 0
    for i in range(30):
        if i % 3 == 2:
            q = random_query(rng)
        else:
            q = sample_query(labels, edges, rng.randint(3, 6), rng)
            if q is None:
                continue
        if oracle.count(og, q, cap_rows=300_000) is None:
            continue  # too large for a quick CPU check
        orows, ophases = oracle.match(og, q)
        for mode in (gv.MODE_DV, gv.MODE_SV):
            res = gv.match(db, gv.Plan.from_text(q, mode))
            got = res.rows()
            assert rows_digest(got) == rows_digest(orows), q
            assert got.shape[0] == orows.shape[0], q  # no duplicates
            if mode == gv.MODE_DV:
                assert res.phase_rows == ophases, q
        checked += 1
    assert checked >= 15
    oracle.free(og)
    db.close()


def test_absent_labels_give_empty_results(native, oracle):
    labels, edges = make_graph(dict(n=200, avg_deg=4.0, vlabels=2, elabels=1, seed=5, hub=0))
    db = gv.Database.from_edges(*_edge_arrays(labels, edges))
    for q in ["v 0 1\nv 1 9\ne 0 1 1\n",            # vertex label absent
              "v 0 1\nv 1 2\nv 2 1\ne 0 1 1\ne 1 2 7\n",  # edge label absent
              "v 0 9\nv 1 9\nv 2 9\ne 0 1 1\ne 1 2 1\ne 0 2 1\n"]:
        res = gv.match(db, gv.Plan.from_text(q))
        assert res.num_rows == 0
        assert res.rows().shape[0] == 0
    db.close()


def test_reduction_with_more_than_16_pairs_is_empty_like_the_reference(native, oracle):
    # a 20-clique in the data, queried as a 19-clique: its last vertex closes
    # 17 same-label back edges in one reduction phase, and the reference then
    # emits nothing (src/cpumine.cpp:499-502, src/gpumine.cpp:759-762)
    n = 20
    labels = list(range(1, n + 1))
    edges = [(a, b, 1) for a in range(n) for b in range(a + 1, n)]
    arrs = _edge_arrays(labels, edges)
    clique = lambda k: query_text(list(range(1, k + 1)), [(a, b, 1) for a in range(k) for b in range(a + 1, k)])
    plan = gv.Plan.from_text(clique(19))
    assert max(int(l.split()[4]) for l in plan.describe().splitlines() if l.startswith("phase")) == 17
    db = gv.Database.from_edges(*arrs)
    og = oracle.from_edges(*arrs)
    assert oracle.match(og, clique(19))[0].shape[0] == 0
    assert gv.match(db, plan).num_rows == 0
    # 16 pairs still reduce: the 18-clique has exactly one labelled embedding
    assert gv.match(db, gv.Plan.from_text(clique(18))).num_rows == oracle.match(og, clique(18))[0].shape[0] == 1
    oracle.free(og)
    db.close()


def test_count_only_and_budget(native, enron_dir):
    db = gv.loadDataBase(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    q = (enron_dir / "Enron_4_6_0.query").read_text()
    plan = gv.Plan.from_text(q)
    res = gv.match(db, plan, count_only=True)
    assert res.num_rows == 157502 and res.device_ptr is None
    with pytest.raises(gv.GenevaError) as ei:
        gv.match(db, plan, budget_bytes=1024)
    assert ei.value.status == 4
    db.close()


def test_step_api_chain_equals_match(native, enron_dir):
    import ctypes
    torch = pytest.importorskip("torch")
    lib = native
    db = gv.loadDataBase(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    plan = gv.Plan.from_text((enron_dir / "Enron_4_6_0.query").read_text())
    nsteps = lib.gva_plan_num_steps(plan._h, db._h)
    assert nsteps >= 5
    cur = None
    rows = 0
    stream = torch.cuda.current_stream().cuda_stream
    for s in range(nsteps):
        win = lib.gva_plan_step_width_in(plan._h, db._h, s)
        wout = lib.gva_plan_step_width_out(plan._h, db._h, s)
        scratch = torch.empty(max(1, lib.gva_step_scratch_bytes(rows)), dtype=torch.uint8, device="cuda")
        cap = 1
        out = torch.empty(cap * wout, dtype=torch.int32, device="cuda")
        n = ctypes.c_uint64()
        args = lambda o, c: (db._h, plan._h, s, cur.data_ptr() if cur is not None else None, rows,
                             o.data_ptr(), c, ctypes.byref(n), scratch.data_ptr(), scratch.numel(), stream)
        st = lib.gva_step_run(*args(out, cap))
        if st == 4:  # grow to the reported size and rerun
            cap = n.value
            out = torch.empty(max(1, cap * wout), dtype=torch.int32, device="cuda")
            st = lib.gva_step_run(*args(out, cap))
        assert st == 0, lib.gva_last_error()
        cur, rows = out[: n.value * wout], n.value
        assert win in (0, wout - 1, wout)
    torch.cuda.synchronize()
    chained = cur.view(torch.int32).cpu().numpy().view(np.uint32).reshape(rows, -1)
    ref = gv.match(db, plan).rows()
    assert np.array_equal(chained, ref)
    db.close()


def test_cli_gpumine_enron(native, enron_dir, tmp_path):
    kat = json.loads((GOLDEN / "enron" / "enron.json").read_text())
    exe = gv.library_path().parent / "gpumine"
    for name in ("gpumine", "gpumineSV"):
        exe = gv.library_path().parent / name
        r = subprocess.run([str(exe), str(enron_dir / "Enron.mygraph"), str(enron_dir / "Enron.metadata"),
                            str(enron_dir / "Enron_4_6_0.query")], cwd=tmp_path, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "Result: 157502 extra size0" in r.stdout
        assert "PartialRowNum: 157502 embLen:  4" in r.stdout
        assert "phase 0 type E edge label:3" in r.stdout
        rows = np.loadtxt(tmp_path / "partialResultsGPU.txt", dtype=np.uint32)
        assert rows_digest(rows) == (kat["rows"], kat["sha256"])
