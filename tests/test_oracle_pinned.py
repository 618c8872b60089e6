"""The oracle is pinned against the reference's own outputs (no GPU).

Golden vectors come from the reference binaries compiled from source
(tests/golden/make_golden.py): plan text from src/genMatchOrderCPU.cpp, row
sets from src/cpumine.cpp on graphs converted by tools/genDatabase.cpp, and
the Enron known answer (157,502 distinct rows).
"""
import json

import pytest

from conftest import GOLDEN
from oracle_lib import rows_digest


def test_oracle_planner_matches_reference(oracle, golden_plans):
    bad = [g["q"] for g in golden_plans if oracle.plan(g["q"]) != g["plan"]]
    assert not bad, f"{len(bad)} plans differ, first:\n{bad[0]}"


@pytest.fixture(scope="module")
def oracle_graphs(oracle):
    gs = {}
    for p in (GOLDEN / "graphs").glob("*.mygraph"):
        gs[p.stem] = oracle.load(p, p.with_suffix(".metadata"))
    yield gs
    for g in gs.values():
        oracle.free(g)


def test_oracle_rows_match_reference_cpumine(oracle, oracle_graphs, golden_matches):
    assert len(golden_matches) >= 90
    for m in golden_matches:
        rows, _ = oracle.match(oracle_graphs[m["graph"]], m["q"])
        cnt, dig = rows_digest(rows)
        assert cnt == m["rows"], (m["graph"], m["q"])
        assert dig == m["sha256"], (m["graph"], m["q"])
        # the oracle reads stripped lists: no duplicate rows, unlike cpumine
        assert rows.shape[0] == cnt


def test_oracle_enron_known_answer(oracle, enron_dir):
    kat = json.loads((GOLDEN / "enron" / "enron.json").read_text())
    g = oracle.load(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    q = (enron_dir / "Enron_4_6_0.query").read_text()
    rows, phases = oracle.match(g, q)
    oracle.free(g)
    assert kat["rows"] == 157502 and kat["raw_rows"] == 158112
    assert rows_digest(rows) == (kat["rows"], kat["sha256"])
    assert phases[0] == 13891 and phases[2] == 6123 and phases[-1] == 157502
    assert oracle.plan(q) == kat["plan"]
