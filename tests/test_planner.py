"""Product planner (gva_plan_*, host-only) against the reference planner's
plans (src/genMatchOrderCPU.cpp) and the oracle's restatement."""
import random

import pytest

import geneva_b200 as gv
from querygen import random_query


def test_planner_matches_reference_plans(native, golden_plans):
    bad = []
    for g in golden_plans:
        p = gv.Plan.from_text(g["q"], gv.MODE_DV)
        if p.describe() != g["plan"]:
            bad.append(g["q"])
    assert not bad, f"{len(bad)} of {len(golden_plans)} plans differ; first:\n{bad[0]}"


def test_planner_matches_oracle_on_fresh_queries(native, oracle):
    rng = random.Random(99)
    for _ in range(400):
        q = random_query(rng)
        assert gv.Plan.from_text(q).describe() == oracle.plan(q), q


def _phases(desc):
    out = []
    for line in desc.splitlines():
        t = line.split()
        if t[0] == "phase":
            out.append((t[2], int(t[3]), [int(x) for x in t[5:]]))
    return out


def test_single_vertex_mode_splits_phases(native, golden_plans):
    for g in golden_plans[:300]:
        dv = _phases(gv.Plan.from_text(g["q"], gv.MODE_DV).describe())
        sv = _phases(gv.Plan.from_text(g["q"], gv.MODE_SV).describe())
        split = []
        for typ, el, pairs in dv:
            for i in range(0, len(pairs), 2):
                split.append((typ, el, pairs[i:i + 2]))
        assert sv == split
        assert gv.Plan.from_text(g["q"], gv.MODE_SV).columns == gv.Plan.from_text(g["q"]).columns


def test_columns_follow_match_order(native):
    p = gv.genMatchOrder("v 0 2\nv 1 1\nv 2 3\nv 3 1\ne 0 1 3\ne 0 2 1\ne 1 3 2\ne 1 2 2\n")
    assert p.columns == [0, 1, 2, 3]
    assert p.num_phases == 4


@pytest.mark.parametrize("text,status", [
    ("", gv.MODE_DV),
    ("v 0 1\n", 2),
    ("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n", 6),            # disconnected
    ("v 0 1\nv 1 1\ne 0 0 1\ne 0 1 1\n", 6),          # self-loop
    ("v 0 1\nv 2 1\ne 0 2 1\n", 2),                   # ids not 0..n-1
    ("".join(f"v {i} 1\n" for i in range(33)) + "".join(f"e {i} {i+1} 1\n" for i in range(32)), 6),
])
def test_planner_errors(native, text, status):
    with pytest.raises(gv.GenevaError) as ei:
        gv.Plan.from_text(text)
    assert ei.value.status in (2, 6)


def test_huge_symmetry_is_rejected_not_enumerated(native):
    """A 14-vertex clique of one label has 14! automorphisms: the reference
    would enumerate them for ever; the planner stops at a bound and reports
    the query as unsupported, quickly."""
    import time
    n = 14
    text = "".join(f"v {i} 1\n" for i in range(n)) + "".join(
        f"e {i} {j} 1\n" for i in range(n) for j in range(i + 1, n))
    t0 = time.perf_counter()
    with pytest.raises(gv.GenevaError) as e:
        gv.Plan.from_text(text)
    assert e.value.status == 6 and "symmetric" in str(e.value)
    assert time.perf_counter() - t0 < 30
    # symmetric but small: planned as usual (a 7-vertex star, 6! automorphisms)
    star = "".join(f"v {i} 1\n" for i in range(7)) + "".join(f"e 0 {j} 1\n" for j in range(1, 7))
    assert gv.Plan.from_text(star).num_phases > 0


def test_bad_mode_rejected(native):
    with pytest.raises(gv.GenevaError) as ei:
        gv.Plan.from_text("v 0 1\nv 1 1\ne 0 1 1\n", 7)
    assert ei.value.status == 5


def test_batch_planning_equals_one_by_one(native, golden_plans):
    """gva_plan_batch (host threads) gives the reference's plans, per query
    the same as gva_plan_from_text, and reports which query failed."""
    qs = [g["q"] for g in golden_plans]
    plans = gv.Plan.batch_from_texts(qs)
    assert [p.describe() for p in plans] == [g["plan"] for g in golden_plans]
    sv = gv.Plan.batch_from_texts(qs[:300], gv.MODE_SV)
    assert [p.describe() for p in sv] == [gv.Plan.from_text(q, gv.MODE_SV).describe() for q in qs[:300]]
    bad = qs[:400] + ["v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n"] + qs[400:600]  # a disconnected pattern at index 400
    with pytest.raises(gv.GenevaError) as e:
        gv.Plan.batch_from_texts(bad)
    assert "query 400" in str(e.value)
