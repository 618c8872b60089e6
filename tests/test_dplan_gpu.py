"""The device planner (gva_dplan.cu: the heap-free planner of gva_dplan.h,
one query per thread on the GPU) against the host planner: plan texts
(phases, pair orientation, restrictions, repeat flags, record stats, columns)
equal on the reference's 1,500 golden queries, on seeded random queries and
on patterns mined from the 20,000-graph database; batched counts with device
planning equal to host planning."""
import random

import numpy as np
import pytest

import geneva_b200 as gv
from geneva_b200 import workloads
from querygen import random_query

pytestmark = pytest.mark.gpu


def _same(texts):
    dev = gv.Plan.batch_from_texts_device(texts)
    host = gv.Plan.batch_from_texts(texts)
    bad = [t for t, a, b in zip(texts, dev, host) if a.describe() != b.describe()]
    for p in dev + host:
        p.close()
    return bad


def test_device_plans_match_reference_plans(native, golden_plans):
    texts = [g["q"] for g in golden_plans]
    dev = gv.Plan.batch_from_texts_device(texts)
    bad = [g["q"] for g, p in zip(golden_plans, dev) if p.describe() != g["plan"]]
    assert not bad, f"{len(bad)} of {len(texts)} device plans differ from the reference's; first:\n{bad[0]}"


def test_device_plans_equal_host_plans_on_random_queries(native):
    rng = random.Random(2024)
    texts = [random_query(rng) for _ in range(60000)]
    bad = _same(texts)
    assert not bad, f"{len(bad)} differ; first:\n{bad[0]}"


def test_device_plans_equal_host_plans_on_mined_patterns(native):
    db = workloads.config2(seed=2)
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    pats, _ = gv.mine(gdb, 5, 400)
    texts = [p.text for p in pats]
    assert len(texts) > 5000
    bad = _same(texts)
    assert not bad, f"{len(bad)} of {len(texts)} differ; first:\n{bad[0]}"
    # counting with device planning gives the host-planned counts
    sample = texts[:: max(1, len(texts) // 2000)]
    a, sa, _ = gv.batch_count_texts(gdb, sample, support=True, plan_on_device=True)
    b, sb, _ = gv.batch_count_texts(gdb, sample, support=True)
    assert np.array_equal(a, b) and np.array_equal(sa, sb)
    gdb.close()
