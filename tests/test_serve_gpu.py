"""Serving loop: every request's result is the same alone and in the mix."""
import random
import time

import numpy as np
import pytest

import geneva_b200 as gv
from geneva_b200 import workloads
from geneva_b200.serve import Server, percentile

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served_db(native):
    db = workloads.graph_database(400, 10, 30, 3.0, 4, None, 2, seed=88, name="serve")
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    gdb.set_graphs(db.first)
    yield db, gdb
    gdb.close()


def test_results_alone_equal_results_in_the_mix(served_db):
    db, gdb = served_db
    pats = workloads.sample_patterns(db, 60, 3, 8, seed=3)
    alone = []
    for p in pats:  # each request by itself
        c, sup, _ = gv.batch_count(gdb, [gv.Plan.from_text(p)], support=True)
        alone.append((int(c[0]), int(sup[0])))
    mine_alone, _ = gv.mine(gdb, 3, 20)

    srv = Server(gdb, budget_bytes=1 << 30)
    rng = random.Random(5)
    reqs, mreq = [], None
    for i, p in enumerate(pats):
        reqs.append(srv.submit_match(p))
        if i == 20:
            mreq = srv.submit_mine(3, 20)
        time.sleep(rng.expovariate(2000.0))  # staggered arrivals join running rounds
    got = [r.future.result(timeout=300) for r in reqs]
    mined, _ = mreq.future.result(timeout=300)
    srv.close()
    assert got == alone
    key = lambda ps: sorted((p.text, p.support, p.embeddings) for p in ps)
    assert key(mined) == key(mine_alone)
    lat = [r.latency for r in reqs]
    assert all(l > 0 for l in lat) and percentile(lat, 99) >= percentile(lat, 50)
    assert srv.rounds > 0


def test_tight_admission_budget_still_completes(served_db):
    db, gdb = served_db
    pats = workloads.sample_patterns(db, 30, 3, 6, seed=11)
    want = [int(gv.batch_count(gdb, [gv.Plan.from_text(p)])[0][0]) for p in pats]
    srv = Server(gdb, budget_bytes=64 << 10, support=False)  # the engine splits work to fit
    reqs = [srv.submit_match(p) for p in pats]
    got = [r.future.result(timeout=300)[0] for r in reqs]
    srv.close()
    assert got == want


def test_bad_request_fails_alone(served_db):
    _, gdb = served_db
    srv = Server(gdb)
    bad = srv.submit_match("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n")  # disconnected pattern
    good = srv.submit_match("v 0 1\nv 1 2\ne 0 1 1\n")
    with pytest.raises(gv.GenevaError):
        bad.future.result(timeout=60)
    assert good.future.result(timeout=60)[0] >= 0
    srv.close()


def test_mni_mining_requests_on_a_second_graph(served_db):
    """Mining requests against a separate single graph (MNI support) give the
    same patterns in the mix as alone, while matching requests keep flowing."""
    db, gdb = served_db
    g4 = workloads.rmat_graph(9, 3000, 4, 1.0, seed=6, name="serve_rmat")
    mdb = gv.Database.from_edges(g4.vlabels, g4.src, g4.dst, g4.elabels)
    alone, _ = gv.mine(mdb, 3, 40, support="mni")
    pats = workloads.sample_patterns(db, 20, 3, 6, seed=13)
    want = [int(gv.batch_count(gdb, [gv.Plan.from_text(p)])[0][0]) for p in pats]
    srv = Server(gdb, budget_bytes=1 << 30, mine_db=mdb)
    m = srv.submit_mine(3, 40)
    reqs = [srv.submit_match(p) for p in pats]
    got = [r.future.result(timeout=300)[0] for r in reqs]
    mined, _ = m.future.result(timeout=300)
    srv.close()
    assert got == want
    key = lambda ps: sorted((p.text, p.support) for p in ps)
    assert key(mined) == key(alone) and len(mined) > 0
    mdb.close()
