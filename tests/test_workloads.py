"""Seeded workload generators and host-side containers (CPU only)."""
import numpy as np

import geneva_b200 as gv
from geneva_b200 import workloads


def test_config3_queries_are_induced_connected_subgraphs():
    db = workloads.config1(seed=1)
    qs = workloads.config3_queries(db, 60, seed=7)
    assert len(qs) == 60
    for q in qs:
        vs = [l for l in q.splitlines() if l.startswith("v ")]
        es = [l for l in q.splitlines() if l.startswith("e ")]
        assert 3 <= len(vs) <= 8
        # connected: union-find over the pattern edges
        parent = list(range(len(vs)))

        def root(x):
            while parent[x] != x:
                x = parent[x]
            return x
        for e in es:
            _, a, b, _ = e.split()
            parent[root(int(a))] = root(int(b))
        assert len({root(i) for i in range(len(vs))}) == 1
    assert workloads.config3_queries(db, 60, seed=7) == qs  # seeded


def test_config_databases_have_their_shapes():
    c1 = workloads.config1(seed=1)
    assert len(c1.first) - 1 == 1000 and set(np.unique(c1.vlabels[1:])) <= {1, 2, 3, 4}
    assert set(np.unique(c1.elabels)) == {1}
    sizes = np.diff(c1.first)
    assert sizes.min() >= 10 and sizes.max() <= 30
    deg = 2 * c1.num_edges / c1.num_vertices
    assert 2.7 < deg < 3.3


def test_mined_patterns_container():
    texts = ["v 0 1\nv 1 2\ne 0 1 1\n", "v 0 3\nv 1 3\nv 2 1\ne 0 1 2\ne 1 2 1\n"]
    blob = np.frombuffer(b"".join(t.encode() + b"\0" for t in texts), dtype=np.uint8)
    off = np.array([0, len(texts[0]) + 1], dtype=np.uint64)
    mp = gv.MinedPatterns(blob, off, np.array([1, 2], np.uint32), np.array([5, 7], np.uint32),
                          np.array([10, 20], np.uint64))
    assert len(mp) == 2 and mp.text(1) == texts[1]
    assert mp[0].text == texts[0] and mp[-1].support == 7 and mp[1].embeddings == 20
    assert [p.edges for p in mp] == [1, 2] and [p.edges for p in mp[0:2]] == [1, 2]
    assert mp.text_bytes == sum(len(t) for t in texts)


def test_batch_planning_of_nothing(native):
    assert list(gv.Plan.batch_from_texts([])) == []
