"""Seeded generators for query patterns and small labelled data graphs.

Shared by the fixture script (make_golden.py) and the tests.  Query text uses
the reference .query format: `v <id> <label>` lines, then `e <s> <d> <label>`
lines (exp/datasets/Enron/Enron_4_6_0.query).  Graph text uses the reference
.g format read by tools/genDatabase.cpp:769-800.
"""
from __future__ import annotations

import random
from typing import Dict, List, Optional, Sequence, Tuple

Edge = Tuple[int, int, int]


def query_text(labels: Sequence[int], edges: Sequence[Edge]) -> str:
    out = [f"v {i} {l}" for i, l in enumerate(labels)]
    out += [f"e {s} {d} {l}" for s, d, l in edges]
    return "\n".join(out) + "\n"


def _random_connected(n: int, p_extra: float, rng: random.Random) -> List[Tuple[int, int]]:
    order = list(range(n))
    rng.shuffle(order)
    es = set()
    for i in range(1, n):
        a, b = order[i], order[rng.randrange(i)]
        es.add((min(a, b), max(a, b)))
    for a in range(n):
        for b in range(a + 1, n):
            if (a, b) not in es and rng.random() < p_extra:
                es.add((a, b))
    es = sorted(es)
    rng.shuffle(es)
    return es


def random_query(rng: random.Random) -> str:
    n = rng.choice([2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 12])
    vl = rng.choice([1, 1, 2, 2, 3, 4, 6])
    el = rng.choice([1, 1, 2, 3])
    p = rng.choice([0.0, 0.1, 0.2, 0.35, 0.5, 0.7])
    if vl == 1 and n > 7:
        p = min(p, 0.25)  # keep automorphism groups enumerable
    pairs = _random_connected(n, p, rng)
    labels = [rng.randint(1, vl) for _ in range(n)]
    edges = [(a, b, rng.randint(1, el)) if rng.random() < 0.5 else (b, a, rng.randint(1, el)) for a, b in pairs]
    return query_text(labels, edges)


def structured_queries() -> List[str]:
    qs: List[str] = []
    # triangles: every vertex/edge label coincidence pattern (triangle scores 0..33)
    for vls in [(1, 1, 1), (1, 1, 2), (1, 2, 1), (2, 1, 1), (1, 2, 3)]:
        for els in [(1, 1, 1), (1, 1, 2), (1, 2, 1), (2, 1, 1), (1, 2, 3)]:
            qs.append(query_text(vls, [(0, 1, els[0]), (1, 2, els[1]), (0, 2, els[2])]))
    for n in range(3, 8):  # cliques, one label
        qs.append(query_text([1] * n, [(a, b, 1) for a in range(n) for b in range(a + 1, n)]))
    for n in range(4, 10):  # cycles
        qs.append(query_text([1] * n, [(i, (i + 1) % n, 1) for i in range(n)]))
        qs.append(query_text([1 + (i % 2) for i in range(n)], [(i, (i + 1) % n, 1) for i in range(n)]))
    for n in range(2, 9):  # stars and paths
        qs.append(query_text([1] * (n + 1), [(0, i, 1) for i in range(1, n + 1)]))
        qs.append(query_text([2] + [1] * n, [(0, i, 1 + (i % 2)) for i in range(1, n + 1)]))
        qs.append(query_text([1] * (n + 1), [(i, i + 1, 1) for i in range(n)]))
    qs.append(query_text([1] * 5, [(0, 2, 1), (0, 3, 1), (0, 4, 1), (1, 2, 1), (1, 3, 1), (1, 4, 1)]))  # K2,3
    qs.append(query_text([1] * 6, [(a, b, 1) for a in range(3) for b in range(3, 6)]))  # K3,3
    qs.append(query_text([1] * 6, [(0, i, 1) for i in range(1, 6)] + [(i, i % 5 + 1, 1) for i in range(1, 6)]))
    qs.append(query_text([1, 1, 1, 1, 1], [(0, 1, 1), (1, 2, 1), (2, 3, 1), (3, 0, 1), (2, 4, 1), (3, 4, 1)]))
    qs.append("v 0 2\nv 1 1\nv 2 3\nv 3 1\ne 0 1 3\ne 0 2 1\ne 1 3 2\ne 1 2 2\n")  # Enron_4_6_0 shape
    qs.append("# comment line\nv 0 1\nv 1 1\nv 2 2\n# another\ne 0 1 1\ne 1 2 1\ne 0 2 1\n")
    qs.append("v 0 1\nv 1 2\nv 2 1\ne 0 1 1\ne 0 1 1\ne 1 2 1\n")  # duplicate edge line
    qs.append("v 0 1\nv 1 1\ne 0 1 1\n")
    return qs


def make_graph(spec: Dict) -> Tuple[List[int], List[Edge]]:
    """Random connected labelled graph: spanning tree + uniform extra edges to
    the target average degree, optional hub vertex 0; no self loops or
    duplicate edges.  Vertex ids 0..n-1."""
    rng = random.Random(spec["seed"])
    n = spec["n"]
    labels = [rng.randint(1, spec["vlabels"]) for _ in range(n)]
    es = set()
    for i in range(1, n):
        j = rng.randrange(i)
        es.add((min(i, j), max(i, j)))
    target = int(spec["avg_deg"] * n / 2)
    while len(es) < target:
        a, b = rng.randrange(n), rng.randrange(n)
        if a != b:
            es.add((min(a, b), max(a, b)))
    hub = spec.get("hub", 0)
    if hub:
        for b in rng.sample(range(1, n), min(hub, n - 1)):
            es.add((0, b))
    edges = [(a, b, rng.randint(1, spec["elabels"])) for a, b in sorted(es)]
    return labels, edges


def write_g(labels: Sequence[int], edges: Sequence[Edge]) -> str:
    out = [f"v {i} {l}" for i, l in enumerate(labels)]
    out += [f"e {a} {b} {l}" for a, b, l in edges]
    return "\n".join(out) + "\n"


def sample_query(labels: Sequence[int], edges: Sequence[Edge], k: int, rng: random.Random) -> Optional[str]:
    """A connected k-vertex pattern taken from the data graph (so it matches):
    the growth tree plus each other induced edge with probability 1/2."""
    adj: Dict[int, Dict[int, int]] = {}
    for a, b, l in edges:
        adj.setdefault(a, {})[b] = l
        adj.setdefault(b, {})[a] = l
    start = rng.choice(list(adj.keys()))
    chosen = [start]
    tree = []
    while len(chosen) < k:
        frontier = [(u, w) for u in chosen for w in adj[u] if w not in chosen]
        if not frontier:
            return None
        u, w = rng.choice(frontier)
        chosen.append(w)
        tree.append((u, w))
    idx = {v: i for i, v in enumerate(rng.sample(chosen, len(chosen)))}
    es = {(min(idx[u], idx[w]), max(idx[u], idx[w])): adj[u][w] for u, w in tree}
    for i, u in enumerate(chosen):
        for w in chosen[i + 1:]:
            key = (min(idx[u], idx[w]), max(idx[u], idx[w]))
            if w in adj[u] and key not in es and rng.random() < 0.5:
                es[key] = adj[u][w]
    qlabels = [0] * k
    for v, i in idx.items():
        qlabels[i] = labels[v]
    return query_text(qlabels, [(a, b, l) for (a, b), l in sorted(es.items())])
