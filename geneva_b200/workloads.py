"""Seeded synthetic databases and query batches.

The reference ships only the Enron graph; the benchmark configurations are
described by their shapes, so they are generated here from a seed:

  graph database (1,000 or 20,000 graphs)  -> one disjoint-union data graph,
      global ids 1..V, graph g owning ids [first[g], first[g+1]);
  query batch                              -> connected patterns sampled from
      the database (so every pattern has at least one embedding).

Everything is numpy; vertex ids are 1-based uint32 as the reference requires
(src/gpumine.cpp:1-3), edge labels are 1..P.
"""
from __future__ import annotations

import random
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np


@dataclass
class GraphDB:
    name: str
    vlabels: np.ndarray          # uint32, len V+1, entry 0 unused
    src: np.ndarray              # uint32 edge endpoints (each undirected edge once)
    dst: np.ndarray
    elabels: np.ndarray          # uint32, 1..P
    first: np.ndarray            # int64, len G+1: graph g owns ids [first[g], first[g+1])
    params: Dict = field(default_factory=dict)
    cache: Dict = field(default_factory=dict, repr=False, compare=False)  # derived lookups, built on first use

    @property
    def num_vertices(self) -> int:
        return len(self.vlabels) - 1

    @property
    def num_edges(self) -> int:
        return len(self.src)

    def graph_of(self, v: np.ndarray) -> np.ndarray:
        return np.searchsorted(self.first, v, side="right") - 1

    def to_g_text(self) -> str:
        """The .g text read by tools/genDatabase.cpp (ids shifted to 0-based)."""
        lines = [f"v {i - 1} {int(self.vlabels[i])}" for i in range(1, len(self.vlabels))]
        lines += [f"e {int(a) - 1} {int(b) - 1} {int(l)}" for a, b, l in zip(self.src, self.dst, self.elabels)]
        return "\n".join(lines) + "\n"


def zipf_labels(rng: np.random.Generator, n: int, k: int, s: float) -> np.ndarray:
    p = np.arange(1, k + 1, dtype=np.float64) ** (-s)
    p /= p.sum()
    return (rng.choice(k, size=n, p=p) + 1).astype(np.uint32)


def graph_database(num_graphs: int, vmin: int, vmax: int, avg_deg: float, vlabel_k: int, vlabel_zipf: Optional[float],
                   elabel_k: int, seed: int, name: str) -> GraphDB:
    """Connected graphs: random spanning tree plus uniformly random extra edges
    up to the target average degree; no self-loops or multi-edges."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(vmin, vmax + 1, size=num_graphs)
    first = np.zeros(num_graphs + 1, dtype=np.int64)
    first[1:] = np.cumsum(sizes)
    first += 1
    V = int(first[-1] - 1)
    # spanning trees: local vertex i > 0 attaches to a uniform j < i
    gid = np.repeat(np.arange(num_graphs), sizes)
    local = np.arange(V) - (first[gid] - 1)
    base = first[gid]
    tree_mask = local > 0
    par = np.floor(rng.random(V) * np.maximum(local, 1)).astype(np.int64)
    ts = (base + local)[tree_mask]
    td = (base + par)[tree_mask]
    # extra edges per graph: target edges = round(avg_deg * n / 2)
    target = np.rint(avg_deg * sizes / 2).astype(np.int64)
    need = np.maximum(target - (sizes - 1), 0)
    es, ed = [ts], [td]
    key_all = set()
    a = np.minimum(ts, td)
    b = np.maximum(ts, td)
    keys = (a.astype(np.uint64) << np.uint64(32)) | b.astype(np.uint64)
    have = np.unique(keys)
    remaining = need.copy()
    for _ in range(8):
        if remaining.sum() == 0:
            break
        cnt = (remaining * 2 + 4)
        g = np.repeat(np.arange(num_graphs), cnt)
        u = first[g] + np.floor(rng.random(len(g)) * sizes[g]).astype(np.int64)
        v = first[g] + np.floor(rng.random(len(g)) * sizes[g]).astype(np.int64)
        ok = u != v
        g, u, v = g[ok], u[ok], v[ok]
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        k = (lo.astype(np.uint64) << np.uint64(32)) | hi.astype(np.uint64)
        k, idx = np.unique(k, return_index=True)
        g, lo, hi = g[idx], lo[idx], hi[idx]
        fresh = ~np.isin(k, have)
        g, lo, hi, k = g[fresh], lo[fresh], hi[fresh], k[fresh]
        # keep at most remaining[g] per graph (random order within graph)
        order = np.lexsort((rng.random(len(g)), g))
        g, lo, hi, k = g[order], lo[order], hi[order], k[order]
        start = np.searchsorted(g, np.arange(num_graphs))
        rank = np.arange(len(g)) - start[g]
        take = rank < remaining[g]
        es.append(lo[take])
        ed.append(hi[take])
        have = np.union1d(have, k[take])
        remaining -= np.bincount(g[take], minlength=num_graphs)
    src = np.concatenate(es).astype(np.uint32)
    dst = np.concatenate(ed).astype(np.uint32)
    if vlabel_zipf is None:
        vl = rng.integers(1, vlabel_k + 1, size=V).astype(np.uint32)
    else:
        vl = zipf_labels(rng, V, vlabel_k, vlabel_zipf)
    vlabels = np.zeros(V + 1, dtype=np.uint32)
    vlabels[1:] = vl
    el = rng.integers(1, elabel_k + 1, size=len(src)).astype(np.uint32)
    return GraphDB(name, vlabels, src, dst, el, first,
                   dict(graphs=num_graphs, vmin=vmin, vmax=vmax, avg_deg=avg_deg, vertex_labels=vlabel_k,
                        vertex_label_zipf=vlabel_zipf, edge_labels=elabel_k, seed=seed))


def config1(seed: int = 1) -> GraphDB:
    """1,000 graphs, |V|~U[10,30], avg degree 3, 4 uniform vertex labels, unlabeled edges."""
    return graph_database(1000, 10, 30, 3.0, 4, None, 1, seed, "config1")


def config2(seed: int = 2) -> GraphDB:
    """20,000 graphs, |V|~U[20,60], avg degree 4, 16 vertex labels Zipf(1.2), 3 edge labels."""
    return graph_database(20000, 20, 60, 4.0, 16, 1.2, 3, seed, "config2")


def _edges_by_graph(db: GraphDB) -> Tuple[np.ndarray, np.ndarray]:
    """Edge indices grouped by the graph of their source (a stable sort, so
    each graph's edges keep their order in the edge arrays) and each graph's
    range in that list; computed once per database."""
    cached = db.cache.get("edges_by_graph")
    if cached is None:
        gsrc = db.graph_of(db.src.astype(np.int64))
        order = np.argsort(gsrc, kind="stable")
        bounds = np.searchsorted(gsrc[order], np.arange(len(db.first)))
        cached = (order, bounds)
        db.cache["edges_by_graph"] = cached
    return cached


def _adjacency(db: GraphDB, g: int):
    order, bounds = _edges_by_graph(db)
    idx = order[bounds[g]:bounds[g + 1]]
    adj: Dict[int, Dict[int, int]] = {}
    for a, b, l in zip(db.src[idx].tolist(), db.dst[idx].tolist(), db.elabels[idx].tolist()):
        adj.setdefault(a, {})[b] = l
        adj.setdefault(b, {})[a] = l
    return adj


def sample_patterns(db: GraphDB, count: int, vmin: int, vmax: int, seed: int, p_extra: float = 0.5) -> List[str]:
    """Connected patterns grown inside random database graphs: the growth tree
    plus each other induced edge with probability p_extra; labels copied."""
    rng = random.Random(seed)
    out: List[str] = []
    G = len(db.first) - 1
    while len(out) < count:
        g = rng.randrange(G)
        adj = _adjacency(db, g)
        if not adj:
            continue
        k = rng.randint(vmin, vmax)
        start = rng.choice(sorted(adj))
        chosen = [start]
        tree = []
        while len(chosen) < k:
            fr = [(u, w) for u in chosen for w in adj[u] if w not in chosen]
            if not fr:
                break
            u, w = rng.choice(fr)
            chosen.append(w)
            tree.append((u, w))
        if len(chosen) < k:
            continue
        idx = {v: i for i, v in enumerate(chosen)}
        es = {(min(idx[u], idx[w]), max(idx[u], idx[w])): adj[u][w] for u, w in tree}
        for i, u in enumerate(chosen):
            for w in chosen[i + 1:]:
                key = (min(idx[u], idx[w]), max(idx[u], idx[w]))
                if w in adj[u] and key not in es and rng.random() < p_extra:
                    es[key] = adj[u][w]
        lines = [f"v {i} {int(db.vlabels[v])}" for i, v in enumerate(chosen)]
        lines += [f"e {a} {b} {l}" for (a, b), l in sorted(es.items())]
        out.append("\n".join(lines) + "\n")
    return out


def config2_patterns(db: GraphDB, count: int = 16384, seed: int = 1000) -> List[str]:
    """The pattern list matched against the 20,000-graph database: `count`
    connected patterns of 2-7 vertices (a random growth tree inside a random
    graph plus each other edge among the chosen vertices with probability
    1/2, labels copied), so every pattern has at least one embedding."""
    return sample_patterns(db, count, 2, 7, seed=seed)


def config3_queries(db: GraphDB, count: int = 4096, seed: int = 1000) -> List[str]:
    """4,096 query patterns of 3-8 vertices, each a connected induced subgraph
    (every database edge among the chosen vertices kept) of a random graph of
    `db`, so every query has at least one embedding."""
    return sample_patterns(db, count, 3, 8, seed=seed, p_extra=1.0)


def _sorted_unique(x: np.ndarray) -> np.ndarray:
    x = np.sort(x, kind="quicksort")
    if len(x) == 0:
        return x
    keep = np.empty(len(x), dtype=bool)
    keep[0] = True
    np.not_equal(x[1:], x[:-1], out=keep[1:])
    return x[keep]


def rmat_graph(scale: int, num_edges: int, vlabel_k: int, vlabel_zipf: Optional[float], seed: int,
               a: float = 0.57, b: float = 0.19, c: float = 0.19, name: str = "rmat") -> GraphDB:
    """One R-MAT graph (Chakrabarti et al.): 2**scale vertices, each edge's
    endpoints chosen bit by bit from the quadrant probabilities (a, b, c,
    1-a-b-c); self-loops and duplicate edges dropped and edges redrawn until
    `num_edges` distinct undirected edges exist.  Vertex labels Zipf over
    `vlabel_k` labels (uniform when vlabel_zipf is None); one edge label.
    Returned as a one-graph database (first = [1, V + 1])."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    ta, tab, tabc = int(a * 65536), int((a + b) * 65536), int((a + b + c) * 65536)
    keys = np.empty(0, dtype=np.uint64)
    for _ in range(64):
        need = num_edges - len(keys)
        if need <= 0:
            break
        m = int(need * 1.2) + 1024
        src = np.zeros(m, dtype=np.uint32)
        dst = np.zeros(m, dtype=np.uint32)
        for _lvl in range(scale):
            # quadrant q in 0..3 = (src bit, dst bit) from one 16-bit draw
            r = rng.integers(0, 65536, size=m, dtype=np.uint16)
            q = (r >= ta).astype(np.uint8)
            q += r >= tab
            q += r >= tabc
            src <<= 1
            dst <<= 1
            src |= q >> 1
            dst |= q & 1
        ok = src != dst
        lo = np.minimum(src[ok], dst[ok]).astype(np.uint64)
        hi = np.maximum(src[ok], dst[ok]).astype(np.uint64)
        keys = _sorted_unique(np.concatenate([keys, (lo << np.uint64(32)) | hi]))
    if len(keys) > num_edges:  # drop a seeded random surplus
        keys = np.sort(keys[rng.permutation(len(keys))[:num_edges]])
    src = ((keys >> np.uint64(32)) + np.uint64(1)).astype(np.uint32)
    dst = ((keys & np.uint64(0xffffffff)) + np.uint64(1)).astype(np.uint32)
    if vlabel_zipf is None:
        vl = rng.integers(1, vlabel_k + 1, size=n).astype(np.uint32)
    else:
        vl = zipf_labels(rng, n, vlabel_k, vlabel_zipf)
    vlabels = np.zeros(n + 1, dtype=np.uint32)
    vlabels[1:] = vl
    el = np.ones(len(src), dtype=np.uint32)
    first = np.array([1, n + 1], dtype=np.int64)
    return GraphDB(name, vlabels, src, dst, el, first,
                   dict(scale=scale, edges=num_edges, a=a, b=b, c=c, vertex_labels=vlabel_k,
                        vertex_label_zipf=vlabel_zipf, seed=seed))


def config4(seed: int = 4, scale: int = 22, num_edges: int = 64 << 20) -> GraphDB:
    """R-MAT (a=0.57, b=c=0.19) with 2^22 (~4M) vertices and 64M undirected
    edges after dedup, 32 vertex labels Zipf(1.0), one edge label."""
    return rmat_graph(scale, num_edges, 32, 1.0, seed, name="config4")
