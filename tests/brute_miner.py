"""Brute-force frequent-pattern miner for tiny graph databases (test oracle).

Enumerates, in every graph, every connected edge subset of up to K edges,
turns each into a pattern (vertex labels + edge labels) and canonicalises it
by trying every vertex permutation; the support of a pattern is the number of
graphs in which it occurs.  Independent of the product's pattern growth and
canonical codes: use it only on databases of a few hundred small graphs.
"""
from __future__ import annotations

import itertools
from collections import defaultdict
from typing import Dict, FrozenSet, List, Tuple


def canon(vlabels: Tuple[int, ...], edges: Tuple[Tuple[int, int, int], ...]) -> Tuple:
    n = len(vlabels)
    adj = {}
    for a, b, l in edges:
        adj[(a, b)] = adj[(b, a)] = l
    best = None
    for perm in itertools.permutations(range(n)):  # perm[i] = original vertex at position i
        code = tuple(vlabels[perm[i]] for i in range(n)) + tuple(
            adj.get((perm[i], perm[j]), 0) for i in range(n) for j in range(i + 1, n))
        if best is None or code < best:
            best = code
    return (n,) + best


def pattern_from_text(text: str) -> Tuple:
    vl, es = {}, []
    for line in text.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            vl[int(t[1])] = int(t[2])
        elif t[0] == "e":
            es.append((int(t[1]), int(t[2]), int(t[3])))
    labels = tuple(vl[i] for i in range(len(vl)))
    return canon(labels, tuple(es))


def mine(db, max_edges: int, min_support: int) -> Dict[Tuple, int]:
    """db: geneva_b200.workloads.GraphDB.  Returns {canonical code: support}."""
    G = len(db.first) - 1
    g_of = db.graph_of(db.src.astype("int64"))
    by_graph: Dict[int, List[Tuple[int, int, int]]] = defaultdict(list)
    for a, b, l, g in zip(db.src.tolist(), db.dst.tolist(), db.elabels.tolist(), g_of.tolist()):
        by_graph[g].append((a, b, l))
    support: Dict[Tuple, int] = defaultdict(int)
    for g in range(G):
        edges = by_graph.get(g, [])
        inc = defaultdict(list)
        for i, (a, b, _) in enumerate(edges):
            inc[a].append(i)
            inc[b].append(i)
        seen: set = set()
        frontier = {frozenset([i]) for i in range(len(edges))}
        found = set()
        for k in range(1, max_edges + 1):
            for es in frontier:
                vs = sorted({x for i in es for x in edges[i][:2]})
                idx = {v: j for j, v in enumerate(vs)}
                labels = tuple(int(db.vlabels[v]) for v in vs)
                pe = tuple((idx[edges[i][0]], idx[edges[i][1]], edges[i][2]) for i in sorted(es))
                found.add(canon(labels, pe))
            if k == max_edges:
                break
            nxt = set()
            for es in frontier:
                vs = {x for i in es for x in edges[i][:2]}
                for v in vs:
                    for i in inc[v]:
                        if i not in es:
                            nes = es | {i}
                            if nes not in seen:
                                seen.add(nes)
                                nxt.add(nes)
            frontier = nxt
        for c in found:
            support[c] += 1
    return {c: s for c, s in support.items() if s >= min_support}


def build_native(workdir) -> str:
    """Compiles tests/brute_mine.cpp (the same definition in C++, for databases
    of a thousand graphs) into workdir; returns the executable's path."""
    import shutil
    import subprocess
    from pathlib import Path
    exe = Path(workdir) / "brute_mine"
    if not exe.exists():
        cxx = shutil.which("g++") or "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-o", str(exe), str(Path(__file__).with_name("brute_mine.cpp"))],
                       check=True, capture_output=True, text=True)
    return str(exe)


def mine_native(db, max_edges: int, min_support: int, exe: str, workdir) -> Dict[Tuple, int]:
    """mine() computed by the C++ brute force: {canonical code: support}."""
    import subprocess
    from pathlib import Path
    inp = Path(workdir) / f"brute_{db.name}.txt"
    with open(inp, "w") as f:
        V = len(db.vlabels) - 1
        G = len(db.first) - 1
        f.write(f"{V} {len(db.src)} {G}\n")
        f.write(" ".join(map(str, db.vlabels[1:].tolist())) + "\n")
        for a, b, l in zip(db.src.tolist(), db.dst.tolist(), db.elabels.tolist()):
            f.write(f"{a} {b} {l}\n")
        f.write(" ".join(map(str, db.first.tolist())) + "\n")
    r = subprocess.run([exe, str(inp), str(max_edges), str(min_support)], capture_output=True, text=True, check=True)
    out: Dict[Tuple, int] = {}
    for line in r.stdout.splitlines():
        t = list(map(int, line.split()))
        out[tuple(t[1:])] = t[0]
    return out
