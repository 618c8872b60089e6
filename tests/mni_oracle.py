"""MNI (minimum image-based) support oracles for one data graph — test infrastructure.

The reference has no support notion; it enumerates the embeddings of one
pattern (cpumine, src/cpumine.cpp:54-584), symmetry broken by the planner's
automorphism restrictions (src/genMatchOrderCPU.cpp:467-506).  Two
independent ways to get a pattern's image sets from that:

* `mni_from_rows`: the oracle's cpumine rows (one row per automorphism class
  of embeddings) with the columns of each automorphism orbit unioned — the
  image set of u is the set of values in the columns of u's orbit;
* `brute_mni_mine`: every connected edge subset of up to K edges of a tiny
  graph, mapped onto its canonical pattern by every label- and
  edge-preserving vertex order that gives the canonical code (each such
  order is one embedding); image sets collected per canonical vertex.

MNI = the smallest image set over the pattern's vertices.

Parity unpinned against the reference: it has no MNI.  The rows-based form
rests on the oracle's cpumine restatement, which is pinned against the
reference's own binaries (tests/golden).
"""
from __future__ import annotations

import itertools
from collections import defaultdict
from typing import Dict, List, Tuple

import numpy as np


def parse_pattern(text: str) -> Tuple[List[int], Dict[Tuple[int, int], int]]:
    vl: Dict[int, int] = {}
    el: Dict[Tuple[int, int], int] = {}
    for line in text.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            vl[int(t[1])] = int(t[2])
        elif t[0] == "e":
            a, b, l = int(t[1]), int(t[2]), int(t[3])
            el[(a, b)] = el[(b, a)] = l
    return [vl[i] for i in range(len(vl))], el


def orbits(vl: List[int], el: Dict[Tuple[int, int], int]) -> List[int]:
    """orbit[v] = smallest vertex of v's automorphism orbit."""
    n = len(vl)
    orb = list(range(n))
    for perm in itertools.permutations(range(n)):
        if any(vl[perm[i]] != vl[i] for i in range(n)):
            continue
        if all(el.get((perm[a], perm[b])) == l for (a, b), l in el.items()):
            for v in range(n):
                orb[v] = min(orb[v], perm[v])
    # close under transitivity
    changed = True
    while changed:
        changed = False
        for v in range(n):
            if orb[orb[v]] < orb[v]:
                orb[v] = orb[orb[v]]
                changed = True
    return orb


def plan_columns(plan_text: str) -> List[int]:
    """Query vertex of each output column: the init phase's source, then every
    phase's new end vertices in pair order (the reference's posOfVisitedV,
    src/gpumine.cpp:158)."""
    cols: List[int] = []
    for line in plan_text.splitlines():
        t = line.split()
        if not t or t[0] != "phase":
            continue
        npairs = int(t[4])
        pairs = [int(x) for x in t[5:5 + 2 * npairs]]
        for i in range(npairs):
            s, e = pairs[2 * i], pairs[2 * i + 1]
            if not cols:
                cols.append(s)
            if t[2] == "E" and e not in cols:
                cols.append(e)
    return cols


def mni_from_rows(oracle, og, text: str, cap: int = 0) -> int:
    """min(MNI, cap) of `text` from the oracle's rows (cap 0 = exact)."""
    vl, el = parse_pattern(text)
    rows, _ = oracle.match(og, text)
    if rows.size == 0:
        return 0
    cols = plan_columns(oracle.plan(text))
    col_of = {v: i for i, v in enumerate(cols)}
    orb = orbits(vl, el)
    best = None
    for r in set(orb):
        members = [v for v in range(len(vl)) if orb[v] == r]
        images = np.unique(np.concatenate([rows[:, col_of[v]] for v in members]))
        best = len(images) if best is None else min(best, len(images))
    return min(best, cap) if cap else best


def _canon_all(vlabels: Tuple[int, ...], edges: Tuple[Tuple[int, int, int], ...]):
    """(canonical code, every vertex order giving it)."""
    n = len(vlabels)
    adj = {}
    for a, b, l in edges:
        adj[(a, b)] = adj[(b, a)] = l
    best, orders = None, []
    for perm in itertools.permutations(range(n)):  # perm[i] = original vertex at canonical position i
        code = tuple(vlabels[perm[i]] for i in range(n)) + tuple(
            adj.get((perm[i], perm[j]), 0) for i in range(n) for j in range(i + 1, n))
        if best is None or code < best:
            best, orders = code, [perm]
        elif code == best:
            orders.append(perm)
    return (n,) + best, orders


def brute_mni_mine(db, max_edges: int) -> Dict[Tuple, int]:
    """{canonical code: exact MNI} for every connected pattern of up to
    max_edges edges occurring in the one graph of `db` (a GraphDB)."""
    edges = list(zip(db.src.tolist(), db.dst.tolist(), db.elabels.tolist()))
    inc = defaultdict(list)
    for i, (a, b, _) in enumerate(edges):
        inc[a].append(i)
        inc[b].append(i)
    images: Dict[Tuple, List[set]] = {}
    frontier = {frozenset([i]) for i in range(len(edges))}
    seen = set(frontier)
    for k in range(1, max_edges + 1):
        for es in frontier:
            vs = sorted({x for i in es for x in edges[i][:2]})
            idx = {v: j for j, v in enumerate(vs)}
            labels = tuple(int(db.vlabels[v]) for v in vs)
            pe = tuple((idx[edges[i][0]], idx[edges[i][1]], edges[i][2]) for i in sorted(es))
            code, orders = _canon_all(labels, pe)
            sets = images.setdefault(code, [set() for _ in vs])
            for perm in orders:
                for pos in range(len(vs)):
                    sets[pos].add(vs[perm[pos]])
        if k == max_edges:
            break
        nxt = set()
        for es in frontier:
            for v in {x for i in es for x in edges[i][:2]}:
                for i in inc[v]:
                    if i not in es:
                        nes = es | {i}
                        if nes not in seen:
                            seen.add(nes)
                            nxt.add(nes)
        frontier = nxt
    return {code: min(len(s) for s in sets) for code, sets in images.items()}
