"""ctypes front end of the CPU oracle (oracle/liboracle.so) — test infrastructure."""
from __future__ import annotations

import ctypes
import hashlib
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"


def rows_digest(rows: np.ndarray):
    """(distinct row count, sha256 of the sorted distinct rows as little-endian uint32)."""
    if rows.size == 0:
        return 0, hashlib.sha256(b"").hexdigest()
    u = np.unique(np.ascontiguousarray(rows, dtype=np.uint32), axis=0)
    return int(u.shape[0]), hashlib.sha256(np.ascontiguousarray(u).astype("<u4").tobytes()).hexdigest()


class Oracle:
    _inst = None

    @classmethod
    def get(cls) -> "Oracle":
        if cls._inst is None:
            so = ORACLE_DIR / "liboracle.so"
            src = [ORACLE_DIR / "geneva_oracle.cpp", ORACLE_DIR / "geneva_oracle.h"]
            if not so.exists() or any(s.stat().st_mtime > so.stat().st_mtime for s in src):
                subprocess.run(["make", "-C", str(ORACLE_DIR), "liboracle.so"], check=True,
                               capture_output=True)
            cls._inst = cls(so)
        return cls._inst

    def __init__(self, so: Path):
        lib = ctypes.CDLL(str(so))
        vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
        P = ctypes.POINTER
        lib.oracle_graph_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P(vp)]
        lib.oracle_graph_from_edges.argtypes = [vp, u32, vp, vp, vp, u64, P(vp)]
        lib.oracle_graph_free.argtypes = [vp]
        lib.oracle_plan.argtypes = [ctypes.c_char_p, ctypes.c_char_p, sz]
        lib.oracle_plan.restype = sz
        lib.oracle_match.argtypes = [vp, ctypes.c_char_p, P(P(u32)), P(u64), P(ctypes.c_int), P(u64),
                                     ctypes.c_int, P(ctypes.c_int)]
        lib.oracle_count.argtypes = [vp, ctypes.c_char_p, P(u64)]
        lib.oracle_count_capped.argtypes = [vp, ctypes.c_char_p, u64, P(u64)]
        lib.oracle_graph_counts.argtypes = [vp, ctypes.c_char_p, vp, u32, vp, P(u64)]
        lib.oracle_free.argtypes = [vp]
        lib.oracle_last_error.restype = ctypes.c_char_p
        lib.oracle_mni_graph_from_edges.argtypes = [vp, u32, vp, vp, vp, u64, P(vp)]
        lib.oracle_mni_graph_free.argtypes = [vp]
        lib.oracle_mni.argtypes = [vp, ctypes.c_char_p, u32, P(u32), P(u64)]
        self.lib = lib

    def load(self, mygraph, metadata):
        h = ctypes.c_void_p()
        if self.lib.oracle_graph_load(str(mygraph).encode(), str(metadata).encode(), ctypes.byref(h)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return h

    def from_edges(self, vlabels, src, dst, elabel):
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        e = np.ascontiguousarray(elabel, dtype=np.uint32)
        h = ctypes.c_void_p()
        self.lib.oracle_graph_from_edges(vl.ctypes.data, len(vl) - 1, s.ctypes.data, d.ctypes.data,
                                         e.ctypes.data, len(s), ctypes.byref(h))
        return h

    def free(self, g):
        self.lib.oracle_graph_free(g)

    def plan(self, query_text: str) -> str:
        n = self.lib.oracle_plan(query_text.encode(), None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        self.lib.oracle_plan(query_text.encode(), buf, n + 1)
        return buf.value.decode()

    def match(self, g, query_text: str):
        """-> (rows [n, width] uint32, per-phase row counts)"""
        rows_p = ctypes.POINTER(ctypes.c_uint32)()
        n = ctypes.c_uint64()
        w = ctypes.c_int()
        ph = (ctypes.c_uint64 * 64)()
        nph = ctypes.c_int()
        if self.lib.oracle_match(g, query_text.encode(), ctypes.byref(rows_p), ctypes.byref(n), ctypes.byref(w),
                                 ph, 64, ctypes.byref(nph)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        cnt = n.value * w.value
        arr = np.ctypeslib.as_array(rows_p, shape=(max(cnt, 1),))[:cnt].copy().reshape(n.value, w.value)
        self.lib.oracle_free(ctypes.cast(rows_p, ctypes.c_void_p))
        return arr, [int(x) for x in ph[:nph.value]]

    def count(self, g, query_text: str, cap_rows: int = 0):
        """Embedding count, or None when a frontier passes about cap_rows rows."""
        n = ctypes.c_uint64()
        st = self.lib.oracle_count_capped(g, query_text.encode(), cap_rows, ctypes.byref(n))
        if st == 2:
            return None
        if st:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return int(n.value)

    def graph_counts(self, g, query_text: str, first):
        """-> (embeddings per graph [G] uint64, support) for a graph database
        whose graph i owns the vertex ids [first[i], first[i+1])."""
        f = np.ascontiguousarray(first, dtype=np.int64)
        G = len(f) - 1
        out = np.zeros(max(G, 1), dtype=np.uint64)
        n = ctypes.c_uint64()
        if self.lib.oracle_graph_counts(g, query_text.encode(), f.ctypes.data, G, out.ctypes.data, ctypes.byref(n)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        out = out[:G]
        return out, int((out > 0).sum())

    def many_graph_counts(self, g, texts, first, threads: int = 0):
        """graph_counts of every text on a thread pool (the calls release the
        interpreter lock): -> (counts [n] uint64, supports [n] uint32)."""
        import os
        from concurrent.futures import ThreadPoolExecutor
        threads = threads or (os.cpu_count() or 1)
        with ThreadPoolExecutor(max_workers=threads) as ex:
            res = list(ex.map(lambda t: self.graph_counts(g, t, first), texts))
        counts = np.array([int(c.sum()) for c, _ in res], dtype=np.uint64)
        sup = np.array([s for _, s in res], dtype=np.uint32)
        return counts, sup, [c for c, _ in res]

    # ---- MNI on one data graph (CPU existence search) ----
    def mni_graph(self, vlabels, src, dst, elabel):
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        e = np.ascontiguousarray(elabel, dtype=np.uint32)
        h = ctypes.c_void_p()
        self.lib.oracle_mni_graph_from_edges(vl.ctypes.data, len(vl) - 1, s.ctypes.data, d.ctypes.data,
                                             e.ctypes.data, len(s), ctypes.byref(h))
        return h

    def mni_graph_free(self, g):
        self.lib.oracle_mni_graph_free(g)

    def mni(self, g, text: str, cap: int = 0):
        """-> (min(MNI, cap) (cap 0 = exact), rooted searches run)"""
        sup = ctypes.c_uint32()
        ns = ctypes.c_uint64()
        if self.lib.oracle_mni(g, text.encode(), cap, ctypes.byref(sup), ctypes.byref(ns)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return int(sup.value), int(ns.value)
