"""Host-side mirror of the Geneva matching path over the native C ABI.

The reference exposes its GPU path as C++ functions and a CLI:

    loadDataBase(mygraph, metadata)            src/loadDataBase.cpp:309
    genMatchOrder(query, ...)                  src/genMatchOrder.cpp:672
    genMatchOrderSingleV(query, ...)           src/genMatchOrderSingleV.cpp:678
    gpumine <mygraph> <metadata> <query>       src/gpumine.cpp:866
    gpumineSV <mygraph> <metadata> <query>     src/gpumine_singleV.cpp:722

This module offers the same operations with the same argument meaning on top
of ``libgeneva.so`` (include/geneva.h), loaded with ctypes.  The CUDA kernels
are the only compute path: if the library is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from collections import abc as _abc
from dataclasses import dataclass
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "GenevaError", "Database", "probe_graph", "convert_g", "batch_count", "batch_count_texts", "kernel_launches", "mine", "mine_host", "mni_support", "MinedPatterns", "MinedPattern", "Plan", "Result", "MODE_DV", "MODE_SV", "library", "library_path",
    "loadDataBase", "genMatchOrder", "genMatchOrderSingleV", "match", "gpumine", "gpumineSV",
]

MODE_DV = 0
MODE_SV = 1

_PKG = Path(__file__).resolve().parent
_LIB = None


class GenevaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def library_path() -> Path:
    return _PKG / "lib" / "libgeneva.so"


class _DbInfo(ctypes.Structure):
    _fields_ = [("max_vertex_id", ctypes.c_uint32), ("num_vertex_labels", ctypes.c_uint32),
                ("num_partitions", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("num_adjacency", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64)]


class _MatchOpts(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("budget_bytes", ctypes.c_uint64),
                ("count_only", ctypes.c_int), ("profile", ctypes.c_int)]


class _KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 24), ("launches", ctypes.c_uint64), ("ms", ctypes.c_double),
                ("bytes", ctypes.c_double), ("rows", ctypes.c_double)]


REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64),
                             ctypes.c_uint64, ctypes.c_void_p)


EVAL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64,
                           ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p)

SUPPORT_GRAPHS = 0
SUPPORT_MNI = 1


class _MineOpts(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("budget_bytes", ctypes.c_uint64), ("max_edges", ctypes.c_uint32),
                ("min_support", ctypes.c_uint32), ("batch_limit", ctypes.c_uint32), ("profile", ctypes.c_uint32),
                ("reduce", REDUCE_FN), ("reduce_user", ctypes.c_void_p), ("support_mode", ctypes.c_uint32),
                ("mni_cap", ctypes.c_uint32), ("cancel", ctypes.c_void_p), ("sm_percent", ctypes.c_uint32),
                ("host_threads", ctypes.c_uint32)]


class _MineStats(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_uint64), ("frequent", ctypes.c_uint64), ("embeddings", ctypes.c_uint64),
                ("levels", ctypes.c_uint64), ("pruned", ctypes.c_uint64), ("gpu_ms", ctypes.c_double),
                ("host_ms", ctypes.c_double), ("gen_ms", ctypes.c_double), ("plan_ms", ctypes.c_double),
                ("eval_ms", ctypes.c_double), ("merge_ms", ctypes.c_double), ("submit_ms", ctypes.c_double),
                ("round_host_ms", ctypes.c_double), ("wait_ms", ctypes.c_double), ("mni_tasks", ctypes.c_uint64),
                ("mni_rounds", ctypes.c_uint64)]


class _MniOpts(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("cap", ctypes.c_uint32), ("plain", ctypes.c_int),
                ("profile", ctypes.c_int), ("flags", ctypes.c_int)]


BATCH_PLAN_ON_DEVICE = 1
BATCH_HOST_ROUNDS = 2
BATCH_DEVICE_ROUNDS = 4


class _BatchOpts(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("budget_bytes", ctypes.c_uint64), ("profile", ctypes.c_int),
                ("flags", ctypes.c_int)]


class _Tuning(ctypes.Structure):
    _fields_ = [("rows_per_item", ctypes.c_uint32), ("hub", ctypes.c_uint32), ("ms", ctypes.c_double),
                ("default_ms", ctypes.c_double), ("tried", ctypes.c_uint32), ("round_region_mb", ctypes.c_uint32)]


class _BatchStats(ctypes.Structure):
    _fields_ = [("gpu_ms", ctypes.c_double), ("rounds", ctypes.c_uint64), ("splits", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("trie_nodes", ctypes.c_uint64), ("kernels", _KernelStat * 5),
                ("lower_ms", ctypes.c_double), ("submit_ms", ctypes.c_double), ("round_host_ms", ctypes.c_double),
                ("wait_ms", ctypes.c_double), ("session_ms", ctypes.c_double),
                ("round_phase_ms", ctypes.c_double * 5), ("timeline_ms", ctypes.c_double * 9),
                ("device_rounds", ctypes.c_uint64)]


class _MniStats(ctypes.Structure):
    _fields_ = [("gpu_ms", ctypes.c_double), ("rounds", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("tasks", ctypes.c_uint64), ("seeds", ctypes.c_uint64), ("roots", ctypes.c_uint64),
                ("found", ctypes.c_uint64), ("kernel", _KernelStat)]


def _declare(lib):
    P = ctypes.POINTER
    vp, u32, u64, i32, sz, cp = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                                 ctypes.c_size_t, ctypes.c_char_p)
    sig = {
        "gva_last_error": (cp, []),
        "gva_status_string": (cp, [i32]),
        "gva_version": (cp, []),
        "gva_kernel_launches": (u64, []),
        "gva_result_kernel_stats": (i32, [vp, P(_KernelStat), i32]),
        "gva_db_load": (i32, [cp, cp, i32, P(vp)]),
        "gva_db_from_edges": (i32, [vp, u32, vp, vp, vp, u64, i32, P(vp)]),
        "gva_db_get_info": (i32, [vp, P(_DbInfo)]),
        "gva_db_warnings": (cp, [vp]),
        "gva_graph_probe": (i32, [cp, cp, P(_DbInfo), ctypes.c_char_p, sz]),
        "gva_db_free": (None, [vp]),
        "gva_plan_from_file": (i32, [cp, i32, P(vp)]),
        "gva_plan_from_text": (i32, [cp, i32, P(vp)]),
        "gva_plan_batch": (i32, [vp, i32, i32, vp, vp]),
        "gva_plan_describe": (sz, [vp, ctypes.c_char_p, sz]),
        "gva_plan_num_phases": (i32, [vp]),
        "gva_plan_num_vertices": (i32, [vp]),
        "gva_plan_column_vertices": (i32, [vp, P(u32), i32]),
        "gva_plan_free": (None, [vp]),
        "gva_match": (i32, [vp, vp, P(_MatchOpts), P(vp)]),
        "gva_result_num_rows": (u64, [vp]),
        "gva_result_num_columns": (i32, [vp]),
        "gva_result_phase_rows": (i32, [vp, P(u64), i32]),
        "gva_result_device_rows": (vp, [vp]),
        "gva_result_copy_rows": (i32, [vp, vp, u64, u64]),
        "gva_result_write_text": (i32, [vp, cp]),
        "gva_result_gpu_ms": (ctypes.c_double, [vp]),
        "gva_result_free": (None, [vp]),
        "gva_plan_num_steps": (i32, [vp, vp]),
        "gva_plan_step_width_in": (i32, [vp, vp, i32]),
        "gva_plan_step_width_out": (i32, [vp, vp, i32]),
        "gva_step_scratch_bytes": (sz, [u64]),
        "gva_step_run": (i32, [vp, vp, i32, vp, u64, vp, u64, P(u64), vp, sz, vp]),
        "gva_db_set_graphs": (i32, [vp, vp, u32]),
        "gva_convert_g": (i32, [cp, cp, cp, cp]),
        "gva_mine": (i32, [vp, P(_MineOpts), P(vp)]),
        "gva_plan_batch_device": (i32, [i32, vp, i32, vp, vp]),
        "gva_batch_count_texts": (i32, [vp, vp, i32, i32, P(_BatchOpts), vp, vp, vp, vp, P(_BatchStats)]),
        "gva_db_get_tuning": (i32, [vp, P(_Tuning)]),
        "gva_db_set_tuning": (i32, [vp, P(_Tuning)]),
        "gva_db_autotune": (i32, [vp, vp, i32, vp, P(_Tuning)]),
        "gva_mine_host": (i32, [u32, vp, u32, vp, u32, u32, u32, EVAL_FN, vp, REDUCE_FN, vp, P(vp)]),
        "gva_mine_num_patterns": (i32, [vp]),
        "gva_mine_get": (i32, [vp, i32, P(u32), P(u32), P(u64)]),
        "gva_mine_pattern_text": (sz, [vp, i32, ctypes.c_char_p, sz]),
        "gva_mine_get_stats": (i32, [vp, P(_MineStats)]),
        "gva_mine_free": (None, [vp]),
        "gva_mine_kernel_stats": (i32, [vp, P(_KernelStat), i32]),
        "gva_mine_export": (sz, [vp, vp, sz, vp, vp, vp, vp]),
        "gva_batch_count": (i32, [vp, vp, i32, P(_BatchOpts), vp, vp, vp, P(_BatchStats)]),
        "gva_mni_support": (i32, [vp, vp, i32, P(_MniOpts), vp, P(_MniStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def library():
    """The loaded native library (built by geneva_b200.build)."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not path.exists():
            raise GenevaError(6, f"native library missing: {path} (run python -m geneva_b200.build)")
        _LIB = _declare(ctypes.CDLL(str(path)))
    return _LIB


def _check(status: int):
    if status != 0:
        lib = library()
        raise GenevaError(status, lib.gva_last_error().decode())


class Database:
    """Device-resident database (gva_db)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)
        self.num_graphs = 0

    @classmethod
    def load(cls, mygraph: str, metadata: str, device: int = 0) -> "Database":
        h = ctypes.c_void_p()
        _check(library().gva_db_load(str(mygraph).encode(), str(metadata).encode(), device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_edges(cls, vertex_labels, src, dst, edge_labels, device: int = 0) -> "Database":
        vl = np.ascontiguousarray(vertex_labels, dtype=np.uint32)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        el = np.ascontiguousarray(edge_labels, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(library().gva_db_from_edges(vl.ctypes.data, len(vl) - 1, s.ctypes.data, d.ctypes.data,
                                           el.ctypes.data, len(s), device, ctypes.byref(h)))
        return cls(h.value)

    def info(self) -> dict:
        i = _DbInfo()
        _check(library().gva_db_get_info(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _DbInfo._fields_ if f != "reserved"}

    @property
    def warnings(self) -> str:
        return library().gva_db_warnings(self._h).decode()

    def set_graphs(self, first) -> None:
        """Declare graph g as vertex ids [first[g], first[g+1]) (gva_db_set_graphs)."""
        f = np.ascontiguousarray(first, dtype=np.uint64)
        _check(library().gva_db_set_graphs(self._h, f.ctypes.data, len(f) - 1))
        self.num_graphs = len(f) - 1

    @property
    def tuning(self) -> dict:
        """Launch shape of the batched engine's round kernels on this database."""
        t = _Tuning()
        _check(library().gva_db_get_tuning(self._h, ctypes.byref(t)))
        return {"rows_per_item": int(t.rows_per_item), "hub": int(t.hub),
                "round_region_mb": int(t.round_region_mb)}

    def set_tuning(self, rows_per_item: int, hub: int, round_region_mb: int = 0) -> None:
        """round_region_mb: MiB of each frontier region of device-scheduled
        rounds (0 keeps the current size)."""
        t = _Tuning(rows_per_item, hub, 0.0, 0.0, 0, round_region_mb)
        _check(library().gva_db_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, plans, stream: Optional[int] = None) -> dict:
        """Times a calibration batch under each candidate launch shape and keeps
        the fastest (gva_db_autotune)."""
        arr = _plan_handles(plans)
        t = _Tuning()
        _check(library().gva_db_autotune(self._h, arr.ctypes.data, len(plans), stream or None, ctypes.byref(t)))
        return {"rows_per_item": int(t.rows_per_item), "hub": int(t.hub), "ms": float(t.ms),
                "default_ms": float(t.default_ms), "shapes_tried": int(t.tried)}

    def close(self):
        if self._h:
            library().gva_db_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def convert_g(g_path: str, out_prefix: str) -> None:
    """.g -> <out_prefix>.mygraph/.metadata/.reorder, as tools/genDatabase.cpp writes them."""
    p = str(out_prefix)
    _check(library().gva_convert_g(str(g_path).encode(), (p + ".mygraph").encode(), (p + ".metadata").encode(),
                                   (p + ".reorder").encode()))


def probe_graph(mygraph: str, metadata: str) -> dict:
    """Host-only parse of a .mygraph/.metadata pair (gva_graph_probe)."""
    i = _DbInfo()
    buf = ctypes.create_string_buffer(4096)
    _check(library().gva_graph_probe(str(mygraph).encode(), str(metadata).encode(), ctypes.byref(i), buf, 4096))
    d = {f: getattr(i, f) for f, _ in _DbInfo._fields_ if f != "reserved"}
    d["warnings"] = buf.value.decode()
    return d


def _text_array(texts: Sequence[str]):
    """The texts as one NUL-separated buffer and an array of pointers into
    it (what a const char* const* parameter takes), built without a
    per-text ctypes object.  Returns (keep-alive buffer, uint64 pointers)."""
    n = len(texts)
    if n == 0:
        return b"\0", np.zeros(1, dtype=np.uint64)
    buf = ("\0".join(texts) + "\0").encode()
    if buf.count(b"\0") != n:
        raise ValueError("query texts must not contain NUL characters")
    lens = np.fromiter(map(len, texts), dtype=np.int64, count=n)
    if len(buf) == int(lens.sum()) + n:  # one byte per character: offsets from the lengths
        starts = np.cumsum(lens + 1) - (lens + 1)
    else:
        ends = np.flatnonzero(np.frombuffer(buf, dtype=np.uint8) == 0)
        starts = np.empty(n, dtype=np.int64)
        starts[0] = 0
        starts[1:] = ends[:-1] + 1
    base = ctypes.cast(ctypes.c_char_p(buf), ctypes.c_void_p).value
    return buf, starts.astype(np.uint64) + np.uint64(base)


def _plan_handles(plans) -> np.ndarray:
    """Plan handles as a uint64 array: kept by a PlanBatch, else gathered."""
    h = getattr(plans, "_harr", None)
    if h is not None:
        return h
    return np.array([p._h.value or 0 for p in plans] or [0], dtype=np.uint64)


class Plan:
    """Match order + restrictions (gva_plan)."""

    def __init__(self, handle, batch=None):
        self._h = ctypes.c_void_p(handle)
        self._batch = batch  # the PlanBatch owning the handle, if any

    @classmethod
    def from_text(cls, text: str, mode: int = MODE_DV) -> "Plan":
        h = ctypes.c_void_p()
        _check(library().gva_plan_from_text(text.encode(), mode, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def _batch(cls, call, texts: Sequence[str]) -> "PlanBatch":
        n = len(texts)
        buf, ptrs = _text_array(texts)
        out = np.zeros(max(n, 1), dtype=np.uint64)
        st = np.zeros(max(n, 1), dtype=np.int32)
        rc = call(ptrs.ctypes.data, n, out.ctypes.data, st.ctypes.data)
        batch = PlanBatch(out[:n])
        if rc:
            msg = library().gva_last_error().decode()
            batch.close()
            raise GenevaError(rc, msg)
        return batch

    @classmethod
    def batch_from_texts(cls, texts: Sequence[str], mode: int = MODE_DV) -> "PlanBatch":
        """Plans many queries in one call on the host's cores (gva_plan_batch)."""
        return cls._batch(lambda t, n, o, s: library().gva_plan_batch(t, n, mode, o, s), texts)

    @classmethod
    def batch_from_texts_device(cls, texts: Sequence[str], device: int = 0) -> "PlanBatch":
        """DV plans of many queries computed by the device planner
        (gva_plan_batch_device); the same plans as batch_from_texts."""
        return cls._batch(lambda t, n, o, s: library().gva_plan_batch_device(device, t, n, o, s), texts)

    @classmethod
    def from_file(cls, path: str, mode: int = MODE_DV) -> "Plan":
        h = ctypes.c_void_p()
        _check(library().gva_plan_from_file(str(path).encode(), mode, ctypes.byref(h)))
        return cls(h.value)

    def describe(self) -> str:
        lib = library()
        n = lib.gva_plan_describe(self._h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib.gva_plan_describe(self._h, buf, n + 1)
        return buf.value.decode()

    @property
    def columns(self) -> List[int]:
        arr = (ctypes.c_uint32 * 32)()
        n = library().gva_plan_column_vertices(self._h, arr, 32)
        return list(arr[:n])

    @property
    def num_phases(self) -> int:
        return library().gva_plan_num_phases(self._h)

    def close(self):
        # a plan of a PlanBatch only lets go of its handle: the batch frees it
        if self._h and self._batch is None:
            library().gva_plan_free(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PlanBatch(tuple):
    """Plans made together (Plan.batch_from_texts): a tuple of Plan (None
    where a text failed to plan) that owns their handles and keeps them as one
    array, so batched calls take them without a per-plan conversion.  The
    handles are freed when the batch and every plan taken from it are gone,
    or by close()."""

    def __new__(cls, handles: np.ndarray):
        harr = np.array(handles, dtype=np.uint64)
        self = super().__new__(cls, [Plan(int(h)) if h else None for h in harr.tolist()])
        self._harr = harr
        for q in tuple.__iter__(self):
            if q is not None:
                q._batch = self
        return self

    def close(self):
        lib = library()
        for q in tuple.__iter__(self):
            if q is not None:
                q._h = ctypes.c_void_p()
        for h in self._harr.tolist():
            if h:
                lib.gva_plan_free(ctypes.c_void_p(h))
        self._harr = np.zeros(len(self._harr), dtype=np.uint64)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Result:
    """Final frontier on the device plus per-phase row counts (gva_result)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    @property
    def num_rows(self) -> int:
        return int(library().gva_result_num_rows(self._h))

    @property
    def num_columns(self) -> int:
        return int(library().gva_result_num_columns(self._h))

    @property
    def phase_rows(self) -> List[int]:
        arr = (ctypes.c_uint64 * 64)()
        n = library().gva_result_phase_rows(self._h, arr, 64)
        return [int(x) for x in arr[:n]]

    @property
    def gpu_ms(self) -> float:
        return float(library().gva_result_gpu_ms(self._h))

    def kernel_stats(self) -> dict:
        """Per-kernel {launches, ms, bytes} of a profiled match."""
        arr = (_KernelStat * 16)()
        n = library().gva_result_kernel_stats(self._h, arr, 16)
        return {arr[i].name.decode(): dict(launches=int(arr[i].launches), ms=float(arr[i].ms),
                                            bytes=float(arr[i].bytes), rows=float(arr[i].rows)) for i in range(n)}

    @property
    def device_ptr(self) -> Optional[int]:
        return library().gva_result_device_rows(self._h)

    def rows(self, first: int = 0, count: Optional[int] = None, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.num_rows - first if count is None else count
        w = self.num_columns
        if out is None:
            out = np.empty((n, w), dtype=np.uint32)
        if n:
            _check(library().gva_result_copy_rows(self._h, out.ctypes.data, first, n))
        return out

    def write_text(self, path: str):
        _check(library().gva_result_write_text(self._h, str(path).encode()))

    def close(self):
        if self._h:
            library().gva_result_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches() -> int:
    """Kernels launched by the native library in this process."""
    return int(library().gva_kernel_launches())


def match(db: Database, plan: Plan, stream: Optional[int] = None, budget_bytes: int = 0,
          count_only: bool = False, profile: bool = False) -> Result:
    """Runs every phase of `plan` on `db` (gva_match)."""
    o = _MatchOpts(stream or None, budget_bytes, 1 if count_only else 0, 1 if profile else 0)
    h = ctypes.c_void_p()
    _check(library().gva_match(db._h, plan._h, ctypes.byref(o), ctypes.byref(h)))
    return Result(h.value)


def batch_count(db: Database, plans: Sequence[Plan], stream: Optional[int] = None, budget_bytes: int = 0,
                graph_counts: bool = False, support: bool = False, profile: bool = False,
                host_rounds: bool = False, device_rounds: bool = False):
    """Counts embeddings of many plans in shared rounds (gva_batch_count).

    Returns (counts[n] uint64, per_graph, stats) where per_graph is the
    [n, num_graphs] uint64 count matrix when graph_counts, else the [n]
    uint32 supporting-graph counts when support, else None.  host_rounds /
    device_rounds: schedule every round on the host / on the device
    (GVA_BATCH_HOST_ROUNDS / GVA_BATCH_DEVICE_ROUNDS; default: on the device
    for a run in one piece, on the host for one split in halves)."""
    n = len(plans)
    arr = _plan_handles(plans)
    counts = np.zeros(n, dtype=np.uint64)
    gc = np.zeros((n, db.num_graphs), dtype=np.uint64) if graph_counts else None
    sup = np.zeros(n, dtype=np.uint32) if support else None
    o = _BatchOpts(stream or None, budget_bytes, 1 if profile else 0,
                   (BATCH_HOST_ROUNDS if host_rounds else 0) | (BATCH_DEVICE_ROUNDS if device_rounds else 0))
    st = _BatchStats()
    _check(library().gva_batch_count(db._h, arr.ctypes.data, n, ctypes.byref(o), counts.ctypes.data,
                                     gc.ctypes.data if gc is not None else None,
                                     sup.ctypes.data if sup is not None else None, ctypes.byref(st)))
    per_graph = gc if graph_counts else sup
    if graph_counts and support:
        per_graph = (gc, sup)
    return counts, per_graph, _batch_stats_dict(st)


def _batch_stats_dict(st) -> dict:
    return {"gpu_ms": st.gpu_ms, "rounds": int(st.rounds), "device_rounds": int(st.device_rounds),
            "splits": int(st.splits), "launches": int(st.launches),
            "trie_nodes": int(st.trie_nodes), "lower_ms": st.lower_ms, "submit_ms": st.submit_ms,
            "round_host_ms": st.round_host_ms, "wait_ms": st.wait_ms, "session_ms": st.session_ms,
            "round_phase_ms": [float(x) for x in st.round_phase_ms],
            "timeline_ms": [float(x) for x in st.timeline_ms],
            "kernels": {st.kernels[i].name.decode(): dict(launches=int(st.kernels[i].launches),
                                                          ms=float(st.kernels[i].ms), bytes=float(st.kernels[i].bytes),
                                                          rows=float(st.kernels[i].rows))
                        for i in range(5)}}


def batch_count_texts(db: Database, texts: Sequence[str], mode: int = MODE_DV, stream: Optional[int] = None,
                      budget_bytes: int = 0, graph_counts: bool = False, support: bool = False,
                      profile: bool = False, plan_on_device: bool = False):
    """Plans and counts query texts in one call (gva_batch_count_texts): no
    plan handles; plan_on_device plans them with the device planner.
    Returns (counts, per_graph, stats) as batch_count; a text that fails to
    plan raises GenevaError after the others were counted."""
    n = len(texts)
    buf, arr = _text_array(texts)
    counts = np.zeros(n, dtype=np.uint64)
    gc = np.zeros((n, db.num_graphs), dtype=np.uint64) if graph_counts else None
    sup = np.zeros(n, dtype=np.uint32) if support else None
    status = np.zeros(max(n, 1), dtype=np.int32)
    o = _BatchOpts(stream or None, budget_bytes, 1 if profile else 0, BATCH_PLAN_ON_DEVICE if plan_on_device else 0)
    st = _BatchStats()
    _check(library().gva_batch_count_texts(db._h, arr.ctypes.data, n, mode, ctypes.byref(o),
                                           counts.ctypes.data, gc.ctypes.data if gc is not None else None,
                                           sup.ctypes.data if sup is not None else None, status.ctypes.data,
                                           ctypes.byref(st)))
    per_graph = gc if graph_counts else sup
    if graph_counts and support:
        per_graph = (gc, sup)
    return counts, per_graph, _batch_stats_dict(st)


@dataclass
class MinedPattern:
    text: str
    edges: int
    support: int
    embeddings: int


class MinedPatterns(_abc.Sequence):
    """The patterns of one gva_mine call, copied out in one gva_mine_export:
    numpy arrays `edges`, `supports`, `embeddings` and the pattern texts,
    decoded one at a time on access (runs can yield tens of millions)."""

    def __init__(self, blob: np.ndarray, offsets: np.ndarray, edges: np.ndarray, supports: np.ndarray,
                 embeddings: np.ndarray):
        self._blob, self._off = blob, offsets
        self.edges, self.supports, self.embeddings = edges, supports, embeddings

    def __len__(self) -> int:
        return len(self.edges)

    @property
    def text_bytes(self) -> int:
        """Bytes of all pattern texts (without terminators)."""
        return len(self._blob) - len(self)

    def text(self, i: int) -> str:
        a = int(self._off[i])
        b = int(self._off[i + 1]) - 1 if i + 1 < len(self._off) else len(self._blob) - 1
        return self._blob[a:b].tobytes().decode()

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        return MinedPattern(self.text(i), int(self.edges[i]), int(self.supports[i]), int(self.embeddings[i]))


def mine(db: Database, max_edges: int, min_support: int, stream: Optional[int] = None, budget_bytes: int = 0,
         batch_limit: int = 0, profile: bool = False, reduce=None, support: str = "graphs", mni_cap: int = 0,
         cancel: Optional[ctypes.c_int] = None, sm_percent: int = 0, host_threads: int = 0):
    """Frequent connected patterns (gva_mine).

    support="graphs": a pattern's support is the number of database graphs
    holding an embedding (needs Database.set_graphs).  support="mni": the
    minimum image-based support on the whole data graph, reported as
    min(MNI, mni_cap) (mni_cap 0 = min_support, which decides frequency).
    `reduce(supports, embeddings)` (numpy uint32 / uint64 arrays, updated in
    place) combines each level's counts across processes holding disjoint
    graph shards (graph support only).  `cancel` (a ctypes.c_int another
    thread may set to 1) stops the run at its next batch or round boundary
    with GenevaError status 7.  sm_percent (MNI) caps the share of the SMs
    the search kernel fills and host_threads the host threads used (0 = all),
    so that a server's other work keeps running.  Returns (patterns, stats);
    stats["kernels"] is filled when profiling."""
    lib = library()
    cb = _reduce_callback(reduce)
    mode = {"graphs": SUPPORT_GRAPHS, "mni": SUPPORT_MNI}[support]
    o = _MineOpts(stream or None, budget_bytes, max_edges, min_support, batch_limit, 1 if profile else 0, cb, None,
                  mode, mni_cap, ctypes.addressof(cancel) if cancel is not None else None, sm_percent, host_threads)
    h = ctypes.c_void_p()
    _check(lib.gva_mine(db._h, ctypes.byref(o), ctypes.byref(h)))
    return _mine_result(h)


def _reduce_callback(reduce):
    if reduce is None:
        return REDUCE_FN(0)

    def _cb(sp, ep, n, user):
        try:
            sup = np.ctypeslib.as_array(sp, shape=(n,))
            emb = np.ctypeslib.as_array(ep, shape=(n,))
            reduce(sup, emb)
            return 0
        except Exception:
            return 1
    return REDUCE_FN(_cb)


def mine_host(labels, num_edge_labels: int, max_edges: int, min_support: int, evaluate, reduce=None,
              edge_labels=None, host_threads: int = 0):
    """gva_mine's level loop on the host with a Python evaluator
    (gva_mine_host): evaluate(texts) -> (supports, embeddings) for a list of
    candidate query texts; reduce(supports, embeddings) as in mine().  labels
    are the ascending vertex labels, edge labels 1..num_edge_labels (those in
    edge_labels when given).  Returns (patterns, stats)."""
    lib = library()
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    has = np.zeros(num_edge_labels + 1, dtype=np.uint8)
    for el in (edge_labels if edge_labels is not None else range(1, num_edge_labels + 1)):
        has[el] = 1

    def _eval(tp, op, n, sp, ep, user):
        try:
            offs = np.ctypeslib.as_array(op, shape=(n,)).copy()
            texts = [ctypes.string_at(tp + int(o)).decode() for o in offs]
            sup, emb = evaluate(texts)
            np.ctypeslib.as_array(sp, shape=(n,))[:] = np.asarray(sup, dtype=np.uint32)
            np.ctypeslib.as_array(ep, shape=(n,))[:] = np.asarray(emb, dtype=np.uint64)
            return 0
        except Exception:
            return 1
    ecb = EVAL_FN(_eval)
    rcb = _reduce_callback(reduce)
    h = ctypes.c_void_p()
    _check(lib.gva_mine_host(len(lab), lab.ctypes.data, num_edge_labels, has.ctypes.data, max_edges, min_support,
                             host_threads, ecb, None, rcb, None, ctypes.byref(h)))
    return _mine_result(h)


def _mine_result(h):
    lib = library()
    try:
        n = lib.gva_mine_num_patterns(h)
        need = lib.gva_mine_export(h, None, 0, None, None, None, None)
        blob = np.empty(max(need, 1), dtype=np.uint8)
        off = np.empty(n, dtype=np.uint64)
        edges = np.empty(n, dtype=np.uint32)
        sups = np.empty(n, dtype=np.uint32)
        embs = np.empty(n, dtype=np.uint64)
        lib.gva_mine_export(h, blob.ctypes.data, need, off.ctypes.data, edges.ctypes.data, sups.ctypes.data,
                            embs.ctypes.data)
        pats = MinedPatterns(blob[:need], off, edges, sups, embs)
        st = _MineStats()
        _check(lib.gva_mine_get_stats(h, ctypes.byref(st)))
        stats = {f: getattr(st, f) for f, _ in _MineStats._fields_}
        ks = (_KernelStat * 8)()
        n = lib.gva_mine_kernel_stats(h, ks, 8)
        stats["kernels"] = {ks[i].name.decode(): dict(launches=int(ks[i].launches), ms=float(ks[i].ms),
                                                       bytes=float(ks[i].bytes), rows=float(ks[i].rows))
                            for i in range(n)}
    finally:
        lib.gva_mine_free(h)
    return pats, stats


def mni_support(db: Database, patterns: Sequence[str], cap: int = 0, plain: bool = False, stream: Optional[int] = None,
                profile: bool = False):
    """Minimum image-based support of each pattern (.query text) on the data
    graph, as min(MNI, cap) (cap 0 = exact) (gva_mni_support).  plain runs
    one pattern at a time.  Returns (supports uint32[n], stats)."""
    n = len(patterns)
    buf, arr = _text_array(patterns)
    sup = np.zeros(n, dtype=np.uint32)
    o = _MniOpts(stream or None, cap, 1 if plain else 0, 1 if profile else 0, 0)
    st = _MniStats()
    _check(library().gva_mni_support(db._h, arr.ctypes.data, n, ctypes.byref(o), sup.ctypes.data,
                                     ctypes.byref(st)))
    stats = {f: getattr(st, f) for f, _ in _MniStats._fields_ if f != "kernel"}
    k = st.kernel
    stats["kernel"] = dict(name=k.name.decode(), launches=int(k.launches), ms=float(k.ms), bytes=float(k.bytes),
                           rows=float(k.rows))
    return sup, stats


# ---- reference-named entry points -------------------------------------------

def loadDataBase(mygraph: str, metadata: str, device: int = 0) -> Database:
    """src/loadDataBase.cpp:309 — here the database lands in HBM directly."""
    return Database.load(mygraph, metadata, device)


def genMatchOrder(query: str) -> Plan:
    """src/genMatchOrder.cpp:672 — `query` is a .query path or its text."""
    return Plan.from_file(query, MODE_DV) if os.path.exists(str(query)) else Plan.from_text(query, MODE_DV)


def genMatchOrderSingleV(query: str) -> Plan:
    """src/genMatchOrderSingleV.cpp:678."""
    return Plan.from_file(query, MODE_SV) if os.path.exists(str(query)) else Plan.from_text(query, MODE_SV)


def gpumine(mygraph: str, metadata: str, query: str, out: str = "partialResultsGPU.txt",
            mode: int = MODE_DV) -> Result:
    """The gpumine driver (src/gpumine.cpp:866-1072) as a function: loads,
    plans, matches and writes the match-ordered rows to `out`."""
    db = loadDataBase(mygraph, metadata)
    plan = genMatchOrder(query) if mode == MODE_DV else genMatchOrderSingleV(query)
    res = match(db, plan)
    if out:
        res.write_text(out)
    res._db, res._plan = db, plan  # keep alive with the result
    return res


def gpumineSV(mygraph: str, metadata: str, query: str, out: str = "partialResultsGPU.txt") -> Result:
    """The gpumineSV driver (src/gpumine_singleV.cpp:722-928)."""
    return gpumine(mygraph, metadata, query, out, MODE_SV)
