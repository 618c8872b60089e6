"""The C-ABI library loads and exports every entry point include/geneva.h
declares; host-only paths work without a GPU."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

import geneva_b200 as gv
from conftest import GOLDEN, ROOT


def declared_symbols():
    text = (ROOT / "include" / "geneva.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)  # declarations only, not comments
    return sorted(set(re.findall(r"\b(gva_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    syms = declared_symbols()
    assert len(syms) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", str(gv.library_path())], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        assert getattr(native, s) is not None


def test_version_and_status_strings(native):
    assert b"sm_100a" in native.gva_version()
    assert native.gva_status_string(0) == b"ok"
    assert native.gva_status_string(4) == b"out of memory"


def test_probe_golden_graphs_host_only(native, oracle):
    for p in sorted((GOLDEN / "graphs").glob("*.mygraph")):
        info = gv.probe_graph(p, p.with_suffix(".metadata"))
        assert info["warnings"] == ""
        assert info["num_partitions"] >= 1
        assert info["num_adjacency"] > 0 and info["num_adjacency"] % 2 == 0  # undirected


def test_probe_enron_reports_short_header(native, enron_dir):
    info = gv.probe_graph(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    assert info["max_vertex_id"] == 36692
    assert info["num_partitions"] == 3
    assert "declares 4 partitions" in info["warnings"]
    # 183,831 .g edges; duplicates dropped by the converter, both directions stored
    assert 300000 < info["num_adjacency"] <= 2 * 183831


def test_probe_errors(native, tmp_path):
    with pytest.raises(gv.GenevaError) as ei:
        gv.probe_graph(tmp_path / "missing.mygraph", tmp_path / "missing.metadata")
    assert ei.value.status == 1
    (tmp_path / "x.metadata").write_text("1 1 0\n2 1 1\n")
    (tmp_path / "x.mygraph").write_bytes(b"\x01\x00\x00\x00\x09\x00\x00\x00")  # truncated partition
    with pytest.raises(gv.GenevaError) as ei:
        gv.probe_graph(tmp_path / "x.mygraph", tmp_path / "x.metadata")
    assert ei.value.status == 2


def test_load_without_gpu_fails_cleanly(native, enron_dir):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gv.GenevaError) as ei:
        gv.loadDataBase(enron_dir / "Enron.mygraph", enron_dir / "Enron.metadata")
    assert ei.value.status == 3


def test_text_marshalling_and_plan_batches_host_only(native, golden_plans):
    """Query texts go to the library as one buffer and an array of pointers
    into it (one byte per character or not); a plan batch keeps its handles
    in one array and plans like gva_plan_from_text."""
    texts = ["v 0 1\nv 1 2\ne 0 1 1\n", "# Zürich\nv 0 3\nv 1 3\ne 0 1 2\n", ""]
    buf, ptrs = gv._text_array(texts)
    assert [ctypes.string_at(int(p)).decode() for p in ptrs] == texts
    with pytest.raises(ValueError):
        gv._text_array(["v 0 1\0v 1 1"])
    qs = [g["q"] for g in golden_plans[:200]]
    batch = gv.Plan.batch_from_texts(qs)
    assert len(batch) == len(qs) and isinstance(batch, gv.PlanBatch)
    assert [p.describe() for p in batch] == [gv.Plan.from_text(q).describe() for q in qs]
    assert np.array_equal(gv._plan_handles(batch), np.array([p._h.value for p in batch], dtype=np.uint64))
    sub = batch[:5]  # a plain tuple of the batch's plans: handles gathered one by one
    assert list(gv._plan_handles(sub)) == [p._h.value for p in sub]
    batch.close()
    assert all(not p._h for p in batch)
