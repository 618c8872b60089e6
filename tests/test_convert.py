""".g converter (gva_convert_g) against the reference converter's output.

The committed graph fixtures were written by the reference tools/genDatabase.cpp
(tests/golden/make_golden.py) from the seeded .g files querygen.make_graph
builds; the converter must reproduce them byte for byte.
"""
import filecmp
import os
import shutil
import subprocess
from pathlib import Path

import pytest

import geneva_b200 as gv
from conftest import GOLDEN, ROOT
from querygen import make_graph, write_g

SPECS = [
    dict(name="syn_a", n=400, avg_deg=5.0, vlabels=3, elabels=2, seed=1, hub=0),
    dict(name="syn_b", n=1500, avg_deg=3.0, vlabels=4, elabels=3, seed=2, hub=0),
    dict(name="syn_hub", n=6000, avg_deg=2.5, vlabels=3, elabels=2, seed=3, hub=5200),
    dict(name="syn_one", n=800, avg_deg=4.0, vlabels=1, elabels=1, seed=4, hub=0),
]


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: s["name"])
def test_converter_matches_reference_fixtures(native, spec, tmp_path):
    vl, edges = make_graph(spec)
    g = tmp_path / f"{spec['name']}.g"
    g.write_text(write_g(vl, edges))
    gv.convert_g(g, tmp_path / spec["name"])
    for ext in ("mygraph", "metadata"):
        assert filecmp.cmp(tmp_path / f"{spec['name']}.{ext}", GOLDEN / "graphs" / f"{spec['name']}.{ext}",
                           shallow=False), ext
    # the converted files load and probe cleanly
    info = gv.probe_graph(tmp_path / f"{spec['name']}.mygraph", tmp_path / f"{spec['name']}.metadata")
    assert info["warnings"] == "" and info["num_adjacency"] == 2 * len(edges)


def test_converter_reorder_matches_reference_binary(native, tmp_path):
    ref = ROOT / "oracle" / "_ref" / "genDatabase"
    if not ref.exists():
        pytest.skip("reference converter not built here")
    spec = SPECS[2]  # the hub graph: lists long enough for index vertices
    vl, edges = make_graph(spec)
    (tmp_path / "datasets").mkdir()
    (tmp_path / "run").mkdir()
    (tmp_path / "datasets" / "h.g").write_text(write_g(vl, edges))
    subprocess.run([str(ref), "h"], cwd=tmp_path / "run", check=True, capture_output=True)
    gv.convert_g(tmp_path / "datasets" / "h.g", tmp_path / "mine")
    assert filecmp.cmp(tmp_path / "mine.reorder", tmp_path / "run" / "h.reorder", shallow=False)
    assert filecmp.cmp(tmp_path / "mine.mygraph", tmp_path / "datasets" / "h.mygraph", shallow=False)


def test_converter_cli_and_errors(native, tmp_path):
    exe = gv.library_path().parent / "gvaconvert"
    (tmp_path / "x.g").write_text("v 0 1\nv 1 2\nv 2 1\ne 0 1 1\ne 1 2 2\n")
    r = subprocess.run([str(exe), str(tmp_path / "x.g"), str(tmp_path / "x")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert (tmp_path / "x.metadata").read_text().splitlines()[0].split()[2] == "0"
    (tmp_path / "empty.g").write_text("v 0 1\n")
    with pytest.raises(gv.GenevaError):
        gv.convert_g(tmp_path / "empty.g", tmp_path / "empty")
    with pytest.raises(gv.GenevaError):
        gv.convert_g(tmp_path / "missing.g", tmp_path / "missing")


def test_converter_repeated_edges_match_reference_binary(native, tmp_path):
    """Repeated edge lines, in either orientation and around a hub, are
    dropped as the reference drops them (same bytes out)."""
    ref = ROOT / "oracle" / "_ref" / "genDatabase"
    if not ref.exists():
        pytest.skip("reference converter not built here")
    spec = SPECS[2]
    vl, edges = make_graph(spec)
    dup = list(edges) + [(b, a, l) for (a, b, l) in edges[::7]] + list(edges[::11])
    (tmp_path / "datasets").mkdir()
    (tmp_path / "run").mkdir()
    (tmp_path / "datasets" / "d.g").write_text(write_g(vl, dup))
    subprocess.run([str(ref), "d"], cwd=tmp_path / "run", check=True, capture_output=True)
    gv.convert_g(tmp_path / "datasets" / "d.g", tmp_path / "mine")
    assert filecmp.cmp(tmp_path / "mine.reorder", tmp_path / "run" / "d.reorder", shallow=False)
    assert filecmp.cmp(tmp_path / "mine.mygraph", tmp_path / "datasets" / "d.mygraph", shallow=False)
    assert filecmp.cmp(tmp_path / "mine.metadata", tmp_path / "datasets" / "d.metadata", shallow=False)


@pytest.mark.parametrize("seed", range(6))
def test_converter_random_graphs_match_reference_binary(native, tmp_path, seed):
    """Random graphs with up to 6 edge labels (the renumbering splits the
    largest partition by every other one) and hubs: all three files equal the
    reference converter's."""
    import random
    ref = ROOT / "oracle" / "_ref" / "genDatabase"
    if not ref.exists():
        pytest.skip("reference converter not built here")
    rng = random.Random(seed)
    spec = dict(name=f"r{seed}", n=rng.choice([300, 2000, 5000]), avg_deg=rng.choice([1.5, 3.0, 6.0]),
                vlabels=rng.randint(1, 5), elabels=rng.randint(2, 6), seed=500 + seed,
                hub=rng.choice([0, 1]) * rng.randint(150, 280))
    vl, edges = make_graph(spec)
    (tmp_path / "datasets").mkdir()
    (tmp_path / "run").mkdir()
    (tmp_path / "datasets" / "r.g").write_text(write_g(vl, edges))
    subprocess.run([str(ref), "r"], cwd=tmp_path / "run", check=True, capture_output=True)
    gv.convert_g(tmp_path / "datasets" / "r.g", tmp_path / "mine")
    assert filecmp.cmp(tmp_path / "mine.reorder", tmp_path / "run" / "r.reorder", shallow=False)
    assert filecmp.cmp(tmp_path / "mine.mygraph", tmp_path / "datasets" / "r.mygraph", shallow=False)
    assert filecmp.cmp(tmp_path / "mine.metadata", tmp_path / "datasets" / "r.metadata", shallow=False)
