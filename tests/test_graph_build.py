"""The host database build (graph_from_edges) and the init-phase seed groups
(seed_groups) against their definitions on the CPU: tests/graph_build_check.cpp
builds seeded random graphs (repeated and reversed edges, missing edge labels,
hub vertices; large ones so that the multi-threaded sort and fill run) and
checks every (vertex, label) list, the offset tables and both seed orders.
tests/mygraph_roundtrip_check.cpp then takes random .g graphs through the
converter and the .mygraph loader and requires the database the edge-list
build gives after the converter's renumbering.
"""
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("gbuild") / "graph_build_check"
    csrc = ROOT / "geneva_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(ROOT / "tests" / "graph_build_check.cpp"),
                    str(csrc / "gva_graph.cpp"), str(csrc / "gva_plan.cpp")], check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("graphs,seed,max_vertices", [(200, 1, 5000), (3, 2, 300000)])
def test_graph_build_definitions(checker, graphs, seed, max_vertices):
    r = subprocess.run([str(checker), str(graphs), str(seed), str(max_vertices)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout


@pytest.fixture(scope="module")
def roundtrip(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("rt") / "mygraph_roundtrip_check"
    csrc = ROOT / "geneva_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe),
                    str(ROOT / "tests" / "mygraph_roundtrip_check.cpp"), str(csrc / "gva_convert.cpp"),
                    str(csrc / "gva_graph.cpp"), str(csrc / "gva_plan.cpp")], check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2])
def test_converter_and_loader_round_trip(roundtrip, tmp_path, seed):
    r = subprocess.run([str(roundtrip), "40", str(seed), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout
