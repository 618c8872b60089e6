"""The host database build (graph_from_edges) and the init-phase seed groups
(seed_groups) against their definitions on the CPU: tests/graph_build_check.cpp
builds seeded random graphs (repeated and reversed edges, missing edge labels,
hub vertices; large ones so that the multi-threaded sort and fill run) and
checks every (vertex, label) list, the offset tables and both seed orders.
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
