"""The heap-free planner (dplan, geneva_b200/csrc/gva_dplan.h; host and
device code, the miner's planner on the host) against the host planner on the
CPU: tests/dplan_check.cpp plans seeded random connected queries (cycles,
repeated labels and edge lines) both ways; every query dplan accepts must get
the host planner's plan exactly, the rest are left to the host planner.
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
    exe = tmp_path_factory.mktemp("dplan") / "dplan_check"
    csrc = ROOT / "geneva_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(ROOT / "tests" / "dplan_check.cpp"),
                    str(csrc / "gva_plan.cpp"), str(csrc / "gva_graph.cpp")], check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("seed,max_vertices,queries", [(1, 8, 100000), (2, 13, 60000), (3, 32, 20000)])
def test_dplan_equals_host_planner(checker, seed, max_vertices, queries):
    r = subprocess.run([str(checker), str(queries), str(seed), str(max_vertices)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout.strip()
    assert out.startswith("ok"), out
    if max_vertices <= 8:  # mined patterns' sizes: every query planned without the host
        assert out.endswith(", 0 left to the host"), out
