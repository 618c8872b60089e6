"""The miner's planner entry (plan_from_query: a pattern's labels and edge
triples) against the text entry the reference reads (plan_from_text), on the
CPU: tests/plan_query_check.cpp plans seeded random connected queries (cycles,
repeated vertex and edge labels, repeated edge lines) both ways in both modes
and requires identical plans, columns and lowered steps.  plan_from_text is
itself pinned to the reference planner by test_planner.py.
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
    exe = tmp_path_factory.mktemp("planq") / "plan_query_check"
    csrc = ROOT / "geneva_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(ROOT / "tests" / "plan_query_check.cpp"),
                    str(csrc / "gva_plan.cpp"), str(csrc / "gva_graph.cpp")], check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_plan_from_query_equals_plan_from_text(checker, seed):
    r = subprocess.run([str(checker), "20000", str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout
