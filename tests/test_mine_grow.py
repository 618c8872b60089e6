"""The miner's level step (grow_level in geneva_b200/csrc/gva_grow.h) on the CPU.

tests/mine_grow_check.cpp runs level-wise growth with a seeded anti-monotone
stand-in for supports and compares every level's candidate set with a brute
force generator that shares no code with the miner (canonical codes by all
vertex orders, every extension checked against every one-edge-less connected
sub-pattern).  This pins the pruning shortcuts in the miner (wedge table,
order-free invariants, first sub-pattern check before the code) to the plain
definition of a candidate: they may only drop what the definition drops.
The same driver then runs the miner's whole host level loop (mine_levels,
which the GPU miner calls with the device evaluator) with the stand-in as
evaluator and checks every level's evaluated candidates and the returned
frequent patterns (texts, supports) against the brute force.
"""
import shutil
import subprocess

import pytest

from conftest import ROOT

# L vertex labels, P edge labels, max edges, seed, support threshold, threads
CASES = [
    (3, 2, 5, 7, 0.3, 4),       # labelled, heavy pruning
    (4, 2, 4, 9, 0.2, 3),
    (4, 1, 5, 3, 0.08, 2),
    (2, 3, 4, 4, 0.05, 3),      # several edge labels between the same vertex labels
    (1, 1, 6, 2, 0.0, 4),       # unlabelled: every connected graph up to 6 edges (large symmetric cells)
    (260, 1, 4, 11, 0.999, 4),  # more than 256 labels: 2-byte codes
    (3, 2, 4, 5, 0.2, 1),       # one host thread
]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("grow") / "mine_grow_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(ROOT / "tests" / "mine_grow_check.cpp"),
                    str(ROOT / "geneva_b200" / "csrc" / "gva_pool.cpp")],
                   check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("case", CASES, ids=lambda c: "L{}_P{}_e{}_s{}".format(*c[:4]))
def test_grow_level_equals_brute_force(checker, case):
    r = subprocess.run([str(checker), *map(str, case)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().splitlines()[-1].startswith("ok"), r.stdout
