"""The C++ brute-force miner (tests/brute_mine.cpp) against the Python one
(tests/brute_miner.py) on small databases: both enumerate every connected
edge subset of every graph, so they must give the same patterns and supports.
The C++ one then stands in for the Python one on the 1,000-graph database."""
import pytest

from brute_miner import build_native, mine as brute_mine, mine_native
from geneva_b200 import workloads


@pytest.mark.parametrize("max_edges,minsup,vl,el,seed", [(3, 4, 3, 1, 1), (4, 6, 2, 2, 2), (3, 1, 4, 3, 3)])
def test_native_brute_force_equals_python(tmp_path, max_edges, minsup, vl, el, seed):
    db = workloads.graph_database(40, 5, 10, 2.8, vl, None, el, seed=seed, name=f"bm{seed}")
    exe = build_native(tmp_path)
    assert mine_native(db, max_edges, minsup, exe, tmp_path) == brute_mine(db, max_edges, minsup)
