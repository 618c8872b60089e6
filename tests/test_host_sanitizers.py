"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU only):
the CPU test drivers for the miner's host loop, the heap-free planner, the
planner's two entries, the database build and the host worker pool are rebuilt with
-fsanitize=address,undefined and run on small cases; any invalid access, leak
or undefined operation fails the run.
"""
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

import pytest

from conftest import ROOT

CSRC = ROOT / "geneva_b200" / "csrc"
TESTS = ROOT / "tests"
DRIVERS = {
    "mine_grow_check": [TESTS / "mine_grow_check.cpp", CSRC / "gva_pool.cpp"],
    "dplan_check": [TESTS / "dplan_check.cpp", CSRC / "gva_plan.cpp", CSRC / "gva_graph.cpp"],
    "plan_query_check": [TESTS / "plan_query_check.cpp", CSRC / "gva_plan.cpp", CSRC / "gva_graph.cpp"],
    "graph_build_check": [TESTS / "graph_build_check.cpp", CSRC / "gva_graph.cpp", CSRC / "gva_plan.cpp"],
    "mygraph_roundtrip_check": [TESTS / "mygraph_roundtrip_check.cpp", CSRC / "gva_convert.cpp", CSRC / "gva_graph.cpp",
                                CSRC / "gva_plan.cpp"],
    "text_format_check": [TESTS / "text_format_check.cpp", CSRC / "gva_text.cpp"],
    "pool_check": [TESTS / "pool_check.cpp", CSRC / "gva_pool.cpp"],
}
RUNS = [
    ("mine_grow_check", ["3", "2", "4", "7", "0.3", "4"]),
    ("mine_grow_check", ["1", "1", "5", "2", "0.0", "1"]),
    ("dplan_check", ["5000", "1", "8"]),
    ("dplan_check", ["1000", "3", "32"]),
    ("plan_query_check", ["1000", "1"]),
    ("graph_build_check", ["20", "1", "3000"]),
    ("graph_build_check", ["1", "2", "70000"]),  # the threaded sort and fill
    ("mygraph_roundtrip_check", ["10", "3", None]),  # None: a scratch directory
    ("text_format_check", ["2", "8000"]),
    ("pool_check", ["4", "200", "37"]),  # concurrent and nested jobs on the host worker pool
]


@pytest.fixture(scope="module")
def sanitized(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("san")
    probe = subprocess.run([cxx, "-fsanitize=address,undefined", "-x", "c++", "-", "-o", str(out / "probe")],
                           input="int main(){return 0;}", capture_output=True, text=True)
    if probe.returncode != 0:
        pytest.skip("sanitizer runtimes not available")

    def build(item):
        name, srcs = item
        exe = out / name
        subprocess.run([cxx, "-fsanitize=address,undefined", "-fno-omit-frame-pointer", "-g", "-O1", "-std=c++17",
                        "-pthread", "-o", str(exe), *map(str, srcs)], check=True, capture_output=True, text=True)
        return name, exe

    with ThreadPoolExecutor(max_workers=len(DRIVERS)) as ex:
        return dict(ex.map(build, DRIVERS.items()))


@pytest.mark.parametrize("name,args", RUNS, ids=lambda x: x if isinstance(x, str) else "-".join(a or "dir" for a in x))
def test_host_code_is_sanitizer_clean(sanitized, name, args, tmp_path):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    args = [str(tmp_path) if a is None else a for a in args]
    r = subprocess.run([str(sanitized[name]), *args], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    assert r.stdout.strip().splitlines()[-1].startswith("ok"), r.stdout[-2000:]
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-3000:]
