"""The batched engine's step trie (BatchSession::submit) on the host, without
a device: tests/batch_trie_check.cpp builds tries from seeded random plans in
the miner's order (with and without the presorted shortcut the miner uses)
and shuffled, and checks that every plan's path reproduces its own steps, that
each plan ends on its terminal once, and that all three tries have the same
number of nodes (shared prefixes matched once whatever the order).
"""
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def checker(native, tmp_path_factory):
    from geneva_b200 import build
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    lib = ROOT / "geneva_b200" / "lib"
    exe = tmp_path_factory.mktemp("trie") / "batch_trie_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", f"-I{build.cuda_home() / 'include'}", "-o", str(exe),
                    str(ROOT / "tests" / "batch_trie_check.cpp"), f"-L{lib}", "-lgeneva", f"-Wl,-rpath,{lib}"],
                   check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_trie_paths_and_sharing(checker, seed):
    r = subprocess.run([str(checker), "20000", str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout
