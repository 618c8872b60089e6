import gzip
import json
import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(GOLDEN))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def native():
    """The product library, built in-tree if needed."""
    from geneva_b200 import build, library
    if not (ROOT / "geneva_b200" / "lib" / "libgeneva.so").exists():
        build.build()
    return library()


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import Oracle
    return Oracle.get()


@pytest.fixture(scope="session")
def golden_plans():
    with gzip.open(GOLDEN / "plans.jsonl.gz", "rt") as f:
        return [json.loads(l) for l in f]


@pytest.fixture(scope="session")
def golden_matches():
    return json.loads((GOLDEN / "matches.json").read_text())


@pytest.fixture(scope="session")
def enron_dir(tmp_path_factory):
    """Enron .mygraph/.metadata unpacked from the committed fixture."""
    d = tmp_path_factory.mktemp("enron")
    for ext in ("mygraph", "metadata"):
        with gzip.open(GOLDEN / "enron" / f"Enron.{ext}.gz", "rb") as fi:
            (d / f"Enron.{ext}").write_bytes(fi.read())
    shutil.copy(GOLDEN / "enron" / "Enron_4_6_0.query", d / "Enron_4_6_0.query")
    return d
