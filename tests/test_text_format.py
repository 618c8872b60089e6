"""Result rows as text (format_rows, the writer of partialResultsGPU.txt) on
the CPU: tests/text_format_check.cpp compares it with formatting every value
by std::to_string, for every row width 1..32, extreme values, several thread
counts and row counts around the per-thread split.
"""
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_rows_as_text(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "text_format_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(ROOT / "tests" / "text_format_check.cpp"),
                    str(ROOT / "geneva_b200" / "csrc" / "gva_text.cpp")], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout
