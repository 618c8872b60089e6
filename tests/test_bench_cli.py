"""bench.py's reference arm (CPU only): one JSON line with the keys the
benchmark contract needs, on the small graph-database configuration."""
import json
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "mine", "--db",
                        "config1", "--steps", "1", "--warmup", "1", "--sample", "8"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # reference sources absent when the binaries were built
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["metric"] == "embeddings/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "config-1" in d["config"]["workload"]


def test_default_reference_arm_prints_the_gpu_arms_config():
    """The default workload: the reference arm times the same pattern list and
    prints the same config object as the GPU arm (bench.batch_config)."""
    sys.path.insert(0, str(ROOT))
    import bench
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--patterns", "64"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    if "unavailable" in d:
        return
    want = bench.batch_config(type("A", (), {"patterns": 64, "seed": 2})(), 1)
    assert d["config"] == want
    assert d["metric"] == "embeddings/s" and d["value"] > 0 and d["unit"] == "embeddings/s"
    assert d["cpu_baseline"]["process_s_min"] > 0
