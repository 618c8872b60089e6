"""Regenerates the golden fixtures from the reference itself.

Run in a container that has the reference sources (the binaries are built
from them by `make -C oracle ref`):

    python tests/golden/make_golden.py

Writes, under tests/golden/:
  plans.jsonl.gz        random queries + the reference planner's plan text
                        (oracle/_ref/plandump around src/genMatchOrderCPU.cpp)
  graphs/<name>.{mygraph,metadata}   seeded synthetic .g files run through the
                        reference converter (tools/genDatabase.cpp)
  matches.json          per (graph, query): distinct-row count and sha256 of the
                        sorted distinct rows from the reference `cpumine`
  enron/Enron.{mygraph,metadata}.gz + enron.json   the shipped Enron dataset
                        and its known answer for Enron_4_6_0.query

Row hashes: rows are the space-separated lines of partialResultsCPU.txt,
parsed to uint32, de-duplicated (cpumine repeats rows through genDatabase's
index vertices) and sorted lexicographically; sha256 of the little-endian bytes.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import random
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = ROOT / "oracle" / "_ref"
REFERENCE = Path(os.environ.get("GENEVA_REFERENCE", "/root/reference"))

sys.path.insert(0, str(HERE))
from querygen import random_query, structured_queries, sample_query, make_graph, write_g  # noqa: E402


def rows_digest(rows: np.ndarray) -> tuple[int, str]:
    if rows.size == 0:
        return 0, hashlib.sha256(b"").hexdigest()
    u = np.unique(rows.astype(np.uint32), axis=0)
    return int(u.shape[0]), hashlib.sha256(np.ascontiguousarray(u).astype("<u4").tobytes()).hexdigest()


def read_rows(path: Path) -> np.ndarray:
    lines = [l.split() for l in path.read_text().splitlines() if l.strip()]
    if not lines:
        return np.zeros((0, 0), dtype=np.uint32)
    return np.array(lines, dtype=np.uint64).astype(np.uint32)


def ref_plan(query_text: str, work: Path) -> str:
    q = work / "q.query"
    q.write_text(query_text)
    out = work / "plan.txt"
    subprocess.run([str(REF / "plandump"), str(q), str(out)], check=True, timeout=60,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return out.read_text()


def ref_convert(name: str, g_text: str, work: Path) -> Path:
    """tools/genDatabase.cpp reads ../datasets/<name>.g and writes .mygraph/.metadata there."""
    ds = work / "datasets"
    run = work / "run"
    ds.mkdir(exist_ok=True)
    run.mkdir(exist_ok=True)
    (ds / f"{name}.g").write_text(g_text)
    subprocess.run([str(REF / "genDatabase"), name], cwd=run, check=True, timeout=600,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    shutil.move(str(run / f"{name}.reorder"), str(ds / f"{name}.reorder"))
    return ds


def ref_cpumine(ds: Path, name: str, query_text: str, work: Path, timeout=120):
    run = work / "cm"
    run.mkdir(exist_ok=True)
    (run / "q.query").write_text(query_text)
    r = subprocess.run([str(REF / "cpumine"), str(ds / f"{name}.reorder"), "q.query",
                        str(ds / f"{name}.mygraph"), str(ds / f"{name}.metadata")],
                       cwd=run, timeout=timeout, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    return read_rows(run / "partialResultsCPU.txt")


def main():
    if not (REF / "cpumine").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    rng = random.Random(20261203)
    work = Path(tempfile.mkdtemp(prefix="geneva_golden_"))
    try:
        # ---- planner fixtures -------------------------------------------------
        plans = []
        queries = structured_queries()
        while len(queries) < 1500:
            queries.append(random_query(rng))
        for q in queries:
            plans.append({"q": q, "plan": ref_plan(q, work)})
        with gzip.open(HERE / "plans.jsonl.gz", "wt") as f:
            for p in plans:
                f.write(json.dumps(p) + "\n")
        print("plans:", len(plans))

        # ---- synthetic graphs through the reference converter + cpumine -----
        gdir = HERE / "graphs"
        gdir.mkdir(exist_ok=True)
        matches = []
        specs = [
            dict(name="syn_a", n=400, avg_deg=5.0, vlabels=3, elabels=2, seed=1, hub=0),
            dict(name="syn_b", n=1500, avg_deg=3.0, vlabels=4, elabels=3, seed=2, hub=0),
            dict(name="syn_hub", n=6000, avg_deg=2.5, vlabels=3, elabels=2, seed=3, hub=5200),
            dict(name="syn_one", n=800, avg_deg=4.0, vlabels=1, elabels=1, seed=4, hub=0),
        ]
        for spec in specs:
            name = spec["name"]
            vl, edges = make_graph(spec)
            ds = ref_convert(name, write_g(vl, edges), work)
            for ext in ("mygraph", "metadata"):
                shutil.copy(ds / f"{name}.{ext}", gdir / f"{name}.{ext}")
            # the converter renumbers: read back the data graph as the reference stores it
            qrng = random.Random(spec["seed"] * 7919)
            made = 0
            tries = 0
            while made < 24 and tries < 200:
                tries += 1
                k = qrng.randint(3, 6)
                q = sample_query(vl, edges, k, qrng)
                if q is None:
                    continue
                try:
                    rows = ref_cpumine(ds, name, q, work, timeout=60)
                except (subprocess.TimeoutExpired, RuntimeError):
                    continue
                cnt, dig = rows_digest(rows)
                if cnt > 400000:
                    continue
                matches.append({"graph": name, "q": q, "rows": cnt, "sha256": dig,
                                "width": int(rows.shape[1]) if rows.size else 0})
                made += 1
            print(name, "queries:", made)
        (HERE / "matches.json").write_text(json.dumps(matches, indent=0))

        # ---- Enron known answer ---------------------------------------------------
        edir = HERE / "enron"
        edir.mkdir(exist_ok=True)
        src = REFERENCE / "exp" / "datasets"
        for ext in ("mygraph", "metadata"):
            with open(src / f"Enron.{ext}", "rb") as fi, gzip.open(edir / f"Enron.{ext}.gz", "wb") as fo:
                fo.write(fi.read())
        qtext = (src / "Enron" / "Enron_4_6_0.query").read_text()
        ds = work / "enron"
        ds.mkdir()
        run = work / "enron_run"
        run.mkdir()
        (work / "datasets").mkdir(exist_ok=True)
        shutil.copy(src / "Enron.g", work / "datasets" / "Enron.g")
        subprocess.run([str(REF / "genDatabase"), "Enron"], cwd=run, check=True, timeout=600,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        (run / "q.query").write_text(qtext)
        r = subprocess.run([str(REF / "cpumine"), "Enron.reorder", "q.query", str(src / "Enron.mygraph"),
                            str(src / "Enron.metadata")], cwd=run, capture_output=True, text=True, timeout=600)
        raw = read_rows(run / "partialResultsCPU.txt")
        cnt, dig = rows_digest(raw)
        (edir / "Enron_4_6_0.query").write_text(qtext)
        (edir / "enron.json").write_text(json.dumps({
            "query": "Enron_4_6_0.query", "raw_rows": int(raw.shape[0]), "rows": cnt, "sha256": dig,
            "plan": ref_plan(qtext, work)}, indent=1))
        print("enron rows", raw.shape[0], cnt)
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
