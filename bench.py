#!/usr/bin/env python
"""Benchmark of the matching path on the 20,000-graph database.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl geneva|reference]

Workload: the 20,000-graph database (|V|~U[20,60], average degree 4,
16 vertex labels Zipf(1.2), 3 edge labels; seeded, synthetic) resident in HBM,
and a batch of seeded query patterns of 3-7 vertices sampled from it.  One
step matches every pattern of the batch and enumerates every embedding
(gpumine semantics: rows materialised in HBM).  Metric: embeddings/s, the
final rows of all patterns over the step time.

N > 1 (torchrun, one process per GPU): every rank holds the database and
matches its own batch (weak scaling, no collective on the data path); the
step time is the max over ranks.

--impl reference times the reference CPU matcher (oracle/_ref/cpumine,
built from the reference sources) on the same database and patterns, one
process per pattern over all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOAD = ("config-2 database: 20000 graphs, |V|~U[20,60], avg degree 4, 16 vertex labels Zipf(1.2), "
            "3 edge labels; batch of seeded 3-7 vertex patterns sampled from it; every embedding enumerated "
            "and counted per pattern, with its supporting graphs")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="geneva", choices=["geneva", "reference"])
    ap.add_argument("--queries", type=int, default=256, help="patterns per rank per step")
    ap.add_argument("--seed", type=int, default=2)
    return ap.parse_args()


# ----------------------------------------------------------------- clocks ----
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(kernel)
    except Exception:
        return None


# ------------------------------------------------------------ CPU baseline ----
def cpu_baseline_port(db, queries, budget_s=15.0):
    """The oracle (single-threaded restatement of cpumine) on a bounded sample."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import Oracle
    o = Oracle.get()
    g = o.from_edges(db.vlabels, db.src, db.dst, db.elabels)
    t0 = time.perf_counter()
    rows = 0
    done = 0
    for q in queries:
        rows += o.count(g, q)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.free(g)
    return {"value": rows / dt, "unit": "embeddings/s", "cores": 1, "kind": "port",
            "sample": f"first {done} of the {len(queries)} patterns of one step, oracle restatement of cpumine, "
                      f"{rows} embeddings in {dt:.2f} s"}


def reference_arm(args, db, queries):
    """oracle/_ref/cpumine (the reference CPU matcher built from source) on the
    same database (converted by oracle/_ref/genDatabase) and patterns."""
    ref = ROOT / "oracle" / "_ref"
    if not (ref / "cpumine").exists() or not (ref / "genDatabase").exists():
        return {"impl": "reference", "unavailable": "oracle/_ref binaries not built (reference sources absent at build)"}
    work = Path(tempfile.mkdtemp(prefix="geneva_ref_"))
    (work / "datasets").mkdir()
    (work / "run").mkdir()
    (work / "datasets" / "config2.g").write_text(db.to_g_text())
    subprocess.run([str(ref / "genDatabase"), "config2"], cwd=work / "run", check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ds = work / "datasets"
    reorder = work / "run" / "config2.reorder"
    cores = os.cpu_count() or 1

    def one(i_q):
        i, q = i_q
        d = work / f"q{i}"
        d.mkdir(exist_ok=True)
        (d / "q.query").write_text(q)
        subprocess.run([str(ref / "cpumine"), str(reorder), "q.query", str(ds / "config2.mygraph"),
                        str(ds / "config2.metadata")], cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       check=True)
        with open(d / "partialResultsCPU.txt") as f:
            return sum(1 for _ in f)

    # bound each step to about a minute of host time: calibrate on the warm-up
    sample = queries[: min(len(queries), cores * 4)]
    def step():
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            rows = sum(ex.map(one, list(enumerate(sample))))
        return rows, time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    tot_rows, tot_t = 0, 0.0
    for _ in range(args.steps):
        r, t = step()
        tot_rows += r
        tot_t += t
    value = tot_rows / tot_t
    return {
        "metric": "embeddings/s", "value": value, "unit": "embeddings/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "patterns_per_step": len(sample), "seed": args.seed},
        "cpu_baseline": {"value": value, "unit": "embeddings/s", "cores": cores, "kind": "reference",
                         "sample": f"{len(sample)} of the {len(queries)} patterns per step, one cpumine "
                                   f"process per pattern"},
        "e2e": {"value": value, "unit": "embeddings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ GPU arm ----
def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from geneva_b200 import workloads

    if args.impl == "reference":
        if rank != 0:
            return 0
        db = workloads.config2(seed=args.seed)
        queries = workloads.sample_patterns(db, args.queries, 3, 7, seed=1000)
        print(json.dumps(reference_arm(args, db, queries)), flush=True)
        return 0

    import torch
    import geneva_b200 as gv

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    db = workloads.config2(seed=args.seed)
    queries = workloads.sample_patterns(db, args.queries, 3, 7, seed=1000 + rank)
    gdb = gv.Database.from_edges(db.vlabels, db.src, db.dst, db.elabels, device=local)
    gdb.set_graphs(db.first)
    plans = [gv.Plan.from_text(q) for q in queries]
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def batched_step(profile=False):
        counts, support, stats = gv.batch_count(gdb, plans, stream=sp, support=True, profile=profile)
        return int(counts.sum()), stats

    def plain_step():
        rows = 0
        for p in plans:
            r = gv.match(gdb, p, stream=sp, count_only=True)
            rows += r.num_rows
            r.close()
        return rows

    def timed(fn, steps):
        ms, rows = [], 0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # evict L2 between steps (outside the timed events)
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            rows += out if isinstance(out, int) else out[0]
        return ms, rows

    for _ in range(max(args.warmup, 3)):
        batched_step()
        plain_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = gv.kernel_launches()
    step_ms, rows_total = timed(lambda: batched_step()[0], args.steps)
    launches = gv.kernel_launches() - launches0
    clk = clocks.stop()
    plain_ms, plain_rows = timed(plain_step, args.steps)

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t)
        return float(t.item())

    t_sum = max_over_ranks(sum(step_ms))
    rows_all = sum_over_ranks(rows_total)
    value = rows_all / (t_sum / 1000.0)
    plain_value = sum_over_ranks(plain_rows) / (max_over_ranks(sum(plain_ms)) / 1000.0)

    # ---- roofline: one profiled batched step (CUDA events around every kernel)
    with torch.cuda.stream(stream):
        flush.zero_()
    stream.synchronize()
    _, pstats = batched_step(profile=True)
    kstats = {k: v for k, v in pstats["kernels"].items() if v["launches"]}

    # ---- end to end through the public API: pattern text in (planned on the
    # host), per-pattern embedding counts and supports out to host memory
    e2e_steps = max(1, args.steps)
    h2d = sum(len(q.encode()) for q in queries)
    d2h = len(queries) * (8 + 4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_rows = 0
    for _ in range(e2e_steps):
        ps = [gv.Plan.from_text(q) for q in queries]
        counts, support, _ = gv.batch_count(gdb, ps, stream=sp, support=True)
        e2e_rows += int(counts.sum())
        for p in ps:
            p.close()
    torch.cuda.synchronize()
    e2e_t = max_over_ranks(time.perf_counter() - t0)
    e2e_value = sum_over_ranks(e2e_rows) / e2e_t

    peak, peak_kind = measured_peak_gbs()
    name, s = max(kstats.items(), key=lambda kv: kv[1]["ms"]) if kstats else ("none", {"launches": 0, "ms": 0, "bytes": 0})
    per_launch_ms = s["ms"] / max(s["launches"], 1)
    achieved = (s["bytes"] / max(s["launches"], 1)) / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms else 0.0
    traffic = ncu_traffic(name)

    out = None
    if rank == 0:
        out = {
            "metric": "embeddings/s", "value": value, "unit": "embeddings/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": t_sum / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded generator of the configuration's shapes)",
            "config": {"workload": WORKLOAD, "patterns_per_rank_per_step": len(queries), "seed": args.seed,
                       "path": "batched: all patterns of a step advance together (gva_batch_count)",
                       "outputs": "embeddings and supporting-graph count per pattern",
                       "l2": "flushed between steps (512 MiB write)",
                       "parallelism": f"replicated database, patterns sharded over {world} rank(s)"},
            "plain": {"value": plain_value, "unit": "embeddings/s", "ms_per_step": sum(plain_ms) / args.steps,
                      "path": "one gva_match per pattern (count only), same patterns",
                      "batched_over_plain": value / plain_value if plain_value else None},
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "launches": s["launches"], "kernel_ms": s["ms"]},
            "kernels": kstats,
            "batch": {k: pstats[k] for k in ("rounds", "splits", "launches", "trie_nodes")},
            "e2e": {"value": e2e_value, "unit": "embeddings/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "pattern text planned on the host each step; counts and supports copied to host"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if world == 1:
            out["cpu_baseline"] = cpu_baseline_port(db, queries)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    gdb.close()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
