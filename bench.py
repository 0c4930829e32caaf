"""Benchmark: batched star-join queries on a 600,000,000-row fact table.

Workload (the headline metric's configuration): 8 int32 fact columns
(orderdate, custkey, suppkey, partkey, quantity, discount, revenue, supplycost;
19.2 GB resident in HBM) with the SSB-shaped date / customer / supplier / part
dimensions, and batches of queries drawn by seed from four templates (T0 range
filters + scalar SUM; T1 date join + GROUP BY year; T2 three joins + GROUP BY
(nation, year); T3 four joins + GROUP BY (brand, year)).  Synthetic data,
generated on the device from a counter-based hash (practice_b200/datagen.py).

One step = one batch of queries over the whole fact table.  ``--mode plain``
runs the batch one query at a time with the plain fused kernels (the drop-in
path); ``--mode shared`` runs it as one shared-scan launch.  The JSON line
reports queries/s of the whole job, per-query latency percentiles, the
roofline of the dominant kernel against measured HBM bandwidth, the CPU
baseline (the reference's own primitives compiled for the host, timed on a
bounded row sample), clocks sampled during the timed region and the end-to-end
figure through the public API (result read back to the host each query).

Multi-GPU (torchrun): every rank holds its own 600M-row table and runs its own
batch (independent replicas, no collective on the data path); value sums the
queries of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "queries/s + p50/p99 ms, shared-scan vs plain, 600M-row fact; % of HBM peak"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="plain", choices=["plain", "shared"])
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-rows", type=int, default=4_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(ngpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value: float, device) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    import torch
    if pg is not None:
        pg.barrier(device_ids=[device.index])
    torch.cuda.synchronize(device)


# ------------------------------------------------------------- CPU baseline


def cpu_baseline(plans_full, args, batch_rows: int):
    """The reference's CPU path on a bounded row sample of the same batch.

    Uses oracle/_ref (the reference's own crystal primitives compiled for the
    host with OpenMP) when it was built, else the oracle restatement."""
    import numpy as np

    from oracle import refbase
    from practice_b200 import datagen, queries

    n = min(args.cpu_sample_rows, batch_rows)
    ht = datagen.host_tables(args.seed, n, queries.C4_COLS)
    plans = queries.batch(args.batch, args.seed, n)
    t, kind, cores = refbase.time_batch(plans, ht, n)
    scale = batch_rows / n
    qps = len(plans) / (t * scale)
    return {"value": qps, "unit": "queries/s", "cores": cores, "kind": kind,
            "sample": f"{len(plans)}-query batch on the first {n:,} of {batch_rows:,} fact rows, "
                      f"time scaled by {scale:.0f}x to the full table ({t:.3f} s measured)"}


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    times = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(None, args, args.rows)
        if i >= args.warmup:
            times.append(cb["value"])
    v = statistics.median(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": args.batch / v * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/u64",
        "data": "synthetic", "config": config_block(args),
        "cpu_baseline": {**cb, "value": v},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args):
    return {"workload": "config4: batched star-join queries, 600M-row fact, 4 templates",
            "fact_rows": args.rows, "fact_columns": 8, "batch_queries": args.batch, "mode": args.mode,
            "seed": args.seed, "parallelism": f"replicas{args.gpus}",
            "l2": "inputs (19.2 GB) larger than L2 (126 MB); no flush needed"}


# ------------------------------------------------------------------ GPU arm


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import numpy as np
    import torch

    from practice_b200 import _lib, queries
    from practice_b200.engine import Database

    world, rank, local, pg = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    db = Database(local)
    db.generate_ssb(args.rows, args.seed + rank, queries.C4_COLS)
    plans = queries.batch(args.batch, args.seed, args.rows)
    mods = [db.compile(p) for p in plans]
    results = [db.alloc_result(m) for m in mods]
    stream = torch.cuda.Stream(device)
    ctxs = []
    for m, (res, val) in zip(mods, results):
        c = _lib.ExecCtx()
        for name, t in db.cols.items():
            c.set_buffer("d_" + name, t.data_ptr(), t.numel())
        for t, n in db.rows.items():
            c.set_rows(t, n)
        c.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
        ctxs.append(c)

    def run_step(record=None):
        # one batch, one query after another on one stream
        for i, (m, c) in enumerate(zip(mods, ctxs)):
            c.execute(m, stream.cuda_stream)
            if record is not None:
                record[i].record(stream)

    # warmup (also loads modules on the device)
    for _ in range(args.warmup):
        run_step()
    stream.synchronize()
    for c in ctxs:
        c.sync()

    # timed region
    sampler = ClockSampler(local)
    barrier(pg, device)
    sampler.start()
    time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    done = [[torch.cuda.Event(enable_timing=True) for _ in mods] for _ in range(args.steps)]
    step_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    scan_ms = [0.0] * len(mods)
    start.record(stream)
    for s in range(args.steps):
        step_start[s].record(stream)
        run_step(done[s])
    end.record(stream)
    end.synchronize()
    clocks = sampler.stop()
    total_ms = start.elapsed_time(end)
    for i, c in enumerate(ctxs):
        c.sync()
        scan_ms[i] = c.timing().scan_ms  # last step's scan kernel duration, per query
    lat = []
    for s in range(args.steps):
        for i in range(len(mods)):
            lat.append(step_start[s].elapsed_time(done[s][i]))
    total_ms = max_over_ranks(pg, total_ms, device)
    barrier(pg, device)

    nq = len(mods) * args.steps * world
    value = nq / (total_ms / 1000.0)
    # roofline of the dominant kernel (the fused scan): algorithmic fact bytes / scan time
    bytes_per_query = [len(p.columns_read()) * 4 * args.rows for p in plans]
    achieved = sum(bytes_per_query) / (sum(scan_ms) / 1000.0) / 1e9
    peak, peak_kind = peaks()
    launches = sum(c.timing().gpu_launches for c in ctxs)

    # end to end through the public API: execute + result read back per query
    e2e = None
    if rank == 0 or True:
        pinned = [torch.empty(r.numel(), dtype=torch.int64, pin_memory=True) for r, _ in results]
        pinned_v = [torch.empty(v.numel(), dtype=torch.int64, pin_memory=True) for _, v in results]
        d2h = sum(p.numel() * 8 + q.numel() * 8 for p, q in zip(pinned, pinned_v))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps // 2)):
            for i, (m, c) in enumerate(zip(mods, ctxs)):
                mm = db.compile(plans[i])  # cache lookup, as QueryEngine does per query
                c.execute(mm, stream.cuda_stream)
                pinned[i].copy_(results[i][0], non_blocking=True)
                pinned_v[i].copy_(results[i][1], non_blocking=True)
            stream.synchronize()
        e2e_s = time.perf_counter() - t0
        e2e = {"value": len(mods) * max(1, args.steps // 2) * world / e2e_s, "unit": "queries/s",
               "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
               "note": "fact table resident in HBM; results read back to pinned host memory every query"}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(plans, args, args.rows)
        except Exception as e:  # reported, not fatal
            cb = {"value": None, "unit": "queries/s", "error": str(e)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/u64", "data": "synthetic",
            "config": config_block(args),
            "latency_ms": {"p50": statistics.median(lat), "p99": float(np.percentile(lat, 99)),
                           "definition": "query completion since its batch started"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                         "kernel": "Scan_LINEORDER (plain fused scan/probe/aggregate)",
                         "algorithmic_bytes": "distinct fact columns read x 4 B x rows, per query"},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
            "cpu_baseline": cb,
            "plain_scan_ms": {"mean": statistics.mean(scan_ms), "min": min(scan_ms), "max": max(scan_ms)},
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
