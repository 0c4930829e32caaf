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
    ap.add_argument("--mode", default="shared", choices=["plain", "shared"])
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-rows", type=int, default=4_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-rate", type=float, default=1000.0, help="Poisson arrivals per second (serving leg)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="requests in the serving leg (0 skips it)")
    ap.add_argument("--serve-low-rate", type=float, default=100.0, help="second, light-load arrival rate")
    ap.add_argument("--serve-slots", type=int, default=1, help="launches in flight in the shared loop")
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
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK); NCCL
    on GPUs, gloo where there are none (the host-side tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
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
    if device.type == "cuda":
        if pg is not None:
            pg.barrier(device_ids=[device.index])
        torch.cuda.synchronize(device)
    elif pg is not None:
        pg.barrier()


def job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time (weak scaling: each rank holds its own replica)."""
    return units_per_rank * world / (max_ms / 1000.0)


# ------------------------------------------------------------- CPU baseline


def cpu_baseline(plans_full, args, batch_rows: int):
    """The reference's CPU path on a bounded row sample of the same batch.

    Uses oracle/_ref (the reference's own crystal primitives compiled for the
    host with OpenMP) when it was built, else the oracle restatement."""
    import numpy as np

    from oracle import refbase
    from practice_b200 import datagen, queries

    n = min(args.cpu_sample_rows, batch_rows)
    ht = datagen.host_tables(args.seed, n, queries.BATCH_COLS)
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


def serving_leg(db, plans, args, shared_tuning):
    """The request loop under a Poisson arrival stream drawn from the batch's
    queries: the shared loop (continuous batching into shared scans) and the
    plain one-query-at-a-time loop over the same stream, plus each query's
    latency alone on an idle GPU."""
    import numpy as np

    from practice_b200 import _lib

    texts = [p.text() for p in plans]

    def stream(srv, rate, n):
        rng = np.random.default_rng(args.seed)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        picks = rng.integers(0, len(plans), n)
        srv.stats(reset=True)
        ids = []
        t0 = time.perf_counter()
        for i in range(n):
            target = t0 + arrivals[i]
            while time.perf_counter() < target:
                pass
            ids.append(srv.submit(texts[picks[i]]))
        bad = 0
        for rid in ids:
            info = srv.wait(rid)
            bad += int(info.status != 0 or info.kernel_error != 0)
            srv.release(rid)
        st = srv.stats()
        return {"queries_per_s": st.queries_per_s, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms,
                "mean_batch": st.mean_batch, "launches": int(st.launches), "failed": bad,
                "peak_reserved_GB": st.peak_reserved_bytes / 1e9}

    plain = _lib.Server(db.ctx, _lib.server_config(plain_only=1, slots=1))
    try:
        for p in plans:  # the plain loop runs each query with its autotuned kernel
            plain.prepare(p.text(), db.tuning_for(p))
        lone = []
        for t in texts:  # each query alone on an idle GPU, submit to result on the host
            for _ in range(2):
                info = plain.wait(plain.submit(t))
            lone.append(info.latency_ms)
        n_low = max(50, int(args.serve_requests * args.serve_low_rate / args.serve_rate * 3))
        plain_stream = stream(plain, args.serve_rate, args.serve_requests)
        plain_low = stream(plain, args.serve_low_rate, n_low)
    finally:
        plain.close()
    cfg = _lib.server_config(max_batch=64, slots=args.serve_slots)
    if shared_tuning is not None:
        cfg.shared_tuning = shared_tuning
    srv = _lib.Server(db.ctx, cfg)
    try:
        for p in plans:  # short queues run these autotuned plain kernels
            srv.prepare(p.text(), db.tuning_for(p))
        shared_stream = stream(srv, args.serve_rate, args.serve_requests)
        shared_low = stream(srv, args.serve_low_rate, n_low)
    finally:
        srv.close()
    lone_ms = float(np.median(lone))
    return {"arrivals": f"Poisson, drawn from the batch's {len(plans)} queries; budget 40 GiB",
            "lone_query_ms": {"median": lone_ms, "max": float(np.max(lone))},
            "high_load": {"rate_per_s": args.serve_rate, "requests": args.serve_requests,
                          "shared_loop": shared_stream, "plain_loop": plain_stream,
                          "shared_vs_plain_queries_per_s": shared_stream["queries_per_s"] / max(plain_stream["queries_per_s"], 1e-9),
                          "shared_p99_vs_lone": shared_stream["p99_ms"] / lone_ms},
            "light_load": {"rate_per_s": args.serve_low_rate, "requests": n_low,
                           "shared_loop": shared_low, "plain_loop": plain_low,
                           "shared_p99_vs_lone": shared_low["p99_ms"] / lone_ms,
                           "plain_p99_vs_lone": plain_low["p99_ms"] / lone_ms}}


def config_block(args):
    return {"workload": "batched star-join queries from 4 templates over a 600M-row, 8-column int32 fact table",
            "fact_rows": args.rows, "fact_columns": 8, "batch_queries": args.batch, "mode": args.mode,
            "seed": args.seed, "parallelism": f"replicas{args.gpus}",
            "l2": "inputs (19.2 GB) larger than L2 (126 MB); no flush needed"}


# ------------------------------------------------------------------ GPU arm

# DRAM bytes (read + write) per fact row of one shared-scan launch over the
# 8-column batch table, from the ncu capture in
# profiles/SharedScan_LINEORDER_batch32_30M.md (972.2 MB for 30M rows); the
# traffic of a launch grows with its rows.
SHARED_DRAM_BYTES_PER_ROW = (968.458240e6 + 3.693568e6) / 30e6

PLAIN_CANDIDATES = [dict(block_threads=bt, items_per_thread=ipt, stages=st, ctas_per_sm=16, bitmap_budget=bm,
                         prefetch=pf, group_placement=pl)
                    for bt, ipt, st, bm, pf, pl in ((1024, 4, 0, 49152, 1, 0), (1024, 4, 0, 0, 1, 4),
                                                    (512, 2, 0, 0, 1, 4), (1024, 2, 0, 0, 0, 4),
                                                    (512, 8, 4, 0, 0, 0))]
SHARED_CANDIDATES = [dict(block_threads=bt, items_per_thread=ipt, stages=st, ctas_per_sm=2, producer_warps=pw,
                          group_merge=gm)
                     for bt, ipt, st, pw, gm in ((1024, 1, 3, 11, 0), (1024, 1, 3, 11, 3), (1024, 1, 3, 14, 0),
                                                 (1024, 1, 3, 14, 3), (512, 2, 2, 5, 0), (512, 2, 2, 7, 3))]


def time_steps(torch, stream, steps, run_step, sampler=None):
    """CUDA-event time of `steps` calls of run_step on `stream` (ms), plus the
    per-step start events and per-query completion events it records."""
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    step_start = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    marks = []
    start.record(stream)
    for s in range(steps):
        step_start[s].record(stream)
        marks.append(run_step())
    end.record(stream)
    end.synchronize()
    lat = []
    for s in range(steps):
        for ev in marks[s]:
            lat.append(step_start[s].elapsed_time(ev))
    return start.elapsed_time(end), lat


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
    db.generate_ssb(args.rows, args.seed + rank, queries.BATCH_COLS)
    plans = queries.batch(args.batch, args.seed, args.rows)
    stream = torch.cuda.Stream(device)
    peak, peak_kind = peaks()
    union_cols = sorted({c for p in plans for c in p.columns_read()})

    # ---- plain path: one fused kernel per query, one query after another
    for p in plans:
        if db.tuning_for(p) is None:
            db.autotune(p, candidates=PLAIN_CANDIDATES, reps=1, persist=False)
    mods = [db.compile(p, db.tuning_for(p)) for p in plans]
    results = [db.alloc_result(m) for m in mods]
    ctxs = []
    for m, (res, val) in zip(mods, results):
        c = _lib.ExecCtx()
        for name, t in db.cols.items():
            c.set_buffer("d_" + name, t.data_ptr(), t.numel())
        for t, n in db.rows.items():
            c.set_rows(t, n)
        c.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
        ctxs.append(c)

    def plain_step():
        evs = []
        for m, c in zip(mods, ctxs):
            c.execute(m, stream.cuda_stream)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            evs.append(ev)
        return evs

    for _ in range(args.warmup):
        plain_step()
    stream.synchronize()
    for c in ctxs:
        c.sync()
    barrier(pg, device)
    plain_ms, plain_lat = time_steps(torch, stream, args.steps, plain_step)
    for c in ctxs:
        c.sync()
    plain_scan_ms = [c.timing().scan_ms for c in ctxs]
    plain_launches = sum(c.timing().gpu_launches for c in ctxs)
    plain_ms = max_over_ranks(pg, plain_ms, device)
    plain_bytes = sum(len(p.columns_read()) * 4 * args.rows for p in plans)
    plain = {"queries_per_s": job_rate(len(plans) * args.steps, world, plain_ms),
             "ms_per_step": plain_ms / args.steps,
             "p50_ms": statistics.median(plain_lat), "p99_ms": float(np.percentile(plain_lat, 99)),
             "scan_GBps": plain_bytes / (sum(plain_scan_ms) / 1000.0) / 1e9,
             "scan_frac_of_peak": plain_bytes / (sum(plain_scan_ms) / 1000.0) / 1e9 / peak,
             "scan_ms": {"mean": statistics.mean(plain_scan_ms), "min": min(plain_scan_ms), "max": max(plain_scan_ms)}}

    # ---- shared scan: the whole batch in one persistent kernel
    shared = None
    sctx = db.ctx
    if args.mode == "shared" and all(db.shareable(p) for p in plans):
        if db.shared_tuning_for(plans) is None:
            db.autotune_shared(plans, SHARED_CANDIDATES, reps=1)
        tun = db.shared_tuning_for(plans)
        prog = db.shared_program(plans, tun)
        squeries, sparams, sbufs = db.shared_prepare(prog, plans)
        for t, n in db.rows.items():
            sctx.set_rows(t, n)

        def shared_step():
            sctx.shared_execute(prog.module, squeries, sparams, stream.cuda_stream)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            return [ev] * len(plans)

        for _ in range(args.warmup):
            shared_step()
        sctx.sync()
        barrier(pg, device)
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        shared_ms, shared_lat = time_steps(torch, stream, args.steps, shared_step)
        clocks = sampler.stop()
        sctx.sync()
        scan_ms = sctx.timing().scan_ms
        shared_ms = max_over_ranks(pg, shared_ms, device)
        shared_bytes = len(union_cols) * 4 * args.rows
        shared = {"ms_per_step": shared_ms / args.steps, "scan_ms": scan_ms, "bytes": shared_bytes,
                  "lat": shared_lat, "launches": sctx.timing().gpu_launches,
                  "tuning": {k: getattr(tun, k) for k, _ in _lib.Tuning._fields_} if tun else None}
    else:
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        _, _ = time_steps(torch, stream, 1, plain_step)
        clocks = sampler.stop()
        for c in ctxs:
            c.sync()
    barrier(pg, device)

    # ---- end to end through the public API: per-step descriptor upload and
    # every query's result read back to pinned host memory
    e2e_steps = max(2, args.steps)
    if shared is not None:
        pinned = [torch.empty(r.numel(), dtype=torch.int64, pin_memory=True) for r, _, _ in sbufs]
        pinned_v = [torch.empty(v.numel(), dtype=torch.int64, pin_memory=True) for _, v, _ in sbufs]
        h2d = len(squeries) * 40 + len(sparams) * 4
        d2h = sum(p.numel() * 8 + q.numel() * 8 for p, q in zip(pinned, pinned_v))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            prog2 = db.shared_program(plans, db.shared_tuning_for(plans))
            q2, p2, _ = squeries, sparams, None
            sctx.shared_execute(prog2.module, q2, p2, stream.cuda_stream)
            for i, (r, v, _) in enumerate(sbufs):
                pinned[i].copy_(r, non_blocking=True)
                pinned_v[i].copy_(v, non_blocking=True)
            stream.synchronize()
        e2e_s = time.perf_counter() - t0
    else:
        pinned = [torch.empty(r.numel(), dtype=torch.int64, pin_memory=True) for r, _ in results]
        pinned_v = [torch.empty(v.numel(), dtype=torch.int64, pin_memory=True) for _, v in results]
        h2d = 0
        d2h = sum(p.numel() * 8 + q.numel() * 8 for p, q in zip(pinned, pinned_v))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for i, (m, c) in enumerate(zip(mods, ctxs)):
                c.execute(db.compile(plans[i], db.tuning_for(plans[i])), stream.cuda_stream)
                pinned[i].copy_(results[i][0], non_blocking=True)
                pinned_v[i].copy_(results[i][1], non_blocking=True)
            stream.synchronize()
        e2e_s = time.perf_counter() - t0
    e2e = {"value": len(plans) * e2e_steps * world / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h),
           "note": "fact table resident in HBM; query descriptors uploaded and every result read back each step"}

    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0 and shared is not None:
        try:
            serving = serving_leg(db, plans, args, db.shared_tuning_for(plans))
        except Exception as e:  # reported, not fatal
            serving = {"error": str(e)[:300]}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(plans, args, args.rows)
        except Exception as e:  # reported, not fatal
            cb = {"value": None, "unit": "queries/s", "error": str(e)[:200]}

    if rank == 0:
        if shared is not None:
            value = job_rate(len(plans) * args.steps, world, shared["ms_per_step"] * args.steps)
            ms_step = shared["ms_per_step"]
            lat = shared["lat"]
            achieved = shared["bytes"] / (shared["scan_ms"] / 1000.0) / 1e9
            kernel = "SharedScan_LINEORDER (one pass over the union of the batch's fact columns)"
            launches = shared["launches"]
            alg = f"union of fact columns read by the batch ({len(union_cols)}) x 4 B x rows, per launch"
        else:
            value = plain["queries_per_s"]
            ms_step = plain["ms_per_step"]
            lat = plain_lat
            achieved = plain["scan_GBps"]
            kernel = "Scan_LINEORDER (plain fused scan/probe/aggregate)"
            launches = plain_launches
            alg = "distinct fact columns read x 4 B x rows, per query"
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/u64", "data": "synthetic",
            "config": config_block(args),
            "latency_ms": {"p50": statistics.median(lat), "p99": float(np.percentile(lat, 99)),
                           "definition": "query completion since its batch started"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (SHARED_DRAM_BYTES_PER_ROW * args.rows / 1e9) if shared is not None else None,
                         "traffic_unit": "GB per launch (ncu capture of 30M rows scaled by rows)",
                         "kernel": kernel, "algorithmic_bytes": alg},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
            "cpu_baseline": cb,
            "plain": plain,
            "shared_vs_plain": (value / plain["queries_per_s"]) if shared is not None else 1.0,
            "shared_tuning": shared["tuning"] if shared is not None else None,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
