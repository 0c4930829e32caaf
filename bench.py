"""Benchmark: batched star-join queries on a 600,000,000-row fact table.

Workload (the headline metric's configuration): 8 int32 fact columns
(orderdate, custkey, suppkey, partkey, quantity, discount, revenue, supplycost;
19.2 GB resident in HBM) with the SSB-shaped date / customer / supplier / part
dimensions, and batches of 16, 32 or 64 queries drawn by seed from four
templates (T0 range filters + scalar SUM; T1 date join + GROUP BY year; T2
three joins + GROUP BY (nation, year); T3 four joins + GROUP BY (brand,
year)).  Synthetic data, generated on the device from a counter-based hash
(practice_b200/datagen.py).

One step = one batch of queries over the whole fact table.  The headline
(`value`) is the 32-query batch answered by one shared-scan launch; the same
queries as plain fused kernels one after another (the drop-in path) are timed
beside it, and both are timed at 16 and 64 queries too.  The JSON line also
carries: the roofline of the dominant kernel against the measured HBM
bandwidth; the CPU baseline (the reference's own primitives compiled for the
host, over the whole 600M-row table) whose results double as the parity check
of every GPU answer of the run; the plain single-query workloads at their own
sizes (6M-row SSB Q1.1 shape, 60M-row Q3.1 shape and its nullable variant),
each with kernel time, roofline, end-to-end rate, the reference CPU path at
full size and a bit-exact check; clocks sampled during the timed region; the
end-to-end figure through the public API; and the serving loop under Poisson
arrivals.

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
# B200 HBM3e nominal bandwidth (~8 TB/s), reported beside the measured copy peak.
NOMINAL_HBM_GBS = 8000.0
DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="shared", choices=["plain", "shared"])
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--batch-sizes", default="16,32,64", help="shared-scan batches timed beside the headline")
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-rows", type=int, default=40_000_000,
                    help="rows of each reference-arm step (a bounded sample of the table)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the 6M / 60M single-query legs")
    ap.add_argument("--config-rows", default="6000000,60000000", help="rows of the Q1.1 leg and the Q3.1 legs")
    ap.add_argument("--serve-rates", default="50,1000,2000", help="Poisson arrival rates of the serving leg (q/s)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="most requests per rate (0 skips the leg)")
    ap.add_argument("--serve-burst", type=int, default=128,
                    help="large-domain queries (330 MB results) submitted at once: more than the budget holds")
    ap.add_argument("--serve-chunk-rows", type=int, default=75_000_000,
                    help="row range of one launch of the circular loop (0 skips it)")
    ap.add_argument("--serve-slots", type=int, default=1, help="launches in flight in the shared loop")
    ap.add_argument("--serve-warm", type=int, default=256, help="untimed warm-up queries per serving loop")
    return ap.parse_args(argv)


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


def pct(xs, q):
    import numpy as np
    return float(np.percentile(xs, q)) if len(xs) else None


# ------------------------------------------------------------- CPU baseline


def reference_arm(args):
    """The reference's CPU path (its own crystal primitives compiled for the
    host with OpenMP, oracle/_ref; the oracle restatement where that library
    was not built) on the headline batch, each step a bounded row sample of
    the fact table, rate scaled to the whole table."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import refbase
    from practice_b200 import datagen, queries

    n = min(args.cpu_sample_rows, args.rows)
    ht = datagen.host_tables(args.seed, n, queries.BATCH_COLS)
    plans = queries.batch(args.batch, args.seed, n)
    times = []
    kind = cores = None
    for i in range(args.warmup + args.steps):
        t, kind, cores = refbase.time_batch(plans, ht, n)
        if i >= args.warmup:
            times.append(t)
    t = statistics.median(times)
    scale = args.rows / n
    v = len(plans) / (t * scale)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": len(plans) / v * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/u64",
        "data": "synthetic", "config": config_block(args),
        "cpu_baseline": {"value": v, "unit": "queries/s", "cores": cores, "kind": kind,
                         "sample": f"{len(plans)}-query batch on the first {n:,} of {args.rows:,} fact rows per step, "
                                   f"median {t:.3f} s scaled by {scale:.0f}x to the full table"},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args):
    return {"workload": "batched star-join queries from 4 templates over a 600M-row, 8-column int32 fact table",
            "fact_rows": args.rows, "fact_columns": 8, "batch_queries": args.batch, "mode": args.mode,
            "seed": args.seed, "parallelism": f"replicas{args.gpus}",
            "l2": "inputs (19.2 GB) larger than L2 (126 MB); no flush needed"}


# ------------------------------------------------------------------ GPU arm

# DRAM bytes (read + write) per fact row of one shared-scan launch over the
# 8-column batch table, by path: ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) of one 30M-row launch of the 32-query batch (per-query
# masks: 972.6 MB; aggregate cubes: 964.9 MB); the traffic of a launch grows
# with its rows.
SHARED_DRAM_BYTES_PER_ROW = {"masks": (968.457472e6 + 4.109056e6) / 30e6, "cube": (961.588480e6 + 3.345152e6) / 30e6}

PLAIN_CANDIDATES = [dict(block_threads=bt, items_per_thread=ipt, stages=st, ctas_per_sm=16, bitmap_budget=bm,
                         prefetch=pf, group_placement=pl, compact=cp, table_budget=tb)
                    for bt, ipt, st, bm, pf, pl, cp, tb in (
                        (1024, 4, 0, 49152, 1, 0, 0, 98304), (1024, 4, 0, 49152, 1, 0, 0, 0),
                        (1024, 4, 0, 0, 1, 4, 0, 0), (512, 2, 0, 0, 1, 4, 0, 0), (1024, 2, 0, 0, 0, 4, 0, 98304),
                        (512, 8, 4, 0, 0, 0, 0, 0), (1024, 4, 0, 49152, 1, 0, 1, 98304),
                        (512, 4, 0, 49152, 1, 0, 1, 98304), (1024, 2, 0, 49152, 1, 0, 1, 98304),
                        (1024, 2, 0, 49152, 1, 0, 1, 0), (1024, 4, 0, 49152, 1, 0, 2, 0),
                        (1024, 2, 0, 49152, 1, 0, 2, 0), (1024, 4, 0, 49152, 3, 0, 0, 98304),
                        (1024, 8, 0, 49152, 1, 0, 2, 0))]
# Per-query mask path (cube = 0) launch shapes, then the aggregate-cube path at
# 1, 2 and 4 rows per lane (the runtime falls back to the mask path when the
# batch's attribute ranges do not allow cubes).
SHARED_CANDIDATES = [dict(block_threads=bt, items_per_thread=ipt, stages=st, ctas_per_sm=2, producer_warps=pw,
                          group_merge=gm, cube=0)
                     for bt, ipt, st, pw, gm in ((1024, 1, 3, 11, 0), (1024, 1, 3, 11, 3), (1024, 1, 3, 14, 0),
                                                 (1024, 1, 3, 14, 3), (512, 2, 2, 5, 0), (512, 2, 2, 7, 3))]
SHARED_CANDIDATES += [dict(block_threads=1024, items_per_thread=1, stages=3, ctas_per_sm=2, producer_warps=11,
                           group_merge=3, cube=c) for c in (1, 2, 4)]


def bound_ctx(db, module, res, val):
    """A C-ABI execution context bound to the database's tables and one result buffer."""
    from practice_b200 import _lib

    c = _lib.ExecCtx()
    for name, t in db.cols.items():
        c.set_buffer("d_" + name, t.data_ptr(), t.numel())
    for name, t in db.valid.items():
        c.set_null_bitmap("d_" + name, t.data_ptr(), t.numel())
    for t, n in db.rows.items():
        c.set_rows(t, n)
    c.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
    return c


def result_words(res, val, final_words):
    import numpy as np
    w = res.cpu().numpy().view(np.uint64)[:final_words].copy()
    v = val.cpu().numpy().view(np.uint64)[: (final_words + 63) // 64].copy()
    return w, v


def plain_leg(torch, db, plans, stream, args, pg, device):
    """Every plan as its autotuned plain fused kernel, one after another.
    Returns the timing summary, per-step per-query durations and results."""
    for p in plans:
        if db.tuning_for(p) is None:
            db.autotune(p, candidates=PLAIN_CANDIDATES, reps=1, persist=False)
    mods = [db.compile(p, db.tuning_for(p)) for p in plans]
    bufs = [db.alloc_result(m) for m in mods]
    ctxs = [bound_ctx(db, m, r, v) for m, (r, v) in zip(mods, bufs)]

    def step():
        evs = []
        for m, c in zip(mods, ctxs):
            c.execute(m, stream.cuda_stream)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            evs.append(ev)
        return evs

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    for c in ctxs:
        c.sync()
    barrier(pg, device)
    starts, marks = [], []
    for _ in range(args.steps):
        s0 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        starts.append(s0)
        marks.append(step())
    stream.synchronize()
    scan_ms = []
    for c in ctxs:
        c.sync()
        scan_ms.append(c.timing().scan_ms)
    launches = sum(c.timing().gpu_launches for c in ctxs)
    # durations[s][i]: query i of step s, from the previous query's end
    durations = []
    for s0, evs in zip(starts, marks):
        prev, d = s0, []
        for ev in evs:
            d.append(prev.elapsed_time(ev))
            prev = ev
        durations.append(d)
    results = [result_words(r, v, int(m.info.final_words)) for m, (r, v) in zip(mods, bufs)]
    for c in ctxs:
        c.close()
    return {"scan_ms": scan_ms, "durations": durations, "launches_per_step": launches,
            "tunings": [db.tuning_for(p) for p in plans]}, results


def plain_summary(pl, plans, b, args, world, pg, device, peak):
    import numpy as np
    per_step = [sum(d[:b]) for d in pl["durations"]]
    ms = max_over_ranks(pg, sum(per_step), device)
    lat = [sum(d[: i + 1]) for d in pl["durations"] for i in range(b)]
    byts = sum(len(p.columns_read()) * 4 * args.rows for p in plans[:b])
    scan_s = sum(pl["scan_ms"][:b]) / 1000.0
    return {"queries_per_s": job_rate(b * args.steps, world, ms), "ms_per_step": ms / args.steps,
            "p50_ms": statistics.median(lat), "p99_ms": pct(lat, 99),
            "scan_GBps": byts / scan_s / 1e9, "scan_frac_of_peak": byts / scan_s / 1e9 / peak,
            "scan_ms": {"mean": float(np.mean(pl["scan_ms"][:b])), "min": min(pl["scan_ms"][:b]),
                        "max": max(pl["scan_ms"][:b])}}


def shared_leg(torch, db, plans, stream, args, pg, device, sample_clocks: bool):
    """The batch as one shared-scan launch per step (autotuned launch shape)."""
    from practice_b200 import _lib

    if db.shared_tuning_for(plans) is None:
        db.autotune_shared(plans, SHARED_CANDIDATES, reps=1)
    tun = db.shared_tuning_for(plans)
    prog = db.shared_program(plans, tun)
    squeries, sparams, sbufs, sarena = db.shared_prepare_arena(prog, plans)
    sctx = db.ctx
    for t, n in db.rows.items():
        sctx.set_rows(t, n)

    def step():
        sctx.shared_execute(prog.module, squeries, sparams, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    sctx.sync()
    barrier(pg, device)
    sampler = None
    if sample_clocks:
        sampler = ClockSampler(device.index)
        sampler.start()
        time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    scan = []
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    end.synchronize()
    clocks = sampler.stop() if sampler else None
    sctx.sync()
    ms = max_over_ranks(pg, start.elapsed_time(end), device)
    tm = sctx.timing()
    scan.append(tm.scan_ms)
    results = [result_words(r, v, words) for r, v, words in sbufs]
    return {"ms_per_step": ms / args.steps, "scan_ms": tm.scan_ms, "launches_per_step": tm.gpu_launches,
            "graph": tm.graph, "path": "cube" if tm.mode == 1 else "masks", "tuning": {k: getattr(tun, k) for k, _ in _lib.Tuning._fields_} if tun else None,
            "prog": prog, "squeries": squeries, "sparams": sparams, "sbufs": sbufs, "sarena": sarena,
            "clocks": clocks}, results


def e2e_shared(torch, db, plans, sh, stream, args, world):
    """The batch end to end through the public API: the query descriptors and
    literals uploaded, the shared scan, and every query's result and validity
    words read back to pinned host memory (one copy of the batch's result
    arena), each step."""
    sctx = db.ctx
    arena = sh["sarena"]
    pinned = torch.empty(arena.numel(), dtype=torch.int64, pin_memory=True)
    h2d = len(sh["squeries"]) * 40 + len(sh["sparams"]) * 4
    d2h = pinned.numel() * 8
    steps = max(2, args.steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        prog = db.shared_program(plans, db.shared_tuning_for(plans))
        sctx.shared_execute(prog.module, sh["squeries"], sh["sparams"], stream.cuda_stream)
        with torch.cuda.stream(stream):
            pinned.copy_(arena, non_blocking=True)
        stream.synchronize()
    e2e_s = time.perf_counter() - t0
    return {"value": len(plans) * steps * world / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h),
            "note": "fact table resident in HBM; query descriptors uploaded and every result read back each step"}


def compare(results, accs, validity: bool = False):
    """Indexes of GPU result buffers that differ from the combined CPU results
    (result words always; validity words too when the checker computes them)."""
    import numpy as np
    bad = []
    for i, ((w, v), a) in enumerate(zip(results, accs)):
        fw = len(w)
        if not np.array_equal(w, a.words[:fw]) or (validity and not np.array_equal(v, a.validity[: (fw + 63) // 64])):
            bad.append(i)
    return bad


def batch_cpu_and_parity(db, plans_all, plain_results, shared_results, args):
    """The reference's CPU path over the whole 600M-row table (range by range,
    copied back from the device) for every query of the largest batch: its
    time is the CPU baseline of the headline batch, its results check every
    GPU answer of the run."""
    from oracle import chunked, refharness
    from practice_b200 import queries

    dims, _, dim_rows = chunked.device_dims(db)
    fetch = chunked.device_fetch(db, queries.BATCH_COLS)
    if refharness.available():
        accs, spent, cores = chunked.run_reference(plans_all, fetch, args.rows, dims, dim_rows,
                                                   chunk_rows=25_000_000)
        kind = "reference"
        head_s = sum(a.seconds for a in accs[: args.batch])
    else:
        head, spent, cores = chunked.run_oracle(plans_all[: args.batch], fetch, args.rows, dims, {}, dim_rows,
                                                chunk_rows=25_000_000)
        rest, _, _ = chunked.run_oracle(plans_all[args.batch:], fetch, args.rows, dims, {}, dim_rows,
                                        chunk_rows=25_000_000) if len(plans_all) > args.batch else ([], 0, 0)
        accs = head + rest
        kind = "port"
        head_s = spent
    parity = {"checker": "reference primitives (oracle/_ref)" if kind == "reference" else "oracle restatement",
              "fact_rows": args.rows, "queries": len(plans_all)}
    bad_plain = compare(plain_results, accs, validity=kind == "port")
    parity["plain_bit_exact"] = not bad_plain
    for b, res in shared_results.items():
        bad = compare(res, accs[:b], validity=kind == "port")
        parity[f"shared_{b}_bit_exact"] = not bad
        if bad:
            parity[f"shared_{b}_mismatch"] = bad[:8]
    if bad_plain:
        parity["plain_mismatch"] = bad_plain[:8]
    parity["bit_exact"] = all(v for k, v in parity.items() if k.endswith("bit_exact"))
    cb = {"value": args.batch / head_s, "unit": "queries/s", "cores": cores, "kind": kind,
          "sample": f"the whole {args.rows:,}-row table in 25M-row ranges, the {args.batch}-query batch "
                    f"({head_s:.1f} s inside the reference calls; no extrapolation)"}
    return cb, parity


# ----------------------------------------------------- single-query configs


def config_leg(torch, name, plan_fn, rows, cols, nulls, args, device, peak, stream):
    """One plain fused query at its own table size: kernel time and roofline,
    end to end through the C ABI with the result read back, the reference's
    CPU path over the whole table, and a bit-exact check of the GPU result."""
    import numpy as np

    from oracle import chunked, refharness
    from practice_b200.engine import Database

    db = Database(device.index)
    db.generate_ssb(rows, args.seed, cols, nulls=nulls)
    plan = plan_fn(rows)
    db.autotune(plan, candidates=PLAIN_CANDIDATES, reps=2, persist=False)
    tun = db.tuning_for(plan)
    m = db.compile(plan, tun)
    res, val = db.alloc_result(m)
    ctx = bound_ctx(db, m, res, val)
    for _ in range(max(3, args.warmup)):
        ctx.execute(m, stream.cuda_stream)
    ctx.sync()
    scan, total = [], []
    reps = max(10, args.steps)
    for _ in range(reps):
        ctx.execute(m, stream.cuda_stream)
        ctx.sync()
        t = ctx.timing()
        scan.append(t.scan_ms)
        total.append(t.total_ms)
    launches = ctx.timing().gpu_launches
    fw = int(m.info.final_words)
    got = result_words(res, val, fw)
    # End to end: execute + result and validity words to pinned host memory.
    pin = torch.empty(res.numel(), dtype=torch.int64, pin_memory=True)
    pin_v = torch.empty(val.numel(), dtype=torch.int64, pin_memory=True)
    torch.cuda.synchronize()
    e2e = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ctx.execute(m, stream.cuda_stream)
        pin.copy_(res, non_blocking=True)
        pin_v.copy_(val, non_blocking=True)
        stream.synchronize()
        e2e.append(time.perf_counter() - t0)
    ctx.close()
    nullable_read = [c for c in plan.columns_read() if c in (nulls or {})]
    byts = len(plan.columns_read()) * 4 * rows + len(nullable_read) * rows / 8
    scan_s = statistics.median(scan) / 1000.0
    # The reference's CPU path over the whole table, from the device-resident rows.
    dims, dval, dim_rows = chunked.device_dims(db)
    fetch = chunked.device_fetch(db, cols)
    try:
        if refharness.available() and not nulls:
            (acc,), cpu_s, cores = chunked.run_reference([plan], fetch, rows, dims, dim_rows,
                                                          chunk_rows=30_000_000)
            kind = "reference"
        else:
            (acc,), cpu_s, cores = chunked.run_oracle([plan], fetch, rows, dims, dval, dim_rows,
                                                       chunk_rows=30_000_000)
            kind = "port"
        exact = not compare([got], [acc], validity=kind == "port")
        cpu = {"value": 1.0 / cpu_s, "unit": "queries/s", "rows_per_s": rows / cpu_s, "cores": cores, "kind": kind,
               "sample": f"the whole {rows:,}-row table"}
    except Exception as e:  # reported, not fatal
        exact, cpu = None, {"error": str(e)[:200]}
    db.reset()
    del db
    torch.cuda.empty_cache()
    gpu_qps = 1000.0 / statistics.median(total)
    return {"workload": name, "fact_rows": rows, "columns_read": len(plan.columns_read()),
            "scan_ms": {"median": statistics.median(scan), "min": min(scan)},
            "query_ms": statistics.median(total),
            "rows_per_s": rows / scan_s,
            "queries_per_s": gpu_qps,
            "roofline": {"bound": "hbm", "achieved": byts / scan_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": byts / scan_s / 1e9 / peak, "frac_of_nominal": byts / scan_s / 1e9 / NOMINAL_HBM_GBS,
                         "algorithmic_bytes": byts},
            "e2e": {"value": 1.0 / statistics.median(e2e), "unit": "queries/s",
                    "rows_per_s": rows / statistics.median(e2e), "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(res.numel() * 8 + val.numel() * 8)},
            "gpu_launches_per_query": launches,
            "tuning": {k: getattr(tun, k) for k in ("block_threads", "items_per_thread", "stages", "group_placement",
                                                     "bitmap_budget", "prefetch", "compact", "table_budget")}
            if tun else None,
            "cpu_baseline": cpu,
            "gpu_vs_cpu": (rows / scan_s) / cpu["rows_per_s"] if "rows_per_s" in cpu else None,
            "parity": {"bit_exact": exact, "checker": cpu.get("kind")}}


def configs_legs(torch, args, device, peak, stream):
    from practice_b200 import queries

    q11_rows, q31_rows = (int(x) for x in args.config_rows.split(","))
    return {
        "q11_6M": config_leg(torch, "SSB Q1.1 shape: date join (year = 1995), discount in [2,4], quantity < 30, "
                                    "SUM(extendedprice*discount)", queries.ssb_q11, q11_rows, queries.Q11_COLS,
                             None, args, device, peak, stream),
        "q31_60M": config_leg(torch, "SSB Q3.1 shape: customer/supplier/date joins, GROUP BY (c_nation, s_nation, "
                                     "d_year), SUM(revenue)", queries.ssb_q31, q31_rows, queries.Q31_COLS, None,
                              args, device, peak, stream),
        "q31_nullable_60M": config_leg(torch, "nullable Q3.1: 10% NULL revenue, 5% NULL c_city, IS [NOT] NULL, "
                                              "COUNT(*), COUNT(revenue), SUM(revenue)", queries.ssb_q31_nullable,
                                       q31_rows, queries.Q31_COLS, {"lo_revenue": 100, "c_city": 50}, args,
                                       device, peak, stream),
    }


# -------------------------------------------------------------- serving


def serving_leg(db, args, shared_tuning):
    """The request loop under Poisson arrival streams of fresh queries (the
    four templates with new constants per request, and 5 % many-group queries
    of up to 62,500 groups): the shared loop (continuous batching into shared
    scans), the circular loop (launches over row ranges that queries join at
    any boundary) and the plain one-query-at-a-time loop over the same streams
    at several rates, each query's latency alone on an idle GPU, and a burst of
    large-domain queries (330 MB results each) that the 40 GiB admission budget
    has to hold back."""
    import numpy as np

    from practice_b200 import _lib, queries
    from practice_b200.engine import shape_key

    rates = [float(x) for x in args.serve_rates.split(",") if x]
    counts = [min(args.serve_requests, max(200, int(r * 2))) for r in rates]
    plans = queries.serving_stream(sum(counts) + 64, args.seed + 7, args.rows)
    reps = {}
    for p in plans:
        reps.setdefault(shape_key(p), p)
    for p in reps.values():  # the plain kernels of every shape, autotuned
        if db.tuning_for(p) is None:
            db.autotune(p, candidates=PLAIN_CANDIDATES, reps=1, persist=False)
    texts = [p.text() for p in plans]
    # Untimed warm-up queries (same mix, other constants): a loop's first
    # launches grow its pinned result landing area and device scratch and run
    # the one-off dimension checks; the timed streams start after them.
    warm_texts = [p.text() for p in queries.serving_stream(args.serve_warm, args.seed + 13, args.rows)]

    warm_failed = []

    def warm(srv):
        ids = [srv.submit(t) for t in warm_texts]
        bad = 0
        for rid in ids:
            info = srv.wait(rid)
            bad += int(info.status != 0 or info.kernel_error != 0)
            srv.release(rid)
        warm_failed.append(bad)

    def stream(srv, rate, first, n):
        rng = np.random.default_rng(args.seed + int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        srv.stats(reset=True)
        ids = []
        t0 = time.perf_counter()
        for i in range(n):
            target = t0 + arrivals[i]
            while time.perf_counter() < target:
                pass
            ids.append(srv.submit(texts[first + i]))
        bad = 0
        for rid in ids:
            info = srv.wait(rid)
            bad += int(info.status != 0 or info.kernel_error != 0)
            srv.release(rid)
        st = srv.stats()
        return {"requests": n, "queries_per_s": st.queries_per_s, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                "max_ms": st.max_ms, "mean_batch": st.mean_batch, "launches": int(st.launches), "failed": bad,
                "peak_reserved_GB": st.peak_reserved_bytes / 1e9}

    out = {"arrivals": "Poisson; fresh constants per request from the 4 templates, 5% many-group queries "
                       "(GROUP BY c_city, s_city: up to 62,500 groups); budget 40 GiB",
           "warmup": f"each loop answers {len(warm_texts)} untimed queries of the same mix, submitted at once, "
                     "before its timed streams", "rates": {}}
    plain = _lib.Server(db.ctx, _lib.server_config(plain_only=1, slots=1))
    lone = []
    try:
        for p in reps.values():
            plain.prepare(p.text(), db.tuning_for(p))
        warm(plain)
        for t in texts[-64:]:  # queries alone on an idle GPU, submit to result on the host
            for _ in range(2):
                info = plain.wait(plain.submit(t))
            lone.append(info.latency_ms)
        first = 0
        for r, n in zip(rates, counts):
            out["rates"][str(int(r))] = {"plain_loop": stream(plain, r, first, n)}
            first += n
    finally:
        plain.close()
    lone_ms = float(np.median(lone))
    out["lone_query_ms"] = {"median": lone_ms, "p99": float(np.percentile(lone, 99)), "max": float(np.max(lone))}
    # The circular loop: each shared launch scans the next range of
    # serve_chunk_rows rows, so an arrival waits for one range, not a whole scan.
    if args.serve_chunk_rows > 0:
        cfg = _lib.server_config(max_batch=64, slots=args.serve_slots, chunk_rows=args.serve_chunk_rows)
        if shared_tuning is not None:
            cfg.shared_tuning = shared_tuning
        srv = _lib.Server(db.ctx, cfg)
        try:
            for p in reps.values():
                srv.prepare(p.text(), db.tuning_for(p))
            warm(srv)
            first = 0
            for r, n in zip(rates, counts):
                row = out["rates"][str(int(r))]
                row["circular_loop"] = stream(srv, r, first, n)
                row["circular_p99_vs_lone"] = row["circular_loop"]["p99_ms"] / lone_ms
                first += n
        finally:
            srv.close()
        out["circular_chunk_rows"] = args.serve_chunk_rows
    cfg = _lib.server_config(max_batch=64, slots=args.serve_slots)
    if shared_tuning is not None:
        cfg.shared_tuning = shared_tuning
    srv = _lib.Server(db.ctx, cfg)
    try:
        for p in reps.values():  # short queues run these autotuned plain kernels
            srv.prepare(p.text(), db.tuning_for(p))
        warm(srv)
        first = 0
        for r, n in zip(rates, counts):
            row = out["rates"][str(int(r))]
            row["shared_loop"] = stream(srv, r, first, n)
            row["shared_vs_plain_queries_per_s"] = row["shared_loop"]["queries_per_s"] / max(
                row["plain_loop"]["queries_per_s"], 1e-9)
            row["shared_p99_vs_lone"] = row["shared_loop"]["p99_ms"] / lone_ms
            row["plain_p99_vs_lone"] = row["plain_loop"]["p99_ms"] / lone_ms
            first += n
        # Burst: more large queries than the budget holds at once.
        import random as _random
        rng = _random.Random(args.seed + 11)
        wide = [queries.wide_groups(rng, args.rows).text() for _ in range(args.serve_burst)]
        srv.stats(reset=True)
        t0 = time.perf_counter()
        ids = [srv.submit(t) for t in wide]
        bad = 0
        for rid in ids:
            info = srv.wait(rid)
            bad += int(info.status != 0 or info.kernel_error != 0)
            srv.release(rid)
        st = srv.stats()
        out["burst"] = {"queries": len(wide), "result_MB_each": 330.0, "wall_s": time.perf_counter() - t0,
                        "peak_reserved_GB": st.peak_reserved_bytes / 1e9, "budget_GB": (40 << 30) / 1e9,
                        "failed": bad, "launches": int(st.launches), "mean_batch": st.mean_batch}
    finally:
        srv.close()
    out["warmup_failed"] = sum(warm_failed)
    return out


# ----------------------------------------------------------------- main


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch

    from practice_b200 import queries
    from practice_b200.engine import Database

    world, rank, local, pg = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    peak, peak_kind = peaks()
    stream = torch.cuda.Stream(device)
    sizes = sorted({int(x) for x in args.batch_sizes.split(",") if x} | {args.batch})
    nmax = max(sizes)

    # Single-query workloads first, each on its own table (freed afterwards).
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = configs_legs(torch, args, device, peak, stream)

    db = Database(local)
    db.generate_ssb(args.rows, args.seed + rank, queries.BATCH_COLS)
    plans_all = queries.batch(nmax, args.seed, args.rows)  # smaller batches are its prefixes
    plans = plans_all[: args.batch]
    union_cols = sorted({c for p in plans for c in p.columns_read()})

    # ---- plain path: one fused kernel per query, one query after another
    pl, plain_results = plain_leg(torch, db, plans_all, stream, args, pg, device)
    plain = plain_summary(pl, plans_all, args.batch, args, world, pg, device, peak)
    plain_by_batch = {b: plain_summary(pl, plans_all, b, args, world, pg, device, peak) for b in sizes}

    # ---- shared scan: each batch in one persistent kernel; the headline batch last (clocks sampled)
    shared_all, shared_results = {}, {}
    if args.mode == "shared" and all(db.shareable(p) for p in plans_all):
        for b in [s for s in sizes if s != args.batch] + [args.batch]:
            sh, res = shared_leg(torch, db, plans_all[:b], stream, args, pg, device, sample_clocks=b == args.batch)
            shared_all[b] = sh
            shared_results[b] = res
    shared = shared_all.get(args.batch)
    if shared is not None:
        clocks = shared["clocks"]
    else:
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        plain_leg(torch, db, plans, stream, args, pg, device)
        clocks = sampler.stop()
    barrier(pg, device)

    # ---- end to end through the public API
    if shared is not None:
        e2e = e2e_shared(torch, db, plans, shared, stream, args, world)
    else:
        e2e = {"value": plain["queries_per_s"], "unit": "queries/s", "h2d_bytes_per_step": 0,
               "d2h_bytes_per_step": 0, "note": "plain mode: results stay on the device"}

    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0 and shared is not None:
        try:
            serving = serving_leg(db, args, db.shared_tuning_for(plans))
        except Exception as e:  # reported, not fatal
            serving = {"error": str(e)[:300]}

    cb, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, parity = batch_cpu_and_parity(db, plans_all, plain_results, shared_results, args)
        except Exception as e:  # reported, not fatal
            cb = {"value": None, "unit": "queries/s", "error": str(e)[:200]}

    if rank == 0:
        if shared is not None:
            value = job_rate(len(plans) * args.steps, world, shared["ms_per_step"] * args.steps)
            ms_step = shared["ms_per_step"]
            achieved = len(union_cols) * 4 * args.rows / (shared["scan_ms"] / 1000.0) / 1e9
            kernel = ("CubeScan_LINEORDER (one pass over the union of the batch's fact columns, one aggregate-cube "
                      "cell update per row and plan shape)" if shared["path"] == "cube" else
                      "SharedScan_LINEORDER (one pass over the union of the batch's fact columns, per-query row masks)")
            launches = shared["launches_per_step"]
            alg = f"union of fact columns read by the batch ({len(union_cols)}) x 4 B x rows, per launch"
            lat = {"p50": ms_step, "p99": ms_step, "definition": "every query of a batch completes with its launch"}
        else:
            value = plain["queries_per_s"]
            ms_step = plain["ms_per_step"]
            achieved = plain["scan_GBps"]
            kernel = "Scan_LINEORDER (plain fused scan/probe/aggregate)"
            launches = pl["launches_per_step"] * len(plans) // len(plans_all)
            alg = "distinct fact columns read x 4 B x rows, per query"
            lat = {"p50": plain["p50_ms"], "p99": plain["p99_ms"], "definition": "query completion since its batch started"}
        batches = {}
        for b in sizes:
            row = {"plain": plain_by_batch[b]}
            if b in shared_all:
                s = shared_all[b]
                ucols = sorted({c for p in plans_all[:b] for c in p.columns_read()})
                s_qps = job_rate(b * args.steps, world, s["ms_per_step"] * args.steps)
                row["shared"] = {"queries_per_s": s_qps, "ms_per_step": s["ms_per_step"], "scan_ms": s["scan_ms"],
                                 "roofline_frac": len(ucols) * 4 * args.rows / (s["scan_ms"] / 1000.0) / 1e9 / peak,
                                 "graph": s["graph"], "path": s["path"], "tuning": s["tuning"]}
                row["shared_vs_plain"] = s_qps / plain_by_batch[b]["queries_per_s"]
            batches[str(b)] = row
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/u64", "data": "synthetic",
            "config": config_block(args),
            "latency_ms": lat,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "nominal_peak": NOMINAL_HBM_GBS, "frac_of_nominal": achieved / NOMINAL_HBM_GBS,
                         "traffic": (SHARED_DRAM_BYTES_PER_ROW[shared["path"]] * args.rows / 1e9
                                     if shared is not None and SHARED_DRAM_BYTES_PER_ROW.get(shared["path"]) else None),
                         "traffic_unit": "GB per launch (ncu capture of 30M rows scaled by rows)",
                         "kernel": kernel, "algorithmic_bytes": alg},
            "clocks": clocks, "e2e": e2e,
            "gpu_launches": launches * args.steps, "gpu_launches_per_step": launches,
            "cpu_baseline": cb,
            "parity": parity,
            "plain": plain,
            "shared_vs_plain": (value / plain["queries_per_s"]) if shared is not None else 1.0,
            "batches": batches,
            "shared_tuning": shared["tuning"] if shared is not None else None,
            "configs": configs,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
