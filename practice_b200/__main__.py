"""Command-line runner: one workload on a generated SSB-shaped table.

    python -m practice_b200 shared --rows 30000000 --batch 32 --reps 3
    python -m practice_b200 plain --rows 30000000 --query T1 --reps 3
    python -m practice_b200 shared ... --tuning block_threads=1024 items_per_thread=1 stages=3

`shared` runs a mixed batch from the four query templates as one shared scan;
`plain` runs one query (a template, the SSB Q1.1 / Q3.1 shapes, an OR-join or
a multi-value hash join) as its own fused kernel.  Each repetition prints the device time of the scan kernel.
Used for kernel profiles: every repetition launches the same kernels on the
same resident tables.
"""
from __future__ import annotations

import argparse
import random


def _tuning(pairs: list[str]):
    from practice_b200.engine import SHARED_DEFAULT, make_tuning

    kw = {}
    for p in pairs:
        k, v = p.split("=", 1)
        kw[k] = int(v)
    return kw, SHARED_DEFAULT, make_tuning


def main(argv: list[str] | None = None) -> None:
    ap = argparse.ArgumentParser(prog="python -m practice_b200")
    ap.add_argument("mode", choices=["shared", "plain", "tour"])
    ap.add_argument("--rows", type=int, default=30_000_000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--query", default="T1", help="T0..T3, q11, q31, q31n (nullable Q3.1) or one of " + ", ".join(EXPANDING) +
                    " (plain mode)")
    ap.add_argument("--template", type=int, default=-1, help="shared mode: draw every query from this template")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tuning", nargs="*", default=[], help="key=value launch-shape overrides")
    args = ap.parse_args(argv)

    from practice_b200 import queries
    from practice_b200.engine import Database

    if args.mode == "tour":
        tour(args)
        return
    kw, shared_default, make_tuning = _tuning(args.tuning)
    cols = {"q11": queries.Q11_COLS, "q31": queries.Q31_COLS, "q31n": queries.Q31_COLS}.get(args.query, queries.BATCH_COLS)
    # The nullable Q3.1 shape reads 10 % NULL revenue and 5 % NULL c_city.
    nulls = {"lo_revenue": 100, "c_city": 50} if args.query == "q31n" else None
    dims = ("DDATE", "CUSTOMER", "SUPPLIER", "PART")
    if args.query in EXPANDING:
        cols = sorted(set(queries.OR_COLS) | set(queries.MHT_COLS))
        dims = dims + ("PARTSUPP",)
    db = Database(0)
    db.generate_ssb(args.rows, args.seed, queries.BATCH_COLS if args.mode == "shared" else cols, nulls=nulls, dims=dims)
    if args.mode == "shared":
        if args.template >= 0:
            rng = random.Random(args.seed)
            plans = [queries.template(args.template, rng, args.rows) for _ in range(args.batch)]
        else:
            plans = queries.batch(args.batch, args.seed, args.rows)
        t = make_tuning(**{**shared_default, **kw})
        for _ in range(args.reps):
            r = db.execute_shared(plans, t)
            path = "aggregate cubes" if r[0].timing.mode == 1 else "per-query masks"
            print(f"shared batch of {len(plans)} ({path}): scan {r[0].timing.scan_ms:.4f} ms, "
                  f"total {r[0].timing.total_ms:.4f} ms, kernel error {r[0].kernel_error}", flush=True)
        return
    q = args.query
    if q.startswith("T"):
        plan = queries.template(int(q[1:]), random.Random(args.seed), args.rows)
    elif q == "q11":
        plan = queries.ssb_q11(args.rows)
    elif q in EXPANDING:
        plan = getattr(queries, EXPANDING[q])(args.rows)
    elif q == "q31n":
        plan = queries.ssb_q31_nullable(args.rows)
    else:
        plan = queries.ssb_q31(args.rows)
    t = make_tuning(**kw) if kw else None
    for _ in range(args.reps):
        r = db.execute(plan, t)
        print(f"{plan.name}: build {r.timing.build_ms:.4f} ms, scan {r.timing.scan_ms:.4f} ms, "
              f"total {r.timing.total_ms:.4f} ms, kernel error {r.kernel_error}", flush=True)


# Plain-mode names of the OR-join and multi-value hash join queries.
EXPANDING = {"or_year": "or_join_year", "or_filter": "or_join_then_filter", "mht_tier": "mht_year_tier",
             "mht_supp": "mht_then_supplier", "mht_brand": "mht_brand"}



def tour(args) -> None:
    """Runs every kernel of the library once or twice on a generated table:
    the plain fused scan (Q1.1-, Q3.1- and nullable Q3.1-shaped queries, a
    parametric one, AVG finalisation, an OR-join and two multi-value hash
    joins with their five build kernels), a shared-scan batch, result
    finalisation on the device and sparse compaction (both entry points)."""
    import numpy as np

    from practice_b200 import _lib, queries
    from practice_b200.engine import SHARED_DEFAULT, Database, make_tuning
    from practice_b200.plan import PlanBuilder, col

    cols = sorted(set(queries.BATCH_COLS) | set(queries.Q11_COLS) | set(queries.OR_COLS))
    db = Database(0)
    db.generate_ssb(args.rows, args.seed, cols, nulls={"c_city": 50},
                    dims=("DDATE", "CUSTOMER", "SUPPLIER", "PART", "PARTSUPP"))
    torch = db.torch
    rng = random.Random(args.seed)
    plans = [queries.ssb_q11(args.rows), queries.ssb_q31(args.rows), queries.ssb_q31_nullable(args.rows)]
    b = PlanBuilder(queries.ssb_tables(args.rows, cols), "LINEORDER", name="avg")
    b.join("DDATE", "lo_orderdate")
    plans.append(b.aggregate([queries._g("d_year")], [("avg", col("lo_supplycost")), ("min", col("lo_quantity"))]))
    plans += [queries.or_join_year(args.rows), queries.mht_year_tier(args.rows), queries.mht_brand(args.rows)]
    for p in plans:
        m = db.compile(p)
        res, val = db.alloc_result(m)
        db.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
        db.ctx.execute(m, torch.cuda.current_stream().cuda_stream)
        db.ctx.sync()
        rows = db.finalize_rows(p, res, val, limit=20)
        print(f"{p.name}: scan {db.ctx.timing().scan_ms:.3f} ms, {len(rows)} rows after device finalisation")
    t = make_tuning(parametric=1)
    p = queries.template(2, rng, args.rows)
    r = db.execute(p, t)
    print(f"parametric {p.name}: scan {r.timing.scan_ms:.3f} ms")
    batch = [queries.template(rng.randrange(4), rng, args.rows) for _ in range(args.batch)]
    r = db.execute_shared(batch, make_tuning(**SHARED_DEFAULT))
    print(f"shared batch of {len(batch)}: scan {r[0].timing.scan_ms:.3f} ms")
    words = torch.from_numpy(r[1].words.view(np.int64).copy()).to(db.device)
    groups = batch[1].group_slots
    ts = batch[1].storage_ts
    dst = torch.empty_like(words)
    cnt = torch.zeros(1, dtype=torch.int64, device=db.device)
    for fn in (_lib.lib.cx_compact_sparse, _lib.lib.cx_compact_sparse_noalloc):
        _lib.check(fn(words.data_ptr(), groups, ts, dst.data_ptr(), cnt.data_ptr(),
                      torch.cuda.current_stream().cuda_stream), "compaction")
    torch.cuda.synchronize()
    print(f"sparse compaction: {int(cnt.item())} groups")


if __name__ == "__main__":
    main()
