"""Command-line runner: one workload on a generated SSB-shaped table.

    python -m practice_b200 shared --rows 30000000 --batch 32 --reps 3
    python -m practice_b200 plain --rows 30000000 --query T1 --reps 3
    python -m practice_b200 shared ... --tuning block_threads=1024 items_per_thread=1 stages=3

`shared` runs a mixed batch from the four query templates as one shared scan;
`plain` runs one query (a template, or the SSB Q1.1 / Q3.1 shapes) as its own
fused kernel.  Each repetition prints the device time of the scan kernel.
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
    ap.add_argument("mode", choices=["shared", "plain"])
    ap.add_argument("--rows", type=int, default=30_000_000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--query", default="T1", help="T0..T3, q11 or q31 (plain mode)")
    ap.add_argument("--template", type=int, default=-1, help="shared mode: draw every query from this template")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tuning", nargs="*", default=[], help="key=value launch-shape overrides")
    args = ap.parse_args(argv)

    from practice_b200 import queries
    from practice_b200.engine import Database

    kw, shared_default, make_tuning = _tuning(args.tuning)
    cols = {"q11": queries.Q11_COLS, "q31": queries.Q31_COLS}.get(args.query, queries.BATCH_COLS)
    db = Database(0)
    db.generate_ssb(args.rows, args.seed, queries.BATCH_COLS if args.mode == "shared" else cols)
    if args.mode == "shared":
        if args.template >= 0:
            rng = random.Random(args.seed)
            plans = [queries.template(args.template, rng, args.rows) for _ in range(args.batch)]
        else:
            plans = queries.batch(args.batch, args.seed, args.rows)
        t = make_tuning(**{**shared_default, **kw})
        for _ in range(args.reps):
            r = db.execute_shared(plans, t)
            print(f"shared batch of {len(plans)}: scan {r[0].timing.scan_ms:.4f} ms, "
                  f"total {r[0].timing.total_ms:.4f} ms, kernel error {r[0].kernel_error}", flush=True)
        return
    q = args.query
    if q.startswith("T"):
        plan = queries.template(int(q[1:]), random.Random(args.seed), args.rows)
    elif q == "q11":
        plan = queries.ssb_q11(args.rows)
    else:
        plan = queries.ssb_q31(args.rows)
    t = make_tuning(**kw) if kw else None
    for _ in range(args.reps):
        r = db.execute(plan, t)
        print(f"{plan.name}: scan {r.timing.scan_ms:.4f} ms, total {r.timing.total_ms:.4f} ms, "
              f"kernel error {r.kernel_error}", flush=True)


if __name__ == "__main__":
    main()
