"""Times the reference's CPU path on a batch of plans (bench.py's CPU-baseline
leg and its `--impl reference` arm).  TEST/BENCH INFRASTRUCTURE ONLY.

Prefers oracle/_ref/libcrystal_ref.so -- the reference's own crystal
primitives (include/crystal/*.h, include/core/inline_math.h) compiled for the
host with OpenMP by `make -C oracle ref` -- and falls back to the oracle
restatement (oracle/crystal_oracle.c, one thread) when that library was not
built.
"""
from __future__ import annotations

import os
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libcrystal_ref.so"


def _dims_rows():
    return {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}


def time_batch(plans, ht, n):
    """Returns (seconds for the whole batch, kind, threads)."""
    if REF_LIB.exists():
        from . import refharness
        return refharness.time_batch(plans, ht, n)
    from . import run_plan
    rows = {"LINEORDER": n, **_dims_rows()}
    t0 = time.perf_counter()
    for p in plans:
        run_plan(p.text(), ht.columns, ht.validity, rows, p.group_slots * p.storage_ts)
    return time.perf_counter() - t0, "port", 1
