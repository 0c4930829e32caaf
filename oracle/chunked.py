"""Chunked CPU checkers for fact tables too large to evaluate in one piece --
TEST/BENCH INFRASTRUCTURE ONLY (tests/, the smoke check and bench.py's
CPU-baseline leg; the product never imports it).

A query's aggregate buffer over a fact table equals the combination of the
buffers over disjoint row ranges of that table, slot by slot, because every
update the reference makes to a slot commutes:

* GROUP BY key slots hold the group's canonical key (the same value in every
  range that touches the group, 0 where none does);
* COUNT and SUM slots are 64-bit modular sums (db::atomic_add_ull,
  include/core/inline_math.h; src/core/visitor.cpp:3017-3195);
* MIN / MAX slots are unsigned 64-bit minima / maxima, MIN starting at ~0
  (src/core/visitor.cpp:2987-3016);
* validity bits OR.

AVG is finalised into doubles and cannot be recombined, so plans with AVG are
refused.  Rows are fetched range by range (from the device-resident table the
GPU used, or from the seeded host generator) and evaluated either by the C
restatement (oracle/crystal_oracle.c, several ranges at once on a thread
pool: ctypes releases the GIL during the call) or by the reference's own
primitives (oracle/_ref, OpenMP inside each call).
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Callable

import numpy as np

from . import run_plan

KEY, ADD, MIN, MAX = 0, 1, 2, 3

# fetch(row0, rows) -> (fact columns, fact validity words); row0 is a multiple of 64.
Fetch = Callable[[int, int], tuple[dict, dict]]


def slot_kinds(plan) -> np.ndarray:
    """How each slot of the storage tuple combines across row ranges."""
    if any(a.fn == "avg" for a in plan.aggs):
        raise ValueError("AVG results are finalised per run and cannot be combined across row ranges")
    kinds = [KEY] * len(plan.groups)
    kinds += [{"count": ADD, "sum": ADD, "min": MIN, "max": MAX}[a.fn] for a in plan.aggs]
    kinds = kinds or [ADD]
    return np.array(kinds, dtype=np.int8)


class Accumulator:
    """Combined result words and validity words of one plan."""

    def __init__(self, plan):
        self.plan = plan
        self.ts = plan.storage_ts
        self.words_n = plan.group_slots * self.ts
        kinds = np.tile(slot_kinds(plan), plan.group_slots)
        self.key = kinds == KEY
        self.add = kinds == ADD
        self.min = kinds == MIN
        self.max = kinds == MAX
        self.words = np.zeros(self.words_n, dtype=np.uint64)
        self.words[self.min] = np.uint64(0xFFFFFFFFFFFFFFFF)
        self.validity = np.zeros((self.words_n + 63) // 64, dtype=np.uint64)
        self.seconds = 0.0  # evaluation time spent on this plan (reference runs)

    def add_part(self, words: np.ndarray, validity: np.ndarray | None) -> None:
        w = np.asarray(words[: self.words_n], dtype=np.uint64)
        acc = self.words
        acc[self.key] = np.where(acc[self.key] == 0, w[self.key], acc[self.key])
        with np.errstate(over="ignore"):
            acc[self.add] = acc[self.add] + w[self.add]
        acc[self.min] = np.minimum(acc[self.min], w[self.min])
        acc[self.max] = np.maximum(acc[self.max], w[self.max])
        if validity is not None and len(self.validity):
            self.validity |= np.asarray(validity[: len(self.validity)], dtype=np.uint64)


def _ranges(row0: int, rows: int, parts: int) -> list[tuple[int, int]]:
    """Splits [row0, row0 + rows) into up to `parts` ranges starting on 64-row boundaries."""
    step = max(64, ((rows + parts - 1) // parts + 63) // 64 * 64)
    return [(r, min(step, row0 + rows - r)) for r in range(row0, row0 + rows, step)]


def _slice_validity(words: np.ndarray, off: int, rows: int) -> np.ndarray:
    return words[off // 64: (off + rows + 63) // 64]


def run_oracle(plans, fetch: Fetch, fact_rows: int, dims: dict, dim_validity: dict, dim_rows: dict,
               chunk_rows: int = 20_000_000, threads: int | None = None):
    """The C restatement over the whole fact table, range by range, with
    `threads` ranges (or plans) in flight.  Returns (accumulators, seconds of
    evaluation, threads)."""
    threads = threads or os.cpu_count() or 1
    accs = [Accumulator(p) for p in plans]
    spent = 0.0
    chunk_rows = max(64, chunk_rows // 64 * 64)
    with ThreadPoolExecutor(max_workers=threads) as pool:
        for c0 in range(0, fact_rows, chunk_rows):
            n = min(chunk_rows, fact_rows - c0)
            cols, valid = fetch(c0, n)
            parts = _ranges(0, n, max(1, threads // max(1, len(plans))))
            jobs = []
            t0 = time.perf_counter()
            for i, p in enumerate(plans):
                for off, m in parts:
                    columns = {**dims, **{c: v[off: off + m] for c, v in cols.items()}}
                    validity = {**dim_validity, **{c: _slice_validity(v, off, m) for c, v in valid.items()}}
                    rows = {"LINEORDER": m, **dim_rows}
                    jobs.append((i, pool.submit(run_plan, p.text(), columns, validity, rows,
                                                p.group_slots * p.storage_ts)))
            for i, f in jobs:
                r = f.result()
                accs[i].add_part(r.words, r.validity)
            spent += time.perf_counter() - t0
    return accs, spent, threads


def run_reference(plans, fetch: Fetch, fact_rows: int, dims: dict, dim_rows: dict, chunk_rows: int = 20_000_000):
    """The reference's own primitives (oracle/_ref, OpenMP over all host
    threads) over the whole fact table, range by range.  Result words only:
    the harness's plans carry no nullable columns.  Returns (accumulators,
    seconds inside the reference calls, threads)."""
    from . import refharness

    accs = [Accumulator(p) for p in plans]
    spent = 0.0
    chunk_rows = max(64, chunk_rows // 64 * 64)
    for c0 in range(0, fact_rows, chunk_rows):
        n = min(chunk_rows, fact_rows - c0)
        cols, _ = fetch(c0, n)
        columns = {**dims, **cols}
        for i, p in enumerate(plans):
            t0 = time.perf_counter()
            w = refharness.run(p, columns, dim_rows, n)
            dt = time.perf_counter() - t0
            spent += dt
            accs[i].seconds += dt
            accs[i].add_part(w, None)
    return accs, spent, refharness.max_threads()


def host_fetch(seed: int, fact_cols, nulls: dict[str, int] | None = None) -> Fetch:
    """Row ranges from the seeded host generator (practice_b200/datagen.py)."""
    from practice_b200 import datagen

    def fetch(row0: int, rows: int):
        cols = {c: datagen.fact_column(c, seed, row0, rows) for c in fact_cols}
        valid = {c: datagen.validity_words(seed, datagen.STREAMS["valid_" + c], rows, pm, row0=row0)
                 for c, pm in (nulls or {}).items() if c.startswith("lo_")}
        return cols, valid

    return fetch


def device_fetch(db, fact_cols) -> Fetch:
    """Row ranges copied back from the device-resident fact table of an engine
    Database (the exact bytes the GPU scanned)."""

    def fetch(row0: int, rows: int):
        cols = {c: db.cols[c][row0: row0 + rows].cpu().numpy() for c in fact_cols}
        valid = {c: db.valid[c][row0 // 64: (row0 + rows + 63) // 64].cpu().numpy().view(np.uint64)
                 for c in db.valid if c in fact_cols}
        return cols, valid

    return fetch


def device_dims(db, dim_tables=("DDATE", "CUSTOMER", "SUPPLIER", "PART")):
    """Dimension columns, their validity words and row counts from a Database."""
    from practice_b200 import datagen

    dims, dval, rows = {}, {}, {}
    for t in dim_tables:
        if t not in db.tables:
            continue
        for c in db.tables[t].cols:
            if c in db.cols:
                dims[c] = db.cols[c].cpu().numpy()
            if c in db.valid:
                dval[c] = db.valid[c].cpu().numpy().view(np.uint64)
        rows[t] = db.rows.get(t, datagen.DIM_ROWS[t])
    return dims, dval, rows
