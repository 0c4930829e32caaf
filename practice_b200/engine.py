"""Host facade over libcrystal_b200.so: resident tables, compiled-query cache,
query execution and result fetch.

This plays the role of the reference's DatabaseInstance + QueryEngine for the
hot path (src/db/database_instance.cpp:138-439, src/core/execution.cpp:652-725):
columns are loaded once and stay resident in HBM, each plan is generated,
compiled (cached by plan text and tuning) and executed through the C ABI, and
results come back as typed rows.  PyTorch only provides device memory and
streams; every kernel comes from the library.
"""
from __future__ import annotations

import itertools
import json
import os
import re
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib, datagen
from .plan import Plan, Table
from .results import rows as result_rows


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("crystal-b200 needs a CUDA device (no CPU fallback exists)")
    return torch


class SharedProgram:
    """A compiled shared-scan program for a set of plan shapes."""

    def __init__(self, module: _lib.Module, shape_keys: list[str], nlits: list[int]):
        self.module = module
        self.shape_keys = shape_keys
        self.nlits = nlits
        self.index = {k: i for i, k in enumerate(shape_keys)}


@dataclass
class QueryResult:
    words: np.ndarray      # u64 result words (final layout)
    validity: np.ndarray   # u64 validity words
    timing: _lib.Timing
    kernel_error: int

    def rows(self, plan: Plan) -> list[tuple]:
        return result_rows(plan, self.words, self.validity)


def shape_key(plan: Plan) -> str:
    """A plan's shape: its text with every integer literal abstracted.  Queries
    of one shape share a launch configuration."""
    return plan.memo("shape", lambda: re.sub(r"\(int -?\d+\)", "(int ?)", plan.text()))


DEFAULT_CANDIDATES = [
    dict(block_threads=bt, items_per_thread=ipt, stages=st, ctas_per_sm=cs)
    for bt, ipt, st, cs in itertools.product((256, 512, 1024), (2, 4, 8), (0, 2, 4), (1, 16))
]


# Shared-scan launch shape before autotuning: one 32-warp CTA per SM, 1024-row
# tiles, a three-stage ring.
SHARED_DEFAULT = dict(block_threads=1024, items_per_thread=1, stages=3, ctas_per_sm=1)


def make_tuning(**kw) -> _lib.Tuning:
    t = _lib.default_tuning()
    for k, v in kw.items():
        setattr(t, k, v)
    return t


def tuning_dict(t: _lib.Tuning) -> dict:
    return {f: getattr(t, f) for f, _ in _lib.Tuning._fields_}


class Database:
    """Resident star-schema tables on one GPU."""

    def __init__(self, device: int = 0):
        torch = _torch()
        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.cols: dict[str, object] = {}      # name -> int32 tensor
        self.valid: dict[str, object] = {}     # name -> int64 tensor of validity words
        self.rows: dict[str, int] = {}         # table -> rows
        self.tables: dict[str, Table] = {}
        self._modules: dict[tuple, _lib.Module] = {}
        self.ctx = _lib.ExecCtx()
        self._bound: set[str] = set()
        self.tuned: dict[str, dict] = {}
        self.tuning_cache = Path(os.environ.get("CRYSTAL_B200_TUNING", Path.home() / ".cache" / "crystal_b200" / "tuning.json"))
        if self.tuning_cache.exists():
            try:
                self.tuned = json.loads(self.tuning_cache.read_text())
            except (OSError, ValueError):
                self.tuned = {}

    def reset(self) -> None:
        """Drops every resident table and starts a fresh execution context."""
        self.ctx.close()
        self.ctx = _lib.ExecCtx()
        self.cols.clear()
        self.valid.clear()
        self.rows.clear()
        self.tables.clear()
        self.__dict__.pop("_colmin", None)

    # ------------------------------------------------------------ loading
    def load_column(self, table: str, name: str, data) -> None:
        torch = self.torch
        if isinstance(data, np.ndarray):
            t = torch.from_numpy(np.ascontiguousarray(data, dtype=np.int32)).to(self.device)
        else:
            t = data
        self.cols[name] = t
        self.rows[table] = int(t.numel()) if table not in self.rows else self.rows[table]
        self.ctx.set_buffer("d_" + name, t.data_ptr(), t.numel())
        self._register_range(name, t)

    def _register_range(self, name: str, t) -> None:
        """Records the column's value range: the shared scan's filter tables
        start at the minimum, and shared joins need non-zero foreign keys."""
        cache = self.__dict__.setdefault("_colmin", {})
        if t.numel() == 0:
            cache[name] = 1
            return
        lo, hi = (int(v) for v in self.torch.aminmax(t))
        cache[name] = lo
        self.ctx.set_column_range("d_" + name, lo, hi)

    def load_validity(self, name: str, words) -> None:
        torch = self.torch
        if isinstance(words, np.ndarray):
            t = torch.from_numpy(np.ascontiguousarray(words).view(np.int64)).to(self.device)
        else:
            t = words
        self.valid[name] = t
        self.ctx.set_null_bitmap("d_" + name, t.data_ptr(), t.numel())

    def set_rows(self, table: str, rows: int) -> None:
        self.rows[table] = rows
        self.ctx.set_rows(table, rows)

    def load_host_tables(self, ht: datagen.HostTables, tables: dict[str, Table]) -> None:
        for tname, t in tables.items():
            present = [c for c in t.cols if c in ht.columns]
            if not present:
                continue
            for c in present:
                self.load_column(tname, c, ht.columns[c])
            self.set_rows(tname, len(ht.columns[present[0]]))
            self.tables[tname] = t
        for c, w in ht.validity.items():
            self.load_validity(c, w)

    def generate_ssb(self, fact_rows: int, seed: int, fact_cols: list[str], nulls: dict[str, int] | None = None,
                     dims: tuple[str, ...] = ("DDATE", "CUSTOMER", "SUPPLIER", "PART")) -> None:
        """Generates the fact table on the device and the dimensions on the host."""
        torch = self.torch
        tables = datagen.ssb_tables(fact_rows, fact_cols)
        for c in fact_cols:
            if c == "lo_commitdate":  # derived from the order date on the host
                self.load_column("LINEORDER", c, datagen.fact_column(c, seed, 0, fact_rows))
                continue
            t = torch.empty(fact_rows, dtype=torch.int32, device=self.device)
            datagen.fact_column_device(c, seed, fact_rows, t.data_ptr(), torch.cuda.current_stream().cuda_stream)
            self.load_column("LINEORDER", c, t)
        self.set_rows("LINEORDER", fact_rows)
        self.tables["LINEORDER"] = tables["LINEORDER"]
        for d in dims:
            for c, v in datagen.dim_columns(d, seed).items():
                self.load_column(d, c, v)
            self.set_rows(d, datagen.DIM_ROWS[d])
            self.tables[d] = tables[d]
        for c, permille in (nulls or {}).items():
            rows = fact_rows if c.startswith("lo_") else datagen.DIM_ROWS[datagen.dim_of_column(c)]
            w = torch.empty((rows + 63) // 64, dtype=torch.int64, device=self.device)
            datagen.validity_device(c, seed, rows, permille, w.data_ptr(), torch.cuda.current_stream().cuda_stream)
            self.load_validity(c, w)
        torch.cuda.synchronize()

    # ----------------------------------------------------------- queries
    def compile(self, plan: Plan, tuning: _lib.Tuning | None = None) -> _lib.Module:
        """The plan's fused kernel.  With `tuning.parametric` set, one module
        serves every plan of the same shape (literals are passed at execute)."""
        tkey = tuple(getattr(tuning, f) for f, _ in _lib.Tuning._fields_) if tuning is not None else None
        key = (shape_key(plan) if tuning is not None and tuning.parametric else plan.text(), tkey)
        m = self._modules.get(key)
        if m is None:
            src = _lib.codegen(plan.text(), tuning)
            m = _lib.Module(src, key=f"{plan.name}_{abs(hash(key))}")
            self._modules[key] = m
        return m

    def tuning_for(self, plan: Plan) -> _lib.Tuning | None:
        """The autotuned launch shape of the plan's shape, if one was tuned."""
        best = self.tuned.get(shape_key(plan))
        return make_tuning(**best["tuning"]) if best else None

    def autotune(self, plan: Plan, candidates: list[dict] | None = None, reps: int = 3, persist: bool = True) -> dict:
        """Times every feasible candidate launch shape on the resident tables
        (CUDA events around the fused scan) and keeps the fastest for the
        plan's shape.  Infeasible shapes (shared memory, registers) are skipped."""
        key = shape_key(plan)
        table = []
        res = val = None
        for cand in candidates or DEFAULT_CANDIDATES:
            t = make_tuning(**cand)
            try:
                m = self.compile(plan, t)
            except _lib.CxError:
                continue
            if res is None or res.numel() < m.info.result_words or val.numel() < m.info.validity_words:
                res, val = self.alloc_result(m)
            for tn, n in self.rows.items():
                self.ctx.set_rows(tn, n)
            self.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
            times = []
            try:
                for _ in range(reps + 1):
                    self.ctx.execute(m, self.torch.cuda.current_stream().cuda_stream)
                    self.ctx.sync()
                    times.append(self.ctx.timing().scan_ms)
            except _lib.CxError:
                continue
            table.append((min(times[1:]), cand))
        if not table:
            raise RuntimeError("autotune: no feasible launch shape")
        table.sort(key=lambda x: x[0])
        best = {"tuning": tuning_dict(make_tuning(**table[0][1])), "scan_ms": table[0][0],
                "tried": len(table)}
        self.tuned[key] = best
        if persist:
            try:
                self.tuning_cache.parent.mkdir(parents=True, exist_ok=True)
                self.tuning_cache.write_text(json.dumps(self.tuned, indent=1))
            except OSError:
                pass
        best["table"] = table
        return best

    # ------------------------------------------------------ shared scans
    def column_min(self, name: str) -> int:
        cache = self.__dict__.setdefault("_colmin", {})
        if name not in cache:
            self._register_range(name, self.cols[name])
        return cache[name]

    def shareable(self, plan: Plan) -> bool:
        """A plan can join a shared scan when its shape compiles into one and
        every foreign key it probes is non-zero (the empty-slot sentinel)."""
        try:
            _lib.shared_codegen([plan.text()])
        except _lib.CxError:
            return False
        for kind, s in plan.steps:
            if kind == "join" and (s.expands or self.column_min(s.fk) <= 0):
                return False
        return True

    def shared_program(self, plans: list[Plan], tuning: _lib.Tuning | None = None) -> SharedProgram:
        keys: list[str] = []
        reps: list[Plan] = []
        for p in plans:
            k = shape_key(p)
            if k not in keys:
                keys.append(k)
                reps.append(p)
        order = sorted(range(len(keys)), key=lambda i: keys[i])
        keys = [keys[i] for i in order]
        reps = [reps[i] for i in order]
        tkey = tuple(getattr(tuning, f) for f, _ in _lib.Tuning._fields_) if tuning is not None else None
        ck = ("shared", tuple(keys), tkey)
        prog = self._modules.get(ck)
        if prog is None:
            src = _lib.shared_codegen([r.text() for r in reps], tuning)
            mod = _lib.Module(src, key=f"shared_{abs(hash(ck))}")
            prog = SharedProgram(mod, keys, [len(_lib.plan_literals(r.text())) for r in reps])
            self._modules[ck] = prog
        return prog

    def shared_prepare(self, prog: SharedProgram, plans: list[Plan]):
        """Per-query result buffers, descriptors and the parameter array."""
        queries, params, bufs, _ = self.shared_prepare_arena(prog, plans)
        return queries, params, bufs

    def shared_prepare_arena(self, prog: SharedProgram, plans: list[Plan]):
        """As shared_prepare, with every query's result and validity words
        placed in one device arena (16-byte aligned views), so that a batch's
        results come back to the host in one copy; returns the arena too."""
        torch = self.torch
        lay, off = [], 0
        for p in plans:
            words = p.group_slots * p.storage_ts
            rw, vw = max(words, 1), max((words + 63) // 64, 1)
            lay.append((words, off, rw, off + (rw + 1) // 2 * 2, vw))
            off += (rw + 1) // 2 * 2 + (vw + 1) // 2 * 2
        arena = torch.empty(max(off, 2), dtype=torch.int64, device=self.device)
        queries, params, bufs = [], [], []
        for p, (words, ro, rw, vo, vw) in zip(plans, lay):
            s = prog.index[shape_key(p)]
            res, val = arena[ro:ro + rw], arena[vo:vo + vw]
            lits = _lib.plan_literals(p.text())
            queries.append(_lib.SharedQuery(s, len(params), res.data_ptr(), res.numel(), val.data_ptr(), val.numel()))
            params.extend(lits)
            bufs.append((res, val, words))
        return queries, params, bufs, arena

    def execute_shared(self, plans: list[Plan], tuning: _lib.Tuning | None = None,
                       stream=None) -> list[QueryResult]:
        torch = self.torch
        if tuning is None:
            tuning = self.shared_tuning_for(plans) or make_tuning(**SHARED_DEFAULT)
        prog = self.shared_program(plans, tuning)
        queries, params, bufs, arena = self.shared_prepare_arena(prog, plans)
        for t, n in self.rows.items():
            self.ctx.set_rows(t, n)
        s = stream if stream is not None else torch.cuda.current_stream()
        self.ctx.shared_execute(prog.module, queries, params, s.cuda_stream)
        err = 0
        try:
            self.ctx.sync()
        except _lib.CxError as e:
            if e.code != -6:
                raise
            err = self.ctx.kernel_error()
        timing = self.ctx.timing()
        host = arena.cpu().numpy().view(np.uint64)
        base = arena.data_ptr()
        out = []
        for res, val, words in bufs:
            ro, vo = (res.data_ptr() - base) // 8, (val.data_ptr() - base) // 8
            w = host[ro:ro + words].copy()
            v = host[vo:vo + (words + 63) // 64].copy()
            out.append(QueryResult(w, v, timing, err))
        return out

    def autotune_shared(self, plans: list[Plan], candidates: list[dict], reps: int = 2) -> dict:
        """Times each candidate launch shape of the shared program for the
        plans' shape set and caches the fastest (keyed by the sorted shapes)."""
        key = "shared|" + "|".join(sorted({shape_key(p) for p in plans}))
        table = []
        for cand in candidates:
            t = make_tuning(**cand)
            try:
                prog = self.shared_program(plans, t)
            except _lib.CxError:
                continue
            queries, params, bufs = self.shared_prepare(prog, plans)
            for tn, n in self.rows.items():
                self.ctx.set_rows(tn, n)
            times = []
            try:
                for _ in range(reps + 1):
                    self.ctx.shared_execute(prog.module, queries, params, self.torch.cuda.current_stream().cuda_stream)
                    self.ctx.sync()
                    times.append(self.ctx.timing().scan_ms)
            except _lib.CxError:
                continue
            table.append((min(times[1:]), cand))
        if not table:
            raise RuntimeError("autotune_shared: no feasible launch shape")
        table.sort(key=lambda x: x[0])
        best = {"tuning": tuning_dict(make_tuning(**table[0][1])), "scan_ms": table[0][0], "tried": len(table)}
        self.tuned[key] = best
        best["table"] = table
        return best

    def shared_tuning_for(self, plans: list[Plan]) -> _lib.Tuning | None:
        best = self.tuned.get("shared|" + "|".join(sorted({shape_key(p) for p in plans})))
        return make_tuning(**best["tuning"]) if best else None

    def finalize_rows(self, plan: Plan, res, val, limit: int | None = None) -> list[tuple]:
        """The plan's result rows, finalised and ordered on the device
        (cx_finalize) from its aggregate buffer (`res`, `val`: device tensors
        left by execute), then copied to the host."""
        from . import results

        torch = self.torch
        finalized = any(a.fn == "avg" for a in plan.aggs)
        ts = plan.visible_ts if finalized else plan.storage_ts
        groups = plan.group_slots
        ncols = plan.visible_ts
        cap = max(groups, 1)
        cols = torch.empty(ncols * cap, dtype=torch.int64, device=self.device)
        cval = torch.empty(ncols * ((cap + 63) // 64), dtype=torch.int64, device=self.device)
        nullable = results.output_nullable(plan) if not plan.sparse else [False] * ncols
        n = _lib.finalize(res.data_ptr(), val.data_ptr(), groups, ts, results.column_types(plan), nullable,
                          plan.sparse, not plan.groups, list(plan.order_by), limit, cols.data_ptr(), cval.data_ptr(),
                          cap, torch.cuda.current_stream().cuda_stream)
        return results.device_rows(plan, cols.cpu().numpy().view(np.uint64), cval.cpu().numpy().view(np.uint64), n, cap)

    def alloc_result(self, module: _lib.Module):
        torch = self.torch
        res = torch.empty(max(int(module.info.result_words), 1), dtype=torch.int64, device=self.device)
        val = torch.empty(max(int(module.info.validity_words), 1), dtype=torch.int64, device=self.device)
        return res, val

    def execute(self, plan: Plan, tuning: _lib.Tuning | None = None, stream=None) -> QueryResult:
        torch = self.torch
        tuning = tuning if tuning is not None else self.tuning_for(plan)
        m = self.compile(plan, tuning)
        res, val = self.alloc_result(m)
        for t, n in self.rows.items():
            self.ctx.set_rows(t, n)
        self.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
        s = stream if stream is not None else torch.cuda.current_stream()
        params = _lib.plan_literals(plan.text()) if tuning is not None and tuning.parametric else None
        self.ctx.execute(m, s.cuda_stream, params)
        err = 0
        try:
            self.ctx.sync()
        except _lib.CxError as e:
            if e.code != -6:
                raise
            err = self.ctx.kernel_error()
        fw = int(m.info.final_words)
        words = res.cpu().numpy().view(np.uint64)[:fw].copy()
        validity = val.cpu().numpy().view(np.uint64)[: (fw + 63) // 64].copy()
        return QueryResult(words, validity, self.ctx.timing(), err)
