"""ctypes driver of oracle/_ref/libcrystal_ref.so (the reference's own crystal
primitives compiled for the host).  TEST/BENCH INFRASTRUCTURE ONLY.

Translates a star-join plan of the supported shape (AND-chains of
`column op literal` filters, PHT_1/PHT_2 joins, GROUP BY over columns, SUM of a
column / product / difference, COUNT(*)) into the harness's query struct.  One
join may expand rows: an OR over two fact keys, or a multi-value hash table
publishing at most one build column.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libcrystal_ref.so"
OPS = {"eq": 0, "ne": 1, "lt": 2, "le": 3, "gt": 4, "ge": 5}


class RefPred(C.Structure):
    _fields_ = [("col", C.c_int), ("op", C.c_int), ("lit", C.c_int)]


class RefJoin(C.Structure):
    _fields_ = [("fk", C.c_int), ("pk", C.c_int), ("payload", C.c_int), ("len", C.c_int), ("keymin", C.c_int),
                ("dim_rows", C.c_int), ("npred", C.c_int), ("preds", RefPred * 8), ("fk2", C.c_int),
                ("multi", C.c_int)]


class RefOperand(C.Structure):
    _fields_ = [("kind", C.c_int), ("idx", C.c_int)]


class RefGroup(C.Structure):
    _fields_ = [("v", RefOperand), ("min", C.c_int), ("card", C.c_int)]


class RefAgg(C.Structure):
    _fields_ = [("fn", C.c_int), ("form", C.c_int), ("a", RefOperand), ("b", RefOperand)]


class RefQuery(C.Structure):
    _fields_ = [("npred", C.c_int), ("preds", RefPred * 8), ("njoin", C.c_int), ("joins", RefJoin * 4),
                ("ngroup", C.c_int), ("groups", RefGroup * 4), ("nagg", C.c_int), ("aggs", RefAgg * 4)]


_lib = None


def available() -> bool:
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = [C.POINTER(RefQuery), C.POINTER(C.c_void_p), C.c_longlong, C.c_void_p, C.c_longlong,
                                C.c_int]
        lib.ref_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def _and_leaves(e):
    if e.op == "and":
        return _and_leaves(e.kids[0]) + _and_leaves(e.kids[1])
    if e.op in OPS and e.kids[0].op == "col" and e.kids[1].op == "int":
        return [(e.kids[0].name, OPS[e.op], e.kids[1].val)]
    raise ValueError(f"predicate shape {e.op} is outside the reference harness")


def translate(plan, dim_rows: dict[str, int]):
    names: list[str] = []

    def idx(c):
        if c not in names:
            names.append(c)
        return names.index(c)

    q = RefQuery()
    payload_of = {}
    fact_preds = []
    joins = []
    for kind, s in plan.steps:
        if kind == "filter":
            fact_preds += _and_leaves(s)
        else:
            joins.append(s)
    if len(fact_preds) > 8 or len(joins) > 4:
        raise ValueError("too many predicates or joins")
    q.npred = len(fact_preds)
    for k, (c, op, lit) in enumerate(fact_preds):
        q.preds[k] = RefPred(idx(c), op, lit)
    q.njoin = len(joins)
    if sum(1 for s in joins if s.expands) > 1:
        raise ValueError("more than one expanding join is outside the reference harness")
    for j, s in enumerate(joins):
        J = q.joins[j]
        J.fk, J.pk = idx(s.fk), idx(s.pk)
        if len(s.more_fks) > 1 or len(s.gathers) > 1:
            raise ValueError("OR-join over more than two keys or MHT with several columns")
        J.fk2 = idx(s.more_fks[0]) if s.more_fks else -1
        J.multi = int(s.multi)
        if s.multi:
            J.payload = idx(s.gathers[0]) if s.gathers else -1
            if s.gathers:
                payload_of[s.gathers[0]] = j
        else:
            J.payload = idx(s.payload) if s.payload else -1
        J.len, J.keymin, J.dim_rows = s.length, s.keymin, dim_rows[s.dim]
        leaves = _and_leaves(s.filter) if s.filter is not None else []
        J.npred = len(leaves)
        for k, (c, op, lit) in enumerate(leaves):
            J.preds[k] = RefPred(idx(c), op, lit)
        if s.payload:
            payload_of[s.payload] = j

    def operand(e):
        if e.op != "col":
            raise ValueError("operand must be a column")
        if e.name in payload_of:
            return RefOperand(1, payload_of[e.name])
        return RefOperand(0, idx(e.name))

    q.ngroup = len(plan.groups)
    for g, gr in enumerate(plan.groups):
        if gr.nullable:
            raise ValueError("nullable group keys are outside the reference harness")
        q.groups[g] = RefGroup(operand(gr.expr), gr.min, gr.card)
    q.nagg = len(plan.aggs)
    for a, ag in enumerate(plan.aggs):
        A = q.aggs[a]
        if ag.fn == "count" and ag.arg.op == "star":
            A.fn = 0
        elif ag.fn == "sum":
            A.fn = 1
            e = ag.arg
            if e.op == "col":
                A.form, A.a = 0, operand(e)
            elif e.op in ("mul", "sub"):
                A.form = 1 if e.op == "mul" else 2
                A.a, A.b = operand(e.kids[0]), operand(e.kids[1])
            else:
                raise ValueError("aggregate shape outside the reference harness")
        else:
            raise ValueError("aggregate outside the reference harness")
    return q, names


def max_threads() -> int:
    return _load().ref_max_threads()


def run(plan, columns: dict[str, np.ndarray], dim_rows: dict[str, int], n_fact: int, threads: int = 0) -> np.ndarray:
    lib = _load()
    q, names = translate(plan, dim_rows)
    arrs = [np.ascontiguousarray(columns[c], dtype=np.int32) for c in names]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    words = plan.group_slots * plan.storage_ts
    out = np.zeros(max(words, 1), dtype=np.uint64)
    rc = lib.ref_run(C.byref(q), ptrs, n_fact, out.ctypes.data, len(out), threads)
    if rc:
        raise RuntimeError("ref_run failed")
    return out[:words]


def time_batch(plans, ht, n):
    """Times the batch with all host threads; returns (seconds, kind, threads)."""
    lib = _load()
    threads = os.cpu_count() or 1
    dims = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}
    prepared = []
    for p in plans:
        q, names = translate(p, dims)
        arrs = [np.ascontiguousarray(ht.columns[c], dtype=np.int32) for c in names]
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        out = np.zeros(max(p.group_slots * p.storage_ts, 1), dtype=np.uint64)
        prepared.append((q, ptrs, arrs, out))
    t0 = time.perf_counter()
    for q, ptrs, _arrs, out in prepared:
        lib.ref_run(C.byref(q), ptrs, n, out.ctypes.data, len(out), threads)
    return time.perf_counter() - t0, "reference", lib.ref_max_threads()
