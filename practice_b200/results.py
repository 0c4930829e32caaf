"""Host-side result fetch: turns the raw aggregate buffer into typed rows.

Restates what the reference's DatabaseInstance / generated materialisation does
with the buffer the fused kernel leaves behind:

* fast sparse output keeps every group tuple with a non-zero slot
  (CompactSparseAggregateResult, src/db/database_instance.cpp:286-307);
* dense output keeps every group with a validity bit or a non-zero value in its
  visible tuple, and a scalar aggregate always yields one row
  (AggregateDenseCount, src/core/visitor.cpp:2605-2630); a slot whose
  nullable column has its validity bit clear is NULL;
* SUM / COUNT / MIN / MAX slots are 64-bit integers (read as int64), AVG slots
  hold IEEE doubles (bit_cast_double_to_ull, :2545).

Row order is normalised by the ORDER BY keys, then by every column, so results
compare independently of the group-table order.
"""
from __future__ import annotations

import math

import numpy as np

from .plan import Plan, expr_nullable


def _bit(v: np.ndarray, i: int) -> bool:
    return bool((int(v[i >> 6]) >> (i & 63)) & 1)


def output_nullable(plan: Plan) -> list[bool]:
    out = [g.nullable for g in plan.groups]
    for a in plan.aggs:
        out.append(False if a.fn == "count" else expr_nullable(a.arg, plan.nullable))
    return out


def rows(plan: Plan, words: np.ndarray, validity: np.ndarray) -> list[tuple]:
    """Typed result rows of a finished query (AVG finalisation already applied)."""
    vts = plan.visible_ts
    finalized = any(a.fn == "avg" for a in plan.aggs)
    ts = vts if finalized else plan.storage_ts
    groups = plan.group_slots
    w = words.view(np.int64)
    nullable = output_nullable(plan)
    out: list[tuple] = []
    for g in range(groups):
        base = g * ts
        if plan.sparse:
            present = any(int(words[base + c]) != 0 for c in range(ts))
        elif not plan.groups:
            present = True
        else:
            present = any(_bit(validity, base + c) or int(words[base + c]) != 0 for c in range(vts))
        if not present:
            continue
        row = []
        for c in range(vts):
            if not plan.sparse and nullable[c] and not _bit(validity, base + c):
                row.append(None)
                continue
            if c >= len(plan.groups) and plan.aggs[c - len(plan.groups)].fn == "avg":
                row.append(float(words[base + c : base + c + 1].view(np.float64)[0]))
            else:
                row.append(int(w[base + c]))
        out.append(tuple(row))
    return order(plan, out)


def _key(v):
    # NULL sorts first; floats compare by value.
    if v is None:
        return (0, 0)
    if isinstance(v, float) and math.isnan(v):
        return (2, 0)
    return (1, v)


def order(plan: Plan, rs: list[tuple]) -> list[tuple]:
    def k(r):
        keys = []
        for c, desc in plan.order_by:
            kv = _key(r[c])
            keys.append((kv[0], -kv[1]) if desc and kv[0] == 1 else kv)
        return tuple(keys) + tuple(_key(v) for v in r)

    return sorted(rs, key=k)


# ------------------------------------------------------------ device rows

def _expr_type(e) -> int:
    """Result type of a GROUP BY expression (src/core/visitor.cpp:77-107):
    comparisons, logic and IS [NOT] NULL are UInt64, CASE takes its branches'
    widest type, everything else (columns, arithmetic, literals) is Int64."""
    if e.op in ("eq", "ne", "lt", "le", "gt", "ge", "and", "or", "not", "isnull", "notnull", "null"):
        return 1
    if e.op == "case":
        t = {_expr_type(e.kids[1]), _expr_type(e.kids[2])}
        return 2 if 2 in t else 0 if 0 in t else 1
    return 0


def column_types(plan: Plan) -> list[int]:
    """Result column types (src/core/visitor.cpp:109-123): GROUP BY keys by
    their expression, AVG Float64, every other aggregate UInt64."""
    out = [_expr_type(g.expr) for g in plan.groups]
    out += [2 if a.fn == "avg" else 1 for a in plan.aggs]
    return out


def device_rows(plan: Plan, cols: np.ndarray, cvalid: np.ndarray, nrows: int, row_cap: int) -> list[tuple]:
    """Typed rows from cx_finalize's columnar output, in its order."""
    types = column_types(plan)
    vw = (row_cap + 63) // 64
    out = []
    for r in range(nrows):
        row = []
        for c, t in enumerate(types):
            if not ((int(cvalid[c * vw + (r >> 6)]) >> (r & 63)) & 1):
                row.append(None)
            elif t == 2:
                row.append(float(cols[c * row_cap + r : c * row_cap + r + 1].view(np.float64)[0]))
            else:
                row.append(int(cols[c * row_cap + r : c * row_cap + r + 1].view(np.int64)[0]))
        out.append(tuple(row))
    return out
