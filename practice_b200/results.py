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
