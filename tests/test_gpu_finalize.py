"""GPU tests of result finalisation on the device (cx_finalize) against a
plain-Python restatement of the reference's generated post-processing:
AggregateDenseCount / AggregateDenseWrite (src/core/visitor.cpp:2589-2697)
and the ORDER BY / LIMIT comparator (src/core/visitor.cpp:307-358): keys in
order, a valid value before NULL, values compared in the column's result type
(group keys Int64, COUNT / SUM UInt64, AVG Float64), ties by row index."""
import functools
import random
import struct

import numpy as np
import pytest

from practice_b200 import datagen, queries, results
from practice_b200.plan import Group, PlanBuilder, col, star

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def db():
    from practice_b200.engine import Database
    return Database(0)


def load(db, seed, n, cols, nulls=None):
    ht = datagen.host_tables(seed, n, cols, nulls)
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, cols))
    return ht


def run(db, plan):
    m = db.compile(plan)
    res, val = db.alloc_result(m)
    for t, n in db.rows.items():
        db.ctx.set_rows(t, n)
    db.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
    db.ctx.execute(m, db.torch.cuda.current_stream().cuda_stream)
    db.ctx.sync()
    return res, val


def bit(v, i):
    return (int(v[i >> 6]) >> (i & 63)) & 1


def reference_rows(plan, words, validity, limit=None):
    types = results.column_types(plan)
    vts = plan.visible_ts
    ts = vts if any(a.fn == "avg" for a in plan.aggs) else plan.storage_ts
    nullable = [False] * vts if plan.sparse else results.output_nullable(plan)
    rows = []  # (values, valid) per present group, in group order
    for g in range(1 if not plan.groups else plan.group_slots):
        base = g * ts
        if not plan.groups:
            present = True
        elif plan.sparse:
            present = any(int(words[base + c]) for c in range(ts))
        else:
            present = any(bit(validity, base + c) or int(words[base + c]) for c in range(vts))
        if present:
            rows.append(([int(words[base + c]) for c in range(vts)],
                         [plan.sparse or not nullable[c] or bool(bit(validity, base + c)) for c in range(vts)]))

    def val(c, x):
        if types[c] == 0:
            return x - (1 << 64) if x >= 1 << 63 else x
        if types[c] == 2:
            return struct.unpack("<d", struct.pack("<Q", x))[0]
        return x

    def cmp(li, ri):  # -1: left first
        (lv, lval), (rv, rval) = rows[li], rows[ri]
        for c, desc in plan.order_by:
            if nullable[c] and lval[c] != rval[c]:
                return -1 if lval[c] else 1
            if nullable[c] and not lval[c]:
                continue
            a, b = val(c, lv[c]), val(c, rv[c])
            if b < a:
                return 1 if not desc else -1
            if a < b:
                return -1 if not desc else 1
        return -1 if li < ri else (1 if li > ri else 0)

    order = list(range(len(rows)))
    if plan.order_by:
        order.sort(key=functools.cmp_to_key(cmp))
    if limit is not None:
        order = order[:limit]
    out = []
    for i in order:
        v, ok = rows[i]
        out.append(tuple(None if not ok[c] else val(c, v[c]) if types[c] != 1 else
                         (v[c] - (1 << 64) if v[c] >= 1 << 63 else v[c]) for c in range(vts)))
    return out


def check(db, plan, limit=None):
    res, val = run(db, plan)
    words = res.cpu().numpy().view(np.uint64)
    valid = val.cpu().numpy().view(np.uint64)
    got = db.finalize_rows(plan, res, val, limit)
    ref = reference_rows(plan, words, valid, limit)
    assert got == ref
    return got


def test_q31_dense_and_ordered(db):
    n = 1_000_003
    load(db, 61, n, queries.Q31_COLS)
    got = check(db, queries.ssb_q31(n))  # ORDER BY d_year ASC, revenue DESC
    assert len(got) > 100
    check(db, queries.ssb_q31(n), limit=10)


def test_nullable_groups_order_valid_before_null(db):
    n = 800_011
    load(db, 62, n, queries.Q31_COLS, nulls={"lo_revenue": 100, "c_city": 50})
    got = check(db, queries.ssb_q31_nullable(n))
    assert any(r[0] is None for r in got)
    check(db, queries.ssb_q31_nullable(n), limit=7)


@pytest.mark.parametrize("t", [0, 1, 2, 3])
def test_templates_with_order_and_limit(db, t):
    n = 2_000_017
    load(db, 63, n, queries.BATCH_COLS)
    rng = random.Random(90 + t)
    p = queries.template(t, rng, n)
    if p.groups:
        p.order_by = [(len(p.groups), True), (0, False)]  # by the aggregate, then the first key
    check(db, p)
    check(db, p, limit=5)


def test_large_result_uses_the_global_network(db):
    """More than 2048 rows: the bitonic network runs in global memory."""
    n = 2_000_029
    load(db, 65, n, queries.BATCH_COLS)
    b = PlanBuilder(datagen.ssb_tables(n, queries.BATCH_COLS), "LINEORDER", name="big")
    b.join("DDATE", "lo_orderdate")
    p = b.aggregate([Group(col("lo_quantity"), 1, 50, False), Group(col("lo_discount"), 0, 11, False),
                     queries._g("d_year")], [("sum", col("lo_revenue")), ("count", star())],
                    order_by=[(4, False), (3, True)])
    got = check(db, p)
    assert len(got) > 2048
    check(db, p, limit=100)


def test_kat_and_scalar_results(db):
    from practice_b200 import queries as q
    n = 300_001
    load(db, 64, n, queries.BATCH_COLS)
    tables = datagen.ssb_tables(n, queries.BATCH_COLS)
    b = PlanBuilder(tables, "LINEORDER", name="cnt")
    b.filter(col("lo_quantity").lt(10))
    scalar = b.aggregate([], [("count", star()), ("sum", col("lo_revenue"))])
    check(db, scalar)
    b = PlanBuilder(tables, "LINEORDER", name="avg")
    b.join("DDATE", "lo_orderdate")
    avg = b.aggregate([q._g("d_year")], [("avg", col("lo_revenue")), ("count", star())], order_by=[(1, True)])
    check(db, avg)
    b = PlanBuilder(tables, "LINEORDER", name="grp")
    grp = b.aggregate([Group(col("lo_discount"), 0, 11, False)], [("sum", col("lo_quantity"))], order_by=[(1, False)])
    check(db, grp, limit=3)
