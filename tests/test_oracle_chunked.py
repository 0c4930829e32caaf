"""The chunked checkers: a result combined from row ranges equals the result of
one run over the whole table, bit for bit, for every slot kind (keys, SUM,
COUNT, MIN, MAX, validity), with nullable fact and payload columns, and with
the reference's own primitives as the evaluator."""
import random

import numpy as np
import pytest

import oracle
from oracle import chunked, refharness
from practice_b200 import datagen, queries
from practice_b200.plan import Group, PlanBuilder, col, star

DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}
N = 300_001


def _whole(plan, ht):
    rows = {"LINEORDER": ht.fact_rows, **DIM_ROWS}
    return oracle.run_plan(plan.text(), ht.columns, ht.validity, rows, plan.group_slots * plan.storage_ts)


def _min_max_plan(n):
    t = datagen.ssb_tables(n, queries.BATCH_COLS)
    b = PlanBuilder(t, "LINEORDER", nullable={"lo_revenue"}, name="minmax")
    b.join("DDATE", "lo_orderdate")
    return b.aggregate([Group(col("d_year"), 1992, 7)], [("min", col("lo_revenue")), ("max", col("lo_revenue")),
                                                         ("count", col("lo_revenue")), ("count", star())])


@pytest.fixture(scope="module")
def tables():
    nulls = {"lo_revenue": 100, "c_city": 50}
    cols = sorted(set(queries.Q31_COLS) | set(queries.Q11_COLS) | set(queries.BATCH_COLS))
    return datagen.host_tables(5, N, cols, nulls), cols, nulls


def test_chunked_oracle_equals_one_run(tables):
    ht, cols, nulls = tables
    rng = random.Random(9)
    plans = [queries.ssb_q11(N), queries.ssb_q31(N), queries.ssb_q31_nullable(N), _min_max_plan(N)]
    plans += [queries.template(t, rng, N) for t in range(4)]
    dims = {c: v for c, v in ht.columns.items() if not c.startswith("lo_")}
    dval = {c: v for c, v in ht.validity.items() if not c.startswith("lo_")}
    fetch = chunked.host_fetch(5, cols, nulls)
    accs, spent, threads = chunked.run_oracle(plans, fetch, N, dims, dval, DIM_ROWS, chunk_rows=70_000, threads=4)
    assert spent > 0 and threads == 4
    for p, acc in zip(plans, accs):
        ref = _whole(p, ht)
        np.testing.assert_array_equal(acc.words, ref.words, err_msg=p.name)
        np.testing.assert_array_equal(acc.validity, ref.validity, err_msg=p.name)


def test_chunked_reference_equals_one_run(tables):
    if not refharness.available():
        pytest.skip("oracle/_ref not built (the reference sources are not mounted)")
    ht, cols, _ = tables
    rng = random.Random(10)
    plans = [queries.ssb_q11(N), queries.ssb_q31(N)] + [queries.template(t, rng, N) for t in range(4)]
    dims = {c: v for c, v in ht.columns.items() if not c.startswith("lo_")}
    accs, spent, threads = chunked.run_reference(plans, chunked.host_fetch(5, cols), N, dims, DIM_ROWS,
                                                 chunk_rows=100_000)
    assert threads >= 1
    for p, acc in zip(plans, accs):
        np.testing.assert_array_equal(acc.words, _whole(p, ht).words, err_msg=p.name)


def test_avg_plans_are_refused():
    with pytest.raises(ValueError):
        chunked.slot_kinds(queries.kat_plans()["q1"])
