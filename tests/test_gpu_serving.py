"""GPU tests of the request loop (cx_server_*): queries submitted as they
arrive, admitted against an HBM budget and fused into shared-scan launches,
must each return exactly what the query returns alone (its plain kernel) and
what the CPU oracle returns."""
import random

import numpy as np
import pytest

import oracle
from practice_b200 import _lib, datagen, queries
from practice_b200.plan import PlanBuilder, col

pytestmark = pytest.mark.gpu

DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}


@pytest.fixture(scope="module")
def db():
    from practice_b200.engine import Database
    return Database(0)


def load(db, seed, n):
    ht = datagen.host_tables(seed, n, queries.BATCH_COLS)
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, queries.BATCH_COLS))
    return ht


def oracle_run(plan, ht):
    rows = {"LINEORDER": ht.fact_rows, **DIM_ROWS}
    return oracle.run_plan(plan.text(), ht.columns, ht.validity, rows, plan.group_slots * plan.storage_ts)


def avg_plan(n, y):
    """A query the shared scan does not take (AVG): it runs alone, beside the batches."""
    b = PlanBuilder(datagen.ssb_tables(n, queries.BATCH_COLS), "LINEORDER", name="avg")
    b.filter(col("lo_quantity").lt(25))
    b.join("DDATE", "lo_orderdate", where=col("d_year").ge(y))
    return b.aggregate([queries._g("d_year")], [("avg", col("lo_revenue")), ("count", col("lo_revenue"))])


def check(srv, db, rid, plan, ht, alone=True):
    info = srv.wait(rid, 120_000)
    assert info.status == 0 and info.kernel_error == 0, (info.status, info.kernel_error)
    w, v = srv.fetch(rid, info)
    ref = oracle_run(plan, ht)
    np.testing.assert_array_equal(w, ref.words[: len(w)])
    np.testing.assert_array_equal(v, ref.validity[: len(v)])
    if alone:
        solo = db.execute(plan)
        np.testing.assert_array_equal(w, solo.words)
        np.testing.assert_array_equal(v, solo.validity)
    srv.release(rid)
    return info


def test_server_stream_results_equal_alone_and_oracle(db):
    n = 4_000_037
    ht = load(db, 51, n)
    rng = random.Random(5)
    plans = [queries.template(rng.randrange(4), rng, n) for _ in range(48)]
    plans += [avg_plan(n, 1994)] * 3
    random.Random(6).shuffle(plans)
    # One launch in flight: queries submitted while it runs wait together, so
    # two or more waiting queries form a shared launch.
    srv = _lib.Server(db.ctx, _lib.server_config(max_batch=16, slots=1, min_shared_batch=2))
    try:
        for t in range(4):  # compile the four shapes and the AVG kernel before the stream
            srv.prepare(queries.template(t, random.Random(t), n).text())
        srv.prepare(plans[[p.name for p in plans].index("avg")].text())
        ids = [srv.submit(p.text()) for p in plans]
        infos = [check(srv, db, rid, p, ht) for rid, p in zip(ids, plans)]
        st = srv.stats()
        assert st.completed == len(plans) and st.rejected == 0
        assert st.mean_batch > 1.0, "arrivals while the GPU was busy must share launches"
        assert any(i.shared == 0 for i in infos) and any(i.shared == 1 and i.batch_size > 1 for i in infos)
        assert all(i.latency_ms >= i.queue_ms >= 0 for i in infos)
        assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
    finally:
        srv.close()


def test_server_admission_under_a_small_budget(db):
    """A budget that holds the slots' scratch and a few large result tables:
    queries wait for memory, run in smaller launches and are all still exact;
    a query larger than the whole budget is refused."""
    n = 300_007
    ht = load(db, 52, n)
    rng = random.Random(9)
    tables = datagen.ssb_tables(n, queries.BATCH_COLS)
    big = []
    for k in range(8):  # 1000 brands x 25 nations x 7 years: 4.2 MB of result words each
        b = PlanBuilder(tables, "LINEORDER", name="big")
        b.join("CUSTOMER", "lo_custkey", where=col("c_region").le(k % 5))
        b.join("PART", "lo_partkey")
        b.join("DDATE", "lo_orderdate")
        big.append(b.aggregate([queries._g("p_brand1"), queries._g("c_nation"), queries._g("d_year")],
                               [("sum", col("lo_revenue"))]))
    plans = big + [queries.template(3, rng, n) for _ in range(6)] + [queries.template(1, rng, n) for _ in range(6)]
    # Two slots' dimension indexes (about 14 MB each once grown) plus room for
    # about three of the big result tables at a time.
    budget = 40 << 20
    srv = _lib.Server(db.ctx, _lib.server_config(max_batch=64, slots=2, budget_bytes=budget))
    try:
        b = PlanBuilder(datagen.ssb_tables(n, queries.BATCH_COLS), "LINEORDER", name="huge")
        b.join("CUSTOMER", "lo_custkey")
        b.join("PART", "lo_partkey")
        b.join("DDATE", "lo_orderdate")
        # 1000 brands x 250 cities x 7 years = 1.75M groups: 28 MB of result words alone
        huge = b.aggregate([queries._g("p_brand1"), queries._g("c_city"), queries._g("d_year")],
                           [("sum", col("lo_revenue"))])
        with pytest.raises(_lib.CxError) as e:
            srv.submit(huge.text())
        assert e.value.code == -8
        ids = [srv.submit(p.text()) for p in plans]
        for rid, p in zip(ids, plans):
            check(srv, db, rid, p, ht, alone=False)
        st = srv.stats()
        assert st.completed == len(plans) and st.rejected == 1
        assert st.peak_reserved_bytes <= budget
        assert st.launches >= 3, "the big queries cannot all be admitted at once"
    finally:
        srv.close()


def test_server_plain_only_runs_one_query_per_launch(db):
    n = 200_003
    ht = load(db, 53, n)
    rng = random.Random(10)
    plans = [queries.template(t, rng, n) for t in (0, 1, 2, 3, 1)]
    srv = _lib.Server(db.ctx, _lib.server_config(plain_only=1, slots=1))
    try:
        ids = [srv.submit(p.text()) for p in plans]
        infos = [check(srv, db, rid, p, ht, alone=False) for rid, p in zip(ids, plans)]
        assert all(i.batch_size == 1 and i.shared == 0 for i in infos)
        assert srv.stats().launches == len(plans)
    finally:
        srv.close()


def test_server_short_queues_run_plain_kernels(db):
    """Shareable queries that find fewer than min_shared_batch others waiting
    run alone through their parametric plain kernel; one module per shape
    serves queries with different literals."""
    n = 200_029
    ht = load(db, 54, n)
    rng = random.Random(11)
    plans = [queries.template(t, rng, n) for t in (1, 2, 1, 3, 0, 2)]
    srv = _lib.Server(db.ctx, _lib.server_config(min_shared_batch=1_000_000))
    try:
        infos = []
        for p in plans:
            rid = srv.submit(p.text())
            infos.append(check(srv, db, rid, p, ht, alone=False))
        assert all(i.batch_size == 1 and i.shared == 0 for i in infos)
    finally:
        srv.close()


@pytest.mark.parametrize("chunk", [1_000_000, 1_500_000])
def test_circular_scan_results_equal_alone_and_oracle(db, chunk):
    """Circular scans: each shared launch covers the next row range; queries
    that arrive join at a range boundary, carry their partial results between
    launches and finish after one revolution.  Every result equals the query
    alone and the oracle, also for queries that join in the middle and wrap
    around the end of the table."""
    n = 4_000_037
    ht = load(db, 52, n)
    rng = random.Random(8)
    plans = [queries.template(rng.randrange(4), rng, n) for _ in range(40)]
    plans += [avg_plan(n, 1995)] * 2
    random.Random(9).shuffle(plans)
    srv = _lib.Server(db.ctx, _lib.server_config(max_batch=16, slots=1, min_shared_batch=2, chunk_rows=chunk))
    try:
        for t in range(4):
            srv.prepare(queries.template(t, random.Random(t), n).text())
        srv.prepare(plans[[p.name for p in plans].index("avg")].text())
        ids = []
        for i, p in enumerate(plans):  # arrivals spread over several ranges
            ids.append(srv.submit(p.text()))
            if i % 7 == 6:
                srv.wait(ids[-1], 120_000)
        infos = [check(srv, db, rid, p, ht) for rid, p in zip(ids, plans)]
        st = srv.stats()
        assert st.completed == len(plans) and st.rejected == 0
        assert any(i.shared == 1 for i in infos)
        # A revolution takes ceil(n / chunk) launches, so shared queries ran in several.
        assert st.launches >= (n + chunk - 1) // chunk
    finally:
        srv.close()
