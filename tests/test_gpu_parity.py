"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded tables.  Integer work, so the bar is bit-exact: every word of the
raw aggregate buffer and of its validity bitmap must match."""
import random

import numpy as np
import pytest

import oracle
from practice_b200 import _lib, datagen, queries, results
from practice_b200.engine import SHARED_DEFAULT, make_tuning
from practice_b200.plan import Group, PlanBuilder, and_, col, lit, not_, or_, star

pytestmark = pytest.mark.gpu

DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}


@pytest.fixture(scope="module")
def db():
    from practice_b200.engine import Database
    return Database(0)


def load(db, seed, n, fact_cols, nulls=None):
    ht = datagen.host_tables(seed, n, fact_cols, nulls)
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, fact_cols))
    return ht


def oracle_run(plan, ht):
    rows = {"LINEORDER": ht.fact_rows, **DIM_ROWS}
    return oracle.run_plan(plan.text(), ht.columns, ht.validity, rows, plan.group_slots * plan.storage_ts)


def assert_parity(db, plan, ht, tuning=None):
    ref = oracle_run(plan, ht)
    got = db.execute(plan, tuning)
    assert got.kernel_error == 0
    fw = len(got.words)  # groups x visible tuple after AVG finalisation, else the storage tuple
    np.testing.assert_array_equal(got.words, ref.words[:fw])
    np.testing.assert_array_equal(got.validity, ref.validity[: (fw + 63) // 64])
    return got, ref


@pytest.mark.parametrize("n", [1_000_000, 1_000_003, 511, 1])
def test_q11_shape(db, n):
    ht = load(db, 11, n, queries.Q11_COLS)
    got, _ = assert_parity(db, queries.ssb_q11(n), ht)
    if n >= 1_000_000:
        assert got.words[0] != 0


def test_q31_shape(db):
    n = 2_000_000
    ht = load(db, 12, n, queries.Q31_COLS)
    plan = queries.ssb_q31(n)
    got, _ = assert_parity(db, plan, ht)
    assert len(got.rows(plan)) > 100


def test_q31_nullable(db):
    n = 2_000_003
    ht = load(db, 13, n, queries.Q31_COLS, nulls={"lo_revenue": 100, "c_city": 50})
    plan = queries.ssb_q31_nullable(n)
    got, _ = assert_parity(db, plan, ht)
    rs = got.rows(plan)
    assert any(r[0] is None for r in rs), "NULL c_city must form its own group"
    assert any(r[3] < r[2] for r in rs), "COUNT(revenue) must skip NULL revenue"


@pytest.mark.parametrize("compact", [0, 1, 2])
@pytest.mark.parametrize("t", [0, 1, 2, 3])
def test_shared_scan_templates(db, t, compact):
    n = 1_500_000
    ht = load(db, 14, n, queries.BATCH_COLS)
    rng = random.Random(100 + t)
    tun = _lib.default_tuning()
    tun.compact = compact
    for _ in range(3):
        assert_parity(db, queries.template(t, rng, n), ht, tun)


@pytest.mark.parametrize("bt,ipt,stages,place,merge,bitmaps,compact,prefetch", [
    (128, 4, 4, 0, 0, 98304, 0, 1), (256, 8, 2, 0, 1, 0, 0, 1), (512, 2, 3, 2, 0, 98304, 0, 1),
    (256, 4, 0, 1, 2, 98304, 0, 1), (1024, 1, 2, 0, 2, 0, 0, 1), (256, 4, 6, 2, 1, 98304, 0, 1),
    (1024, 2, 0, 1, 1, 98304, 0, 1), (1024, 4, 0, 0, 0, 49152, 1, 1), (512, 8, 0, 2, 0, 49152, 1, 1),
    (1024, 4, 0, 1, 0, 0, 1, 1), (256, 2, 0, 0, 2, 98304, 1, 1), (1024, 4, 0, 0, 0, 49152, 2, 1),
    (512, 2, 0, 2, 0, 49152, 2, 1), (1024, 4, 0, 0, 0, 49152, 1, 3), (512, 2, 0, 2, 0, 0, 0, 3),
    (1024, 2, 0, 0, 0, 49152, 2, 3), (256, 4, 0, 1, 2, 98304, 0, 2)])
def test_tuning_invariance(db, bt, ipt, stages, place, merge, bitmaps, compact, prefetch):
    n = 777_777
    ht = load(db, 15, n, queries.Q31_COLS, nulls={"lo_revenue": 100, "c_city": 50})
    t = _lib.default_tuning()
    t.block_threads, t.items_per_thread, t.stages, t.group_placement = bt, ipt, stages, place
    t.group_merge, t.bitmap_budget, t.compact, t.prefetch = merge, bitmaps, compact, prefetch
    assert_parity(db, queries.ssb_q31_nullable(n), ht, t)
    assert_parity(db, queries.ssb_q31(n), ht, t)


def test_empty_fact_table(db):
    ht = load(db, 16, 0, queries.Q11_COLS)
    got, ref = assert_parity(db, queries.ssb_q11(0), ht)
    assert int(got.words[0]) == 0


def test_empty_selection_and_all_null(db):
    n = 100_000
    ht = load(db, 17, n, queries.Q31_COLS, nulls={"lo_revenue": 1000, "c_city": 1000})
    assert_parity(db, queries.ssb_q31(n, years=(2050, 2060)), ht)
    plan = queries.ssb_q31_nullable(n)
    got, _ = assert_parity(db, plan, ht)
    assert all(r[0] is None and r[2] == 0 for r in got.rows(plan))


def test_min_max_avg_and_case(db):
    n = 300_001
    ht = load(db, 18, n, queries.BATCH_COLS, nulls={"lo_revenue": 200})
    tabs = datagen.ssb_tables(n, queries.BATCH_COLS)
    nul = {"lo_revenue"}
    b = PlanBuilder(tabs, "LINEORDER", nullable=nul)
    b.filter(or_(col("lo_quantity").lt(10), col("lo_revenue").is_null()))
    b.join("DDATE", "lo_orderdate", where=col("d_month").le(6))
    plan = b.aggregate([Group(col("d_year"), 1992, 7)],
                       [("min", col("lo_revenue")), ("max", col("lo_revenue") - col("lo_supplycost")),
                        ("avg", col("lo_revenue")), ("count", col("lo_revenue")),
                        ("sum", queries.case(col("lo_revenue").is_null(), lit(1), lit(0)))])
    assert_parity(db, plan, ht)
    b = PlanBuilder(tabs, "LINEORDER", nullable=nul)
    b.filter(not_(col("lo_discount").ge(5)))
    plan = b.aggregate([], [("min", col("lo_revenue")), ("max", col("lo_supplycost")), ("avg", col("lo_quantity")),
                            ("count", star()), ("sum", col("lo_quantity") * col("lo_discount") + lit(3))])
    assert_parity(db, plan, ht)


def test_kat_on_gpu(db):
    import json
    from pathlib import Path
    gold = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
    t = gold["nullable_kat"]["columns"]
    n = len(t["id"])
    db.reset()
    for c in t:
        db.load_column("NULLABLE_NUMBERS", c, np.array([v if v is not None else 0 for v in t[c]], dtype=np.int32))
    for c in ("val", "flag"):
        bits = np.zeros(64, dtype=np.uint8)
        bits[:n] = [v is not None for v in t[c]]
        db.load_validity(c, np.packbits(bits, bitorder="little").view("<u8").astype(np.uint64))
    db.set_rows("NULLABLE_NUMBERS", n)
    for q, plan in queries.kat_plans(n).items():
        got = db.execute(plan)
        rs = got.rows(plan)
        if q == "q4":
            assert rs == [(5,)]
            continue
        exp = gold["nullable_kat"]["expected"][q]["rows"]
        assert [list(r) for r in rs] == [[pytest.approx(v) if isinstance(v, float) else v for v in e] for e in exp]


def test_group_domain_violation_is_reported(db):
    """A GROUP BY key outside its catalog domain raises error code 2 (the
    reference folds it silently into another group)."""
    n = 50_000
    ht = load(db, 19, n, queries.BATCH_COLS)
    tabs = datagen.ssb_tables(n, queries.BATCH_COLS)
    b = PlanBuilder(tabs, "LINEORDER")
    b.join("DDATE", "lo_orderdate")
    plan = b.aggregate([Group(col("d_year"), 1992, 5)], [("count", star())])
    ref = oracle_run(plan, ht)
    got = db.execute(plan)
    assert ref.domain_errors > 0
    assert got.kernel_error == 2


def test_device_generator_matches_host(db):
    import torch
    n = 1_000_037
    for c in queries.BATCH_COLS + ["lo_extendedprice"]:
        t = torch.empty(n, dtype=torch.int32, device="cuda")
        datagen.fact_column_device(c, 5, n, t.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t.cpu().numpy(), datagen.fact_column(c, 5, 0, n))
    w = torch.empty((n + 63) // 64, dtype=torch.int64, device="cuda")
    datagen.validity_device("lo_revenue", 5, n, 100, w.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(w.cpu().numpy().view(np.uint64),
                                  datagen.validity_words(5, datagen.STREAMS["valid_lo_revenue"], n, 100))


def test_sparse_compaction(db):
    import torch
    n = 400_000
    ht = load(db, 20, n, queries.BATCH_COLS)
    plan = queries.template(3, random.Random(7), n)
    assert plan.sparse
    got = db.execute(plan)
    src = torch.from_numpy(got.words.view(np.int64)).cuda()
    dst = torch.zeros_like(src)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(_lib.lib.cx_compact_sparse(src.data_ptr(), plan.group_slots, plan.storage_ts, dst.data_ptr(),
                                          cnt.data_ptr(), None))
    torch.cuda.synchronize()
    k = int(cnt.item())
    ts = plan.storage_ts
    tuples = got.words.reshape(-1, ts)
    expect = tuples[(tuples != 0).any(axis=1)]
    assert k == len(expect) > 0
    np.testing.assert_array_equal(dst.cpu().numpy().view(np.uint64)[: k * ts].reshape(-1, ts), expect)


# ------------------------------------------------------------ shared scans

@pytest.mark.parametrize("nq,tune", [(16, None), (37, (512, 2, 2)), (64, (256, 4, 2)), (5, (1024, 1, 1)),
                                     (33, (512, 2, 2, 2)), (48, (1024, 1, 3, 3))])
def test_shared_scan_batch_matches_oracle_per_query(db, nq, tune):
    """Every query of a mixed-template batch run as ONE shared scan equals the
    oracle run on that query alone (same words, same validity bits)."""
    n = 700_001
    ht = load(db, 30 + nq, n, queries.BATCH_COLS)
    plans = queries.batch(nq, 1000 + nq, n)
    t = None
    if tune:
        t = _lib.default_tuning()
        t.block_threads, t.items_per_thread, t.stages = tune[:3]
        if len(tune) > 3:
            t.group_merge = tune[3]  # 2: direct adds for tiny domains too; 3: per-row atomics above 32 groups
    assert all(db.shareable(p) for p in plans)
    got = db.execute_shared(plans, t)
    assert got[0].kernel_error == 0
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words)
        np.testing.assert_array_equal(g.validity, ref.validity)


def test_shared_scan_q31_and_repeat(db):
    """The SSB Q3.1 shape through the shared path, twice in a row (buffers and
    dimension indexes are rebuilt per batch)."""
    n = 500_003
    ht = load(db, 41, n, queries.Q31_COLS)
    plans = [queries.ssb_q31(n, region=r, years=(1992 + r, 1997)) for r in range(5)]
    for _ in range(2):
        got = db.execute_shared(plans)
        for p, g in zip(plans, got):
            ref = oracle_run(p, ht)
            np.testing.assert_array_equal(g.words, ref.words)
            np.testing.assert_array_equal(g.validity, ref.validity)


def test_shared_scan_two_passes(db):
    """A batch larger than one pass (64 queries) runs as consecutive passes
    over the fact table; every query still equals the oracle."""
    n = 300_007
    ht = load(db, 43, n, queries.BATCH_COLS)
    plans = queries.batch(90, 4242, n)
    got = db.execute_shared(plans)
    assert got[0].kernel_error == 0
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words)
        np.testing.assert_array_equal(g.validity, ref.validity)


@pytest.mark.parametrize("rng_lo,rng_hi", [(40, 45), (1000, 2000), (-300, -100)])
def test_shared_scan_values_outside_filter_windows(db, rng_lo, rng_hi):
    """Per-query path: fact values outside the filter tables' window fall back
    to per-query evaluation, so a registered range that misses most values
    gives the same answers.  The aggregate-cube path takes the range as a
    bound and reports the values outside it (kernel error 5) rather than
    answering wrongly."""
    n = 400_009
    ht = load(db, 44, n, queries.BATCH_COLS)
    db.ctx.set_column_range("d_lo_quantity", rng_lo, rng_hi)
    db.ctx.set_column_range("d_lo_discount", rng_lo, rng_hi)
    plans = queries.batch(24, 77, n)
    got = db.execute_shared(plans, make_tuning(**{**SHARED_DEFAULT, "cube": 0}))
    assert got[0].timing.mode == 0
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words)
        np.testing.assert_array_equal(g.validity, ref.validity)
    got = db.execute_shared(plans, make_tuning(**SHARED_DEFAULT))
    assert got[0].timing.mode == 1 and got[0].kernel_error == 5


@pytest.mark.parametrize("cube,nq", [(0, 40), (1, 40), (2, 40), (4, 40), (4, 1), (4, 130)])
def test_shared_scan_cube_and_mask_paths(db, cube, nq):
    """A mixed batch through the aggregate-cube path (cube = rows per lane of
    its scan; one pass whatever the batch size) and through the per-query mask
    path (cube = 0): every query equals the oracle on its own, and the timing
    reports which path ran.  The fact table's size is not a multiple of a warp
    tile, so the ragged last tile is covered."""
    n = 600_011
    ht = load(db, 47, n, queries.BATCH_COLS)
    plans = queries.batch(nq, 4700 + nq, n)
    got = db.execute_shared(plans, make_tuning(**{**SHARED_DEFAULT, "cube": cube}))
    assert got[0].kernel_error == 0
    assert got[0].timing.mode == (1 if cube else 0)
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words, err_msg=p.name)
        np.testing.assert_array_equal(g.validity, ref.validity, err_msg=p.name)


def test_shared_scan_cube_path_falls_back_for_wide_shapes(db):
    """A shape whose cube would exceed 16,777,216 cells (GROUP BY c_city,
    s_city, lo_discount, d_month under region and year filters) sends the whole
    batch down the per-query mask path; the answers still equal the oracle."""
    n = 300_007
    ht = load(db, 48, n, queries.BATCH_COLS)
    rng = random.Random(48)
    plans = [queries.wide_groups(rng, n)] + [queries.template(t, rng, n) for t in range(4)]
    got = db.execute_shared(plans)
    assert got[0].kernel_error == 0 and got[0].timing.mode == 0
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words, err_msg=p.name)
        np.testing.assert_array_equal(g.validity, ref.validity, err_msg=p.name)


def test_shared_scan_residual_filters(db):
    """Conjuncts over two fact columns are evaluated per row and query after
    the mask; they share a batch with filter-table and join-only shapes."""
    n = 350_011
    ht = load(db, 45, n, queries.BATCH_COLS)
    tables = datagen.ssb_tables(n, queries.BATCH_COLS)
    plans = []
    for k in range(3):
        b = PlanBuilder(tables, "LINEORDER", name="R")
        b.filter(and_(col("lo_quantity").lt(col("lo_discount") * lit(5 + k)), col("lo_discount").ge(k)))
        b.join("DDATE", "lo_orderdate", where=col("d_year").ge(1993 + k))
        plans.append(b.aggregate([Group(col("d_year"), 1992, 7, False)],
                                 [("sum", col("lo_revenue")), ("count", star())]))
    for k in range(2):  # a later filter on a join payload joins the dimension's mask
        b = PlanBuilder(tables, "LINEORDER", name="PF")
        b.join("DDATE", "lo_orderdate")
        b.filter(col("d_year").ne(1994 + k))
        plans.append(b.aggregate([Group(col("d_year"), 1992, 7, False)], [("count", star())]))
    rng = random.Random(9)
    plans += [queries.template(t, rng, n) for t in (0, 1, 3)]
    got = db.execute_shared(plans)
    for p, g in zip(plans, got):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(g.words, ref.words)
        np.testing.assert_array_equal(g.validity, ref.validity)


def test_shared_scan_graph_replay(db):
    """A batch is captured into a CUDA graph once; later batches with the same
    pass shapes (same shape mix, new literals and new result buffers) replay
    it and still equal the oracle; direct launches give the same answers."""
    n = 300_017
    ht = load(db, 46, n, queries.BATCH_COLS)
    rng = random.Random(78)
    kinds = [0, 1, 2, 3, 1, 2, 0, 3]
    modes = []
    for _ in range(3):
        plans = [queries.template(t, rng, n) for t in kinds]
        got = db.execute_shared(plans)
        modes.append(got[0].timing.graph)
        for p, g in zip(plans, got):
            ref = oracle_run(p, ht)
            np.testing.assert_array_equal(g.words, ref.words)
            np.testing.assert_array_equal(g.validity, ref.validity)
    assert modes[0] in (1, 2) and modes[1] == 1 and modes[2] == 1, modes
    db.ctx.set_graph_replay(False)
    try:
        plans = [queries.template(t, rng, n) for t in kinds]
        got = db.execute_shared(plans)
        assert got[0].timing.graph == 0
        for p, g in zip(plans, got):
            ref = oracle_run(p, ht)
            np.testing.assert_array_equal(g.words, ref.words)
    finally:
        db.ctx.set_graph_replay(True)


def test_parametric_plain_kernel_serves_every_literal(db):
    """One parametric module per plan shape, the literals passed at launch,
    returns what a kernel compiled for each query's literals returns."""
    n = 250_013
    ht = load(db, 47, n, queries.BATCH_COLS)
    rng = random.Random(81)
    t = _lib.default_tuning()
    t.parametric = 1
    for tpl in range(4):
        plans = [queries.template(tpl, rng, n) for _ in range(3)]
        mods = set()
        for p in plans:
            got = db.execute(p, t)
            mods.add(db.compile(p, t).handle.value)
            assert got.kernel_error == 0
            ref = oracle_run(p, ht)
            np.testing.assert_array_equal(got.words, ref.words[: len(got.words)])
            np.testing.assert_array_equal(got.validity, ref.validity[: (len(got.words) + 63) // 64])
        assert len(mods) == 1


def test_parametric_plain_kernel_nullable_shape(db):
    n = 300_019
    ht = load(db, 48, n, queries.Q31_COLS, nulls={"lo_revenue": 100, "c_city": 50})
    t = _lib.default_tuning()
    t.parametric = 1
    for region, years, floor in ((1, (1993, 1998), 2_000_000), (3, (1992, 1995), 500_000)):
        plan = queries.ssb_q31_nullable(n, region=region, years=years, rev_floor=floor)
        got = db.execute(plan, t)
        ref = oracle_run(plan, ht)
        fw = len(got.words)
        np.testing.assert_array_equal(got.words, ref.words[:fw])
        np.testing.assert_array_equal(got.validity, ref.validity[: (fw + 63) // 64])


@pytest.mark.parametrize("budget", [0, 98304])
@pytest.mark.parametrize("nullable_payload", [False, True])
def test_join_keys_outside_the_slot_window(db, budget, nullable_payload):
    """Foreign keys below the hash window, past it (aliasing into a slot that
    holds another key), equal to 0, the largest dimension key (which HASH maps
    to slot 0) and the int32 extremes: the exact shared-memory bitmaps must
    answer like the full probe (budget 98304) and like no bitmaps (0)."""
    n = 300_007
    ht = load(db, 23, n, queries.Q31_COLS, nulls={"c_city": 70} if nullable_payload else None)
    rng = np.random.default_rng(5)
    odd_cust = np.array([0, -1, 300_000, 300_001, 600_000, 2**31 - 1, -2**31], dtype=np.int64)
    odd_date = np.array([0, 19_920_100, 19_920_101 + 61_131, 19_920_101 + 61_131 + 366, 19_981_231, 2**31 - 1,
                         -2**31, 19_920_101 - 61_131 + 5], dtype=np.int64)
    cust = ht.columns["lo_custkey"].copy()
    date = ht.columns["lo_orderdate"].copy()
    pick = rng.choice(n, 4000, replace=False)
    cust[pick[:2000]] = odd_cust[rng.integers(0, len(odd_cust), 2000)].astype(np.int32)
    date[pick[2000:]] = odd_date[rng.integers(0, len(odd_date), 2000)].astype(np.int32)
    ht.columns["lo_custkey"], ht.columns["lo_orderdate"] = cust, date
    db.load_column("LINEORDER", "lo_custkey", cust)
    db.load_column("LINEORDER", "lo_orderdate", date)
    tabs = datagen.ssb_tables(n, queries.Q31_COLS)
    nullable = {"c_city"} if nullable_payload else set()
    b = PlanBuilder(tabs, "LINEORDER", nullable=nullable)
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").le(3), payload="c_city")
    b.join("DDATE", "lo_orderdate", where=col("d_year").ge(1993))
    b.join("SUPPLIER", "lo_suppkey")
    plan = b.aggregate([Group(col("c_city"), 0, 250, nullable_payload), queries._g("d_year")],
                       [("count", star()), ("sum", col("lo_revenue"))])
    from practice_b200.engine import make_tuning
    for ipt, stages in ((4, 0), (2, 2)):
        assert_parity(db, plan, ht, make_tuning(items_per_thread=ipt, stages=stages, bitmap_budget=budget))


@pytest.mark.parametrize("splits", [[0, 400_000, 1_000_000], [0, 1024, 512_000, 899_968]])
def test_shared_scan_over_row_ranges_accumulates(db, splits):
    """A batch answered by consecutive launches over row ranges -- the first
    zeroing each query's result, the later ones adding to it (keep) -- equals
    the oracle over the whole table, for every query; a query that joins at a
    later range and wraps around to the first covers the table too."""
    n = 1_000_003
    ht = load(db, 41, n, queries.BATCH_COLS)
    plans = queries.batch(12, 41, n)
    prog = db.shared_program(plans)
    qs, params, bufs = db.shared_prepare(prog, plans)
    for t, r in db.rows.items():
        db.ctx.set_rows(t, r)
    stream = db.torch.cuda.current_stream().cuda_stream
    bounds = splits + [n]
    ranges = [(bounds[i], bounds[i + 1] - bounds[i]) for i in range(len(splits))]
    # Queries 0..5 start at the first range; queries 6..11 start at the second
    # and wrap around to the first at the end.
    order_a = ranges
    order_b = ranges[1:] + ranges[:1]
    for k in range(len(ranges)):
        db.ctx.shared_execute_rows(prog.module, qs[:6], params, order_a[k][0], order_a[k][1], keep=[k > 0] * 6,
                                   stream=stream)
        db.ctx.sync()
        db.ctx.shared_execute_rows(prog.module, qs[6:], params, order_b[k][0], order_b[k][1], keep=[k > 0] * 6,
                                   stream=stream)
        db.ctx.sync()
    for p, (res, val, words) in zip(plans, bufs):
        ref = oracle_run(p, ht)
        np.testing.assert_array_equal(res.cpu().numpy().view(np.uint64)[:words], ref.words[:words], err_msg=p.name)


@pytest.mark.parametrize("compact", [0, 1])
def test_payload_tables_with_values_outside_the_catalog_range(db, compact):
    """A payload range narrower than the data (here years 1994-1995 for a
    1992-1998 column) marks the other slots 'fetch from the hash table': the
    result still equals the oracle's; so do the default ranges and no tables."""
    n = 1_000_003
    ht = load(db, 43, n, queries.Q31_COLS)
    plan = queries.ssb_q31(n)
    ref = oracle_run(plan, ht)
    variants = [(plan.text(), 96 * 1024), (plan.text().replace("(prange 1992 7)", "(prange 1994 2)"), 96 * 1024),
                (plan.text(), 0)]
    for text, budget in variants:
        t = _lib.default_tuning()
        t.compact, t.table_budget = compact, budget
        m = _lib.Module(_lib.codegen(text, t), key=f"ptable_{compact}_{budget}_{hash(text)}")
        res, val = db.alloc_result(m)
        for tn, r in db.rows.items():
            db.ctx.set_rows(tn, r)
        db.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
        db.ctx.execute(m, db.torch.cuda.current_stream().cuda_stream)
        db.ctx.sync()
        fw = int(m.info.final_words)
        np.testing.assert_array_equal(res.cpu().numpy().view(np.uint64)[:fw], ref.words[:fw])
        np.testing.assert_array_equal(val.cpu().numpy().view(np.uint64)[: (fw + 63) // 64], ref.validity[: (fw + 63) // 64])


@pytest.mark.parametrize("cube", [0, 2])
def test_shared_scan_duplicate_dimension_key_is_reported(db, cube):
    """Two CUSTOMER rows with the same key make a shared batch that joins
    CUSTOMER fail with kernel error 4 on both paths, rather than answer from
    whichever row was indexed last."""
    n = 100_003
    ht = datagen.host_tables(49, n, queries.BATCH_COLS)
    keys = ht.columns["c_custkey"].copy()
    keys[7] = keys[6]
    ht.columns["c_custkey"] = keys
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, queries.BATCH_COLS))
    plans = [queries.template(2, random.Random(3 + k), n) for k in range(4)]
    got = db.execute_shared(plans, make_tuning(**{**SHARED_DEFAULT, "cube": cube}))
    assert got[0].timing.mode == (1 if cube else 0)
    assert got[0].kernel_error == 4
