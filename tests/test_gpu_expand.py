"""GPU parity of the joins that expand rows: OR-joins over several fact keys
and multi-value hash tables (non-unique build keys), through the C ABI, against
the CPU oracle on the same seeded tables.  Bit-exact on every word of the raw
aggregate buffer and its validity bitmap."""
import dataclasses

import numpy as np
import pytest

import oracle
from practice_b200 import _lib, datagen, queries
from practice_b200.engine import make_tuning

pytestmark = pytest.mark.gpu

DIMS = dict(datagen.DIM_ROWS)
ALL_COLS = sorted(set(queries.OR_COLS + queries.MHT_COLS))


@pytest.fixture(scope="module")
def db():
    from practice_b200.engine import Database
    return Database(0)


def load(db, seed, n, nulls=None):
    ht = datagen.host_tables(seed, n, ALL_COLS, nulls, dims=("DDATE", "SUPPLIER", "PART", "PARTSUPP"))
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, ALL_COLS))
    return ht


def assert_parity(db, plan, ht, tuning=None):
    ref = oracle.run_plan(plan.text(), ht.columns, ht.validity, {"LINEORDER": ht.fact_rows, **DIMS},
                          plan.group_slots * plan.storage_ts)
    got = db.execute(plan, tuning)
    assert got.kernel_error == 0
    fw = len(got.words)
    np.testing.assert_array_equal(got.words, ref.words[:fw])
    np.testing.assert_array_equal(got.validity, ref.validity[: (fw + 63) // 64])
    return got


@pytest.mark.parametrize("n", [2_000_000, 1_000_003, 33, 1])
def test_or_join_year(db, n):
    ht = load(db, 41, n)
    got = assert_parity(db, queries.or_join_year(n), ht)
    if n >= 1_000_000:
        assert got.words[1] != 0
    assert_parity(db, queries.or_join_year(n, (1995, 1998)), ht)


def test_or_join_nullable_second_key_and_payload_filter(db):
    n = 1_500_001
    ht = load(db, 42, n, nulls={"lo_commitdate": 150, "lo_revenue": 80})
    assert_parity(db, queries.or_join_year(n, nullable=("lo_commitdate",)), ht)
    assert_parity(db, queries.or_join_then_filter(n), ht)


@pytest.mark.parametrize("tuning", [None, dict(block_threads=256, items_per_thread=4, stages=2),
                                    dict(block_threads=128, items_per_thread=8, stages=0)])
def test_mht_year_tier(db, tuning):
    n = 1_200_007
    ht = load(db, 43, n)
    t = make_tuning(**tuning) if tuning else None
    for avail in (5000, 10_000, 1):
        got = assert_parity(db, queries.mht_year_tier(n, avail), ht, t)
        if avail == 1:
            assert not got.words.any()


def test_mht_then_pht_and_gathered_filter(db):
    n = 1_000_001
    ht = load(db, 44, n)
    got = assert_parity(db, queries.mht_then_supplier(n), ht)
    assert got.words[1] != 0


@pytest.mark.parametrize("placement", [0, 2])
def test_mht_large_group_domain(db, placement):
    n = 1_000_000
    ht = load(db, 45, n, nulls={"ps_tier": 100})
    t = make_tuning(group_placement=placement)
    assert_parity(db, queries.mht_brand(n), ht, t)
    assert_parity(db, queries.mht_brand(n, nullable_tier=True), ht, t)


@pytest.mark.parametrize("placement", [0, 1, 2])
def test_group_placements_in_item_mode(db, placement):
    """Register (or_join_year default), shared-memory and global group
    tables, each updated per expanded row."""
    n = 700_001
    ht = load(db, 48, n, nulls={"lo_revenue": 60})
    t = make_tuning(group_placement=placement)
    for p in (queries.or_join_year(n), queries.or_join_then_filter(n), queries.mht_year_tier(n)):
        assert_parity(db, p, ht, t)


def test_warp_uniform_expansion(db):
    """group_merge = 1: the expansion runs as a warp-uniform loop with equal
    groups merged across the warp before the atomics."""
    n = 600_011
    ht = load(db, 49, n, nulls={"lo_revenue": 60, "ps_tier": 80})
    for placement in (0, 2):
        t = make_tuning(group_placement=placement, group_merge=1)
        for p in (queries.or_join_then_filter(n), queries.mht_year_tier(n), queries.mht_brand(n, nullable_tier=True)):
            src = _lib.codegen(p.text(), t)
            assert "bool act_" in src
            assert_parity(db, p, ht, t)


def test_or_over_three_keys_and_or_inside_a_multi_value_join(db):
    """(lo_custkey OR lo_suppkey OR lo_partkey) = c_custkey, and
    (lo_partkey OR lo_suppkey) = ps_partkey on the non-unique PARTSUPP key;
    some keys are made equal so the duplicate-key rule is exercised."""
    from practice_b200.plan import PlanBuilder, col, star
    n = 800_017
    cols = ALL_COLS + ["lo_custkey"]
    ht = datagen.host_tables(50, n, cols, dims=("DDATE", "CUSTOMER", "SUPPLIER", "PART", "PARTSUPP"))
    ht.columns["lo_suppkey"][::50] = ht.columns["lo_custkey"][::50]
    ht.columns["lo_partkey"][::70] = ht.columns["lo_suppkey"][::70]
    db.reset()
    db.load_host_tables(ht, datagen.ssb_tables(n, cols))
    tabs = datagen.ssb_tables(n, cols)
    b = PlanBuilder(tabs, "LINEORDER", name="or3")
    b.join("CUSTOMER", ("lo_custkey", "lo_suppkey", "lo_partkey"), where=col("c_region").le(2))
    or3 = b.aggregate([queries._g("c_region")], [("sum", col("lo_revenue")), ("count", star())])
    b = PlanBuilder(tabs, "LINEORDER", name="mht_or")
    b.join("DDATE", "lo_orderdate")
    b.join("PARTSUPP", ("lo_partkey", "lo_suppkey"), where=col("ps_availqty").lt(6000))
    mht_or = b.aggregate([queries._g("d_year"), queries._g("ps_tier")], [("sum", col("lo_revenue")), ("count", star())])
    for p in (or3, mht_or):
        got = assert_parity(db, p, ht)
        assert got.words.any()


def test_mht_slot_collision_raises_a_kernel_error(db):
    n = 100_000
    ht = load(db, 46, n)
    p = queries.mht_year_tier(n)
    steps = [(k, dataclasses.replace(s, length=100_000) if k == "join" and s.multi else s) for k, s in p.steps]
    got = db.execute(dataclasses.replace(p, steps=steps))
    assert got.kernel_error == 4  # ERR_DIM_COLLISION
    with pytest.raises(RuntimeError, match="collision"):
        oracle.run_plan(dataclasses.replace(p, steps=steps).text(), ht.columns, ht.validity,
                        {"LINEORDER": n, **DIMS}, p.group_slots * p.storage_ts)


def test_expanding_plans_are_not_shared(db):
    n = 1000
    load(db, 47, n)
    for p in (queries.or_join_year(n), queries.mht_year_tier(n)):
        assert not db.shareable(p)
        with pytest.raises(_lib.CxError):
            _lib.shared_codegen([p.text()])
