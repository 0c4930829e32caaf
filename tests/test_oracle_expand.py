"""Oracle properties of the joins that expand rows (CPU, no reference build
needed): an OR over two fact keys equals the single-key join on the first key
plus the single-key join on the second key where the keys differ
(visitor.cpp:4587-4640); a multi-value hash table over a unique key equals the
perfect-hash join, and over a dimension holding every row twice doubles every
SUM and COUNT (visitor.cpp:4672-4730); two distinct keys in one MHT slot are an
error."""
import dataclasses

import numpy as np
import pytest

import oracle
from practice_b200 import datagen, queries
from practice_b200.plan import PlanBuilder, and_, col, star

N = 120_007
DIMS = {**{k: v for k, v in datagen.DIM_ROWS.items()}}


@pytest.fixture(scope="module")
def ht():
    cols = sorted(set(queries.OR_COLS + queries.MHT_COLS))
    return datagen.host_tables(31, N, cols, dims=("DDATE", "SUPPLIER", "PART", "PARTSUPP"))


def run(plan, ht, columns=None, rows=None):
    r = {"LINEORDER": N, **DIMS, **(rows or {})}
    return oracle.run_plan(plan.text(), columns or ht.columns, ht.validity, r, plan.group_slots * plan.storage_ts)


def year_plan(fks, pre_filter=None):
    t = datagen.ssb_tables(N, queries.OR_COLS)
    b = PlanBuilder(t, "LINEORDER")
    if pre_filter is not None:
        b.filter(pre_filter)
    b.join("DDATE", fks, where=col("d_year").le(1997))
    return b.aggregate([queries._g("d_year")], [("sum", col("lo_revenue")), ("count", star())])


def test_or_join_is_the_sum_of_its_distinct_key_branches(ht):
    both = run(year_plan(("lo_orderdate", "lo_commitdate")), ht).words
    first = run(year_plan("lo_orderdate"), ht).words
    second = run(year_plan("lo_commitdate", col("lo_commitdate").ne(col("lo_orderdate"))), ht).words
    ts = 3
    for g in range(7):
        for k in (1, 2):
            assert both[g * ts + k] == first[g * ts + k] + second[g * ts + k]
    # Rows whose two keys are equal exist and are counted once.
    assert (ht.columns["lo_commitdate"] == ht.columns["lo_orderdate"]).sum() > 100


def test_or_join_with_null_second_key_counts_the_first_only(ht):
    valid = datagen.validity_words(31, 999, N, 1000)  # every lo_commitdate NULL
    plan = year_plan(("lo_orderdate", "lo_commitdate"))
    plan.nullable = {"lo_commitdate"}
    r = oracle.run_plan(plan.text(), ht.columns, {**ht.validity, "lo_commitdate": valid}, {"LINEORDER": N, **DIMS},
                        plan.group_slots * plan.storage_ts)
    np.testing.assert_array_equal(r.words, run(year_plan("lo_orderdate"), ht).words)


def _as_multi(plan):
    steps = []
    for kind, s in plan.steps:
        if kind == "join" and s.dim == "PART":
            s = dataclasses.replace(s, multi=True, gathers=(s.payload,) if s.payload else (), payload=None)
        steps.append((kind, s))
    return dataclasses.replace(plan, steps=steps)


def part_plan():
    t = datagen.ssb_tables(N, queries.MHT_COLS)
    b = PlanBuilder(t, "LINEORDER")
    b.join("PART", "lo_partkey", where=col("p_mfgr").le(2))
    b.join("DDATE", "lo_orderdate")
    return b.aggregate([queries._g("p_category"), queries._g("d_year")], [("sum", col("lo_revenue")), ("count", star())])


def test_mht_over_a_unique_key_equals_the_perfect_hash_join(ht):
    pht = part_plan()
    mht = _as_multi(pht)
    assert "(multi 1)" in mht.text() and "(multi 1)" not in pht.text()
    np.testing.assert_array_equal(run(mht, ht).words, run(pht, ht).words)
    np.testing.assert_array_equal(run(mht, ht).validity, run(pht, ht).validity)


def test_mht_over_a_doubled_dimension_doubles_sums_and_counts(ht):
    mht = _as_multi(part_plan())
    cols = dict(ht.columns)
    for c in ("p_partkey", "p_mfgr", "p_category", "p_brand1"):
        cols[c] = np.concatenate([ht.columns[c], ht.columns[c][::-1]])
    once = run(mht, ht).words
    twice = run(mht, ht, cols, {"PART": 2 * DIMS["PART"]}).words
    ts = 4
    g = np.arange(len(once) // ts)
    np.testing.assert_array_equal(twice[g * ts + 2], 2 * once[g * ts + 2])
    np.testing.assert_array_equal(twice[g * ts + 3], 2 * once[g * ts + 3])
    np.testing.assert_array_equal(twice[g * ts], once[g * ts])


def test_mht_partsupp_expands_rows(ht):
    p = queries.mht_year_tier(N, avail=10_000)
    r = run(p, ht).words
    count = r[3::4].sum()
    # every fact row matches its part key's PARTSUPP rows (all pass the filter)
    per_key = np.bincount(ht.columns["ps_partkey"], minlength=DIMS["PART"] + 1)
    assert count == per_key[ht.columns["lo_partkey"]].sum()


def test_mht_slot_collision_is_an_error(ht):
    p = queries.mht_year_tier(N)
    steps = [(k, dataclasses.replace(s, length=100_000) if k == "join" and s.multi else s) for k, s in p.steps]
    with pytest.raises(RuntimeError, match="collision"):
        run(dataclasses.replace(p, steps=steps), ht)


def test_or_join_over_three_keys_is_the_sum_of_its_distinct_key_branches(ht):
    """(lo_custkey = c_custkey OR lo_suppkey = c_custkey OR lo_partkey = c_custkey):
    each key probes unless it equals an earlier key of the row."""
    def plan(fks, pre=None):
        b = PlanBuilder(datagen.ssb_tables(N, queries.MHT_COLS + ["lo_custkey"]), "LINEORDER")
        if pre is not None:
            b.filter(pre)
        b.join("CUSTOMER", fks, where=col("c_region").le(2))
        return b.aggregate([queries._g("c_region")], [("sum", col("lo_revenue")), ("count", star())])

    cols = dict(ht.columns)
    cols.update(datagen.dim_columns("CUSTOMER", 31))
    cols["lo_custkey"] = datagen.fact_column("lo_custkey", 31, 0, N)
    # make some keys equal so the duplicate rule is exercised
    cols["lo_suppkey"] = cols["lo_suppkey"].copy()
    cols["lo_suppkey"][::50] = cols["lo_custkey"][::50]
    cols["lo_partkey"] = cols["lo_partkey"].copy()
    cols["lo_partkey"][::70] = cols["lo_suppkey"][::70]
    all3 = run(plan(("lo_custkey", "lo_suppkey", "lo_partkey")), ht, cols).words
    k1 = run(plan("lo_custkey"), ht, cols).words
    k2 = run(plan("lo_suppkey", col("lo_suppkey").ne(col("lo_custkey"))), ht, cols).words
    k3 = run(plan("lo_partkey", and_(col("lo_partkey").ne(col("lo_custkey")), col("lo_partkey").ne(col("lo_suppkey")))),
             ht, cols).words
    ts = 3
    for g in range(5):
        for k in (1, 2):
            assert all3[g * ts + k] == k1[g * ts + k] + k2[g * ts + k] + k3[g * ts + k]
    assert all3[1::3].sum() > k1[1::3].sum() > 0
