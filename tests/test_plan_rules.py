"""The plan builder's restatements of the reference visitor's derivations
(CPU): hash-table build parameters (computeBuildInfo, src/core/visitor.cpp:
3864-4016), the PHT_2 payload choice (:3970-4016), result nullability
(resultColumnNullableForExpr, :128-170) and fast sparse output
(aggregateFastSparseOutputEligible, :2215-2231), plus the plan text of
OR-joins and multi-value joins."""
import pytest

from practice_b200 import datagen
from practice_b200.plan import (Group, PlanBuilder, Table, build_params, case, col, expr_nullable, lit, not_,
                                null, or_, sparse_eligible, star)

N = 1000
COLS = ["lo_orderdate", "lo_commitdate", "lo_custkey", "lo_partkey", "lo_revenue", "lo_quantity"]


def tables():
    return datagen.ssb_tables(N, COLS)


def test_build_params_follow_compute_build_info():
    t = tables()
    assert build_params(t["PART"]) == (200_000, 0)          # P_LEN, key minimum 0
    assert build_params(t["CUSTOMER"]) == (300_000, 0)
    assert build_params(t["DDATE"]) == (61_131, 19_920_101)  # one spare slot past 19981230
    assert build_params(t["PARTSUPP"]) == (200_000, 1)      # catalog range of the key column
    assert build_params(Table("X", ["x_key", "x_v"], 77)) == (77, 0)  # no stats: table size


def test_payload_is_the_first_dimension_column_the_aggregate_then_a_later_filter_reads():
    b = PlanBuilder(tables(), "LINEORDER")
    b.join("CUSTOMER", "lo_custkey")
    b.filter(col("c_region").eq(1))
    p = b.aggregate([Group(col("c_nation"), 0, 25)], [("sum", col("lo_revenue"))])
    assert p.steps[0][1].payload == "c_nation"          # aggregate columns win over filter columns
    b = PlanBuilder(tables(), "LINEORDER")
    b.join("CUSTOMER", "lo_custkey")
    b.filter(col("c_region").eq(1))
    p = b.aggregate([], [("sum", col("lo_revenue"))])
    assert p.steps[0][1].payload == "c_region"          # else the first later filter column
    b = PlanBuilder(tables(), "LINEORDER")
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(1))
    p = b.aggregate([], [("count", star())])
    assert p.steps[0][1].payload is None                 # nothing read above the join: PHT_1


@pytest.mark.parametrize("expr,nullable", [
    (null(), True), (star(), False), (lit(3), False),
    (col("lo_revenue"), True), (col("lo_quantity"), False),
    (col("lo_revenue").is_null(), False), (col("lo_revenue").not_null(), False),
    (not_(col("lo_revenue").gt(1)), True), (not_(col("lo_quantity").gt(1)), False),
    (col("lo_quantity") + col("lo_revenue"), True), (or_(col("lo_quantity").gt(1), lit(0)), False),
    (case(col("lo_revenue").gt(1), col("lo_quantity"), lit(0)), False),   # the condition does not count
    (case(col("lo_quantity").gt(1), lit(1), col("lo_revenue")), True),
])
def test_result_nullability(expr, nullable):
    assert expr_nullable(expr, {"lo_revenue"}) is nullable


def _plan(groups, aggs, nullable=(), order_by=None):
    b = PlanBuilder(tables(), "LINEORDER", nullable=nullable)
    b.join("DDATE", "lo_orderdate")
    return b.aggregate(groups, aggs, order_by=order_by)


def test_fast_sparse_output_eligibility():
    year, qty0 = Group(col("d_year"), 1992, 7), Group(col("lo_quantity"), 0, 51)
    assert sparse_eligible(_plan([], [("sum", col("lo_revenue"))]))                    # scalar
    assert sparse_eligible(_plan([year], [("sum", col("lo_revenue"))]))                # key domain starts above 0
    assert not sparse_eligible(_plan([qty0], [("sum", col("lo_revenue"))]))            # zero key, no COUNT
    assert sparse_eligible(_plan([qty0], [("sum", col("lo_revenue")), ("count", star())]))
    assert not sparse_eligible(_plan([year], [("avg", col("lo_revenue"))]))            # hidden count slot
    assert not sparse_eligible(_plan([year], [("min", col("lo_revenue"))]))            # COUNT / SUM only
    assert not sparse_eligible(_plan([year], [("sum", col("lo_revenue"))], nullable={"lo_revenue"}))
    assert sparse_eligible(_plan([year], [("count", col("lo_revenue"))], nullable={"lo_revenue"}))
    assert not sparse_eligible(_plan([year], [("sum", col("lo_revenue"))], order_by=[(1, True)]))  # dense for ORDER BY


def test_or_join_and_multi_value_join_plan_text():
    b = PlanBuilder(tables(), "LINEORDER")
    b.join("DDATE", ("lo_orderdate", "lo_commitdate"))
    b.join("PARTSUPP", "lo_partkey", where=col("ps_availqty").lt(10))
    b.filter(col("ps_supplycost").gt(5))
    p = b.aggregate([Group(col("d_year"), 1992, 7), Group(col("ps_tier"), 0, 5)], [("sum", col("lo_revenue"))])
    text = p.text()
    assert "(fk lo_orderdate lo_commitdate)" in text and "(payload d_year)" in text
    ps = p.steps[1][1]
    assert ps.multi and ps.payload is None and ps.expands
    assert set(ps.gathers) == {"ps_tier", "ps_supplycost"}   # every build column used above the join
    assert "(multi 1)" in text and "(payload ps_tier ps_supplycost)" in text
    assert p.columns_read() == ["lo_orderdate", "lo_commitdate", "lo_partkey", "lo_revenue"]
