"""Query plans of the measured workloads and of the reference's known-answer set.

* ``ssb_q11`` -- plain single query over a 6M-row fact table: date join with
  year = 1995 (PHT_1), discount in [2, 4], quantity < 30,
  SUM(extendedprice * discount) (SSB Q1.1 shape, test/queries/sql/q11.sql).
* ``ssb_q31`` -- four-dimension star: customer region = r, supplier region = r,
  year in [1992, 1997], GROUP BY (c_nation, s_nation, d_year), SUM(revenue),
  ORDER BY year ASC, sum DESC (SSB Q3.1 shape, test/queries/sql/q31.sql).
* ``ssb_q31_nullable`` -- the nullable three-valued-logic variant: NULL revenue and
  NULL customer.city, IS NULL / IS NOT NULL and range predicates that yield
  UNKNOWN (on a fact column and on a joined payload); COUNT(*),
  COUNT(revenue), SUM(revenue) grouped by a nullable key.
* ``template(t, rng)`` -- the four shared-scan templates: T0 range filters +
  scalar SUM; T1 date join + GROUP BY year; T2 three joins + GROUP BY
  (nation, year); T3 four joins + GROUP BY (brand, year) (<= 7,000 groups).
* ``serving_stream`` / ``city_pairs`` / ``wide_groups`` -- the serving workload:
  the templates with fresh constants per request plus a many-group query
  (up to 62,500 groups); and a large-domain query (8.25M group slots, a
  330 MB result, <= 90,000 groups present) for admission under the budget.
* ``kat_*`` -- the five queries of test/nullable_data/queries.sql.
* ``or_join_year`` -- the OR-join over two fact keys of
  test/queries/sql/custom1.sql: (lo_orderdate = d_datekey OR lo_commitdate =
  d_datekey), year in [1992, 1997], GROUP BY d_year, SUM(revenue).
* ``mht_*`` -- joins on PARTSUPP, whose key ps_partkey is non-unique, so each
  fact row expands to every matching build row (multi-value hash table,
  test/queries/sql/mht/non_unique_projection.sql semantics under an aggregate).
"""
from __future__ import annotations

import random

from .datagen import GROUP_STATS, ssb_tables
from .plan import Group, Plan, PlanBuilder, Table, and_, case, col, lit, not_, or_, star

Q11_COLS = ["lo_orderdate", "lo_quantity", "lo_discount", "lo_extendedprice"]
Q31_COLS = ["lo_orderdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_revenue", "lo_supplycost"]
BATCH_COLS = ["lo_orderdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_quantity", "lo_discount",
           "lo_revenue", "lo_supplycost"]
OR_COLS = ["lo_orderdate", "lo_commitdate", "lo_revenue"]
MHT_COLS = ["lo_orderdate", "lo_suppkey", "lo_partkey", "lo_quantity", "lo_revenue"]


def _g(name: str, nullable: bool = False) -> Group:
    mn, card = GROUP_STATS[name]
    return Group(col(name), mn, card, nullable)


def ssb_q11(fact_rows: int = 6_000_000, year: int = 1995, disc: tuple[int, int] = (2, 4), qty: int = 30) -> Plan:
    t = ssb_tables(fact_rows, Q11_COLS)
    b = PlanBuilder(t, "LINEORDER", name="ssb_q11")
    b.filter(and_(col("lo_discount").ge(disc[0]), col("lo_discount").le(disc[1]), col("lo_quantity").lt(qty)))
    b.join("DDATE", "lo_orderdate", where=col("d_year").eq(year))
    return b.aggregate([], [("sum", col("lo_extendedprice") * col("lo_discount"))])


def ssb_q31(fact_rows: int = 60_000_000, region: int = 2, years: tuple[int, int] = (1992, 1997)) -> Plan:
    t = ssb_tables(fact_rows, Q31_COLS)
    b = PlanBuilder(t, "LINEORDER", name="ssb_q31")
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(region))
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(region))
    b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(years[0]), col("d_year").le(years[1])))
    return b.aggregate([_g("c_nation"), _g("s_nation"), _g("d_year")], [("sum", col("lo_revenue"))],
                       order_by=[(2, False), (3, True)])


def ssb_q31_nullable(fact_rows: int = 60_000_000, region: int = 1, years: tuple[int, int] = (1993, 1998),
            rev_floor: int = 2_000_000) -> Plan:
    t = ssb_tables(fact_rows, Q31_COLS)
    nullable = {"lo_revenue", "c_city"}
    b = PlanBuilder(t, "LINEORDER", nullable=nullable, name="ssb_q31_nullable")
    # (revenue >= floor OR revenue IS NULL) AND (NOT (revenue > 9,500,000) OR
    # revenue IS NULL): the range terms are UNKNOWN for a NULL revenue (NOT
    # keeps it UNKNOWN), IS NULL on each OR lets such rows through, so
    # COUNT(revenue) and SUM(revenue) see them and skip them.
    b.filter(and_(or_(col("lo_revenue").ge(rev_floor), col("lo_revenue").is_null()),
                  or_(not_(col("lo_revenue").gt(9_500_000)), col("lo_revenue").is_null())))
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(region), payload="c_city")
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(region))
    b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(years[0]), col("d_year").le(years[1])))
    # IS NOT NULL over a joined payload and a fact column: rows whose city and
    # revenue are both NULL drop out; a NULL city with a known revenue stays
    # and forms the NULL group.
    b.filter(or_(col("c_city").not_null(), col("lo_revenue").not_null()))
    return b.aggregate([_g("c_city", nullable=True), _g("d_year")],
                       [("count", star()), ("count", col("lo_revenue")), ("sum", col("lo_revenue"))],
                       order_by=[(1, False), (0, False)])


def ssb_q31_tables(fact_rows: int) -> dict[str, Table]:
    return ssb_tables(fact_rows, Q31_COLS)


# --------------------------------------------------- OR-joins and MHT joins


def or_join_year(fact_rows: int = 60_000_000, years: tuple[int, int] = (1992, 1997),
                 nullable: tuple[str, ...] = ()) -> Plan:
    t = ssb_tables(fact_rows, OR_COLS)
    b = PlanBuilder(t, "LINEORDER", nullable=nullable, name="or_join_year")
    b.join("DDATE", ("lo_orderdate", "lo_commitdate"),
           where=and_(col("d_year").ge(years[0]), col("d_year").le(years[1])))
    return b.aggregate([_g("d_year")], [("sum", col("lo_revenue"))])


def or_join_then_filter(fact_rows: int = 60_000_000, month: int = 6) -> Plan:
    """OR-join whose payload feeds a later fact-side filter and a grouped
    MIN/MAX/AVG/COUNT over a nullable key (item-mode tail after the OR)."""
    t = ssb_tables(fact_rows, OR_COLS)
    b = PlanBuilder(t, "LINEORDER", nullable=("lo_revenue",), name="or_join_then_filter")
    b.join("DDATE", ("lo_commitdate", "lo_orderdate"), payload="d_month")
    b.filter(or_(col("d_month").le(month), col("lo_revenue").is_null()))
    return b.aggregate([_g("d_month")], [("count", star()), ("min", col("lo_revenue")), ("max", col("lo_revenue")),
                                         ("avg", col("lo_revenue"))])


def mht_year_tier(fact_rows: int = 60_000_000, avail: int = 5000) -> Plan:
    t = ssb_tables(fact_rows, MHT_COLS)
    b = PlanBuilder(t, "LINEORDER", name="mht_year_tier")
    b.join("DDATE", "lo_orderdate")
    b.join("PARTSUPP", "lo_partkey", where=col("ps_availqty").lt(avail))
    return b.aggregate([_g("d_year"), _g("ps_tier")], [("sum", col("lo_revenue")), ("count", star())])


def mht_then_supplier(fact_rows: int = 60_000_000, region: int = 2, tier_max: int = 3) -> Plan:
    """MHT first, a PHT join and a filter over a gathered column after it,
    scalar SUM over a gathered column times a fact column."""
    t = ssb_tables(fact_rows, MHT_COLS)
    b = PlanBuilder(t, "LINEORDER", name="mht_then_supplier")
    b.filter(col("lo_quantity").lt(40))
    b.join("PARTSUPP", "lo_partkey")
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(region))
    b.filter(col("ps_tier").le(tier_max))
    return b.aggregate([], [("sum", col("lo_quantity") * col("ps_supplycost")), ("count", star()),
                            ("max", col("ps_availqty"))])


def mht_brand(fact_rows: int = 60_000_000, nullable_tier: bool = False) -> Plan:
    """MHT after two PHT joins, a large group domain (shared-memory or global
    atomics in item mode) and optionally a nullable gathered group key."""
    t = ssb_tables(fact_rows, MHT_COLS)
    nullable = ("ps_tier",) if nullable_tier else ()
    b = PlanBuilder(t, "LINEORDER", nullable=nullable, name="mht_brand")
    b.join("PART", "lo_partkey", where=col("p_mfgr").le(1))
    b.join("DDATE", "lo_orderdate")
    b.join("PARTSUPP", "lo_partkey")
    return b.aggregate([_g("p_brand1"), _g("d_year"), _g("ps_tier", nullable_tier)],
                       [("sum", col("lo_revenue")), ("count", star())])


# --------------------------------------------------------------- templates

TEMPLATE_NAMES = ["T0_scan_sum", "T1_date_year", "T2_nation_year", "T3_brand_year"]


def template(t: int, rng: random.Random, fact_rows: int = 600_000_000) -> Plan:
    """One query of template t with constants drawn from rng (selectivity
    0.01%-20%)."""
    tables = ssb_tables(fact_rows, BATCH_COLS)
    if t == 0:
        q_hi = rng.randint(2, 50)
        q_lo = rng.randint(1, q_hi)
        d_lo = rng.randint(0, 10)
        d_hi = rng.randint(d_lo, min(10, d_lo + 3))
        b = PlanBuilder(tables, "LINEORDER", name="T0")
        b.filter(and_(col("lo_quantity").ge(q_lo), col("lo_quantity").le(q_hi),
                      col("lo_discount").ge(d_lo), col("lo_discount").le(d_hi)))
        return b.aggregate([], [("sum", col("lo_revenue") * col("lo_discount"))])
    if t == 1:
        y_lo = rng.randint(1992, 1998)
        y_hi = rng.randint(y_lo, 1998)
        q = rng.randint(2, 50)
        b = PlanBuilder(tables, "LINEORDER", name="T1")
        b.filter(col("lo_quantity").lt(q))
        b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(y_lo), col("d_year").le(y_hi)))
        return b.aggregate([_g("d_year")], [("sum", col("lo_revenue"))])
    if t == 2:
        r = rng.randint(0, 4)
        s = rng.randint(0, 4)
        y_lo = rng.randint(1992, 1998)
        y_hi = rng.randint(y_lo, 1998)
        b = PlanBuilder(tables, "LINEORDER", name="T2")
        b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(r))
        b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(s))
        b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(y_lo), col("d_year").le(y_hi)))
        return b.aggregate([_g("c_nation"), _g("d_year")], [("sum", col("lo_revenue"))])
    cat = rng.randint(0, 24)
    r = rng.randint(0, 4)
    s = rng.randint(0, 4)
    b = PlanBuilder(tables, "LINEORDER", name="T3")
    b.join("PART", "lo_partkey", where=col("p_category").eq(cat))
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(s))
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").le(r))
    b.join("DDATE", "lo_orderdate")
    return b.aggregate([_g("p_brand1"), _g("d_year")], [("sum", col("lo_revenue") - col("lo_supplycost"))])


def batch(n: int, seed: int, fact_rows: int = 600_000_000) -> list[Plan]:
    rng = random.Random(seed)
    return [template(rng.randrange(4), rng, fact_rows) for _ in range(n)]


def wide_groups(rng: random.Random, fact_rows: int = 600_000_000) -> Plan:
    """A large-domain query of the serving stream: customer and supplier region
    joins, a year, a 3-value discount range; GROUP BY (c_city, s_city,
    lo_discount, d_month).  The group domain is 250 * 250 * 11 * 12 =
    8,250,000 slots (a 330 MB result buffer) of which at most 50 * 50 * 3 * 12 =
    90,000 groups occur."""
    tables = ssb_tables(fact_rows, BATCH_COLS)
    r = rng.randint(0, 4)
    s = rng.randint(0, 4)
    y = rng.randint(1992, 1998)
    d0 = rng.randint(0, 8)
    b = PlanBuilder(tables, "LINEORDER", name="T4")
    b.filter(and_(col("lo_discount").ge(d0), col("lo_discount").le(d0 + 2)))
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(r))
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(s))
    b.join("DDATE", "lo_orderdate", where=col("d_year").eq(y))
    return b.aggregate([_g("c_city"), _g("s_city"), _g("lo_discount"), _g("d_month")], [("sum", col("lo_revenue"))])


def city_pairs(rng: random.Random, fact_rows: int = 600_000_000) -> Plan:
    """A many-group query of the serving stream: customer regions up to r,
    a supplier region, a year range; GROUP BY (c_city, s_city), SUM(revenue):
    up to 62,500 groups (a 1.5 MB result)."""
    tables = ssb_tables(fact_rows, BATCH_COLS)
    r = rng.randint(0, 4)
    s = rng.randint(0, 4)
    y_lo = rng.randint(1992, 1998)
    y_hi = rng.randint(y_lo, 1998)
    b = PlanBuilder(tables, "LINEORDER", name="T5")
    b.join("CUSTOMER", "lo_custkey", where=col("c_region").le(r))
    b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(s))
    b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(y_lo), col("d_year").le(y_hi)))
    return b.aggregate([_g("c_city"), _g("s_city")], [("sum", col("lo_revenue"))])


def serving_stream(n: int, seed: int, fact_rows: int = 600_000_000, many_share: float = 0.05) -> list[Plan]:
    """Requests of the serving workload: the four batch templates with fresh
    random constants each, and with probability `many_share` a many-group
    query (`city_pairs`); group cardinalities from 1 to 62,500."""
    rng = random.Random(seed)
    return [city_pairs(rng, fact_rows) if rng.random() < many_share else template(rng.randrange(4), rng, fact_rows)
            for _ in range(n)]


# ------------------------------------------------------- known-answer set

KAT_COLS = ["id", "grp", "val", "flag"]


def kat_tables(rows: int = 12) -> dict[str, Table]:
    return {"NULLABLE_NUMBERS": Table("NULLABLE_NUMBERS", list(KAT_COLS), rows, fact=True)}


def kat_plans(rows: int = 12, grp_card: int = 4) -> dict[str, Plan]:
    """test/nullable_data/queries.sql q1-q5 as plans (val and flag nullable)."""
    t = kat_tables(rows)
    nul = {"val", "flag"}
    grp = Group(col("grp"), 1, grp_card, False)
    plans = {}
    b = PlanBuilder(t, "NULLABLE_NUMBERS", nullable=nul, name="q1")
    plans["q1"] = b.aggregate([], [("count", star()), ("count", col("val")), ("sum", col("val")), ("avg", col("val"))])
    b = PlanBuilder(t, "NULLABLE_NUMBERS", nullable=nul, name="q2")
    plans["q2"] = b.aggregate([grp], [("count", star()), ("count", col("val")), ("sum", col("val"))],
                              order_by=[(0, False)])
    b = PlanBuilder(t, "NULLABLE_NUMBERS", nullable=nul, name="q3")
    b.filter(col("val").is_null())
    plans["q3"] = b.aggregate([], [("count", star())])
    b = PlanBuilder(t, "NULLABLE_NUMBERS", nullable=nul, name="q4")
    b.filter(col("flag").eq(1))
    plans["q4"] = b.aggregate([], [("count", star())])
    b = PlanBuilder(t, "NULLABLE_NUMBERS", nullable=nul, name="q5")
    plans["q5"] = b.aggregate([Group(col("grp"), 1, grp_card, False)],
                              [("sum", case(col("val").is_null(), lit(1), lit(0)))], order_by=[(0, False)])
    return plans
