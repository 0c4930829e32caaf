"""The query shapes of tests/golden/visitor/*.sycl as plans of this package's
plan builder, with the same literals oracle/visitor/emit_visitor.cpp gives the
reference's code generator.  The oracle evaluates these plans; the GPU runs the
reference-emitted programs through cx_compile / cx_execute."""
from practice_b200 import datagen, queries
from practice_b200.plan import Group, PlanBuilder, and_, col

ALL_COLS = ["lo_orderdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_quantity", "lo_discount",
            "lo_extendedprice", "lo_revenue", "lo_supplycost"]


def _g(name):
    mn, card = datagen.GROUP_STATS[name]
    return Group(col(name), mn, card, False)


def plan(name: str, n: int):
    t = datagen.ssb_tables(n, ALL_COLS)
    if name == "q11":
        return queries.ssb_q11(n)
    b = PlanBuilder(t, "LINEORDER", name=name)
    if name == "q31":  # the SSB Q3.1 shape without its ORDER BY (the fixture's tree has no sort)
        b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(2))
        b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(2))
        b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(1992), col("d_year").le(1997)))
        return b.aggregate([_g("c_nation"), _g("s_nation"), _g("d_year")], [("sum", col("lo_revenue"))])
    if name == "t0":
        b.filter(and_(col("lo_quantity").ge(5), col("lo_quantity").le(35), col("lo_discount").ge(3),
                      col("lo_discount").le(5)))
        return b.aggregate([], [("sum", col("lo_revenue") * col("lo_discount"))])
    if name == "t1":
        b.filter(col("lo_quantity").lt(25))
        b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(1993), col("d_year").le(1996)))
        return b.aggregate([_g("d_year")], [("sum", col("lo_revenue"))])
    if name == "t2":
        b.join("CUSTOMER", "lo_custkey", where=col("c_region").eq(3))
        b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(1))
        b.join("DDATE", "lo_orderdate", where=and_(col("d_year").ge(1994), col("d_year").le(1998)))
        return b.aggregate([_g("c_nation"), _g("d_year")], [("sum", col("lo_revenue"))])
    if name == "t3":
        b.join("PART", "lo_partkey", where=col("p_category").eq(7))
        b.join("SUPPLIER", "lo_suppkey", where=col("s_region").eq(2))
        b.join("CUSTOMER", "lo_custkey", where=col("c_region").le(3))
        b.join("DDATE", "lo_orderdate")
        return b.aggregate([_g("p_brand1"), _g("d_year")], [("sum", col("lo_revenue") - col("lo_supplycost"))])
    raise KeyError(name)


TRANSLATED = ["q11", "q31", "t0", "t1", "t2", "t3"]
