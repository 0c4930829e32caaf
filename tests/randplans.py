"""Seeded random star-join plans for the fuzz tests (test helper, not product).

`harness_plan` draws only the shapes the reference-primitive harness runs
(AND-chains of `column op literal` fact filters, one-payload joins, GROUP BY
over fact columns or join payloads, COUNT(*) and SUM of a column, a product
or a difference); `engine_plan` adds what only the oracle and the CUDA path
cover: nullable columns under three-valued logic, OR / NOT / IS NULL filters,
MIN / MAX / AVG / COUNT(column), CASE aggregates and filters after joins.
Either may carry one expanding join (an OR over two date keys, or the
multi-value PARTSUPP join)."""
from __future__ import annotations

import random

from practice_b200.datagen import GROUP_STATS, ssb_tables
from practice_b200.plan import Group, PlanBuilder, and_, case, col, lit, not_, or_, star

FACT_COLS = ["lo_orderdate", "lo_commitdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_quantity",
             "lo_discount", "lo_revenue", "lo_supplycost"]
DIMS = ("DDATE", "CUSTOMER", "SUPPLIER", "PART", "PARTSUPP")
FK = {"DDATE": "lo_orderdate", "CUSTOMER": "lo_custkey", "SUPPLIER": "lo_suppkey", "PART": "lo_partkey",
      "PARTSUPP": "lo_partkey"}
PAYLOADS = {"DDATE": ["d_year", "d_month"], "CUSTOMER": ["c_region", "c_nation"],
            "SUPPLIER": ["s_region", "s_nation"], "PART": ["p_mfgr", "p_category"], "PARTSUPP": ["ps_tier"]}
OPS = ("eq", "ne", "lt", "le", "gt", "ge")


def _cmp(rng, c, lo, hi):
    return getattr(col(c), rng.choice(OPS))(rng.randint(lo, hi))


def _dim_filter(rng, dim):
    if dim == "DDATE":
        y = rng.randint(1992, 1998)
        return and_(col("d_year").ge(y), col("d_year").le(rng.randint(y, 1998)))
    if dim in ("CUSTOMER", "SUPPLIER"):
        p = dim[0].lower()
        return getattr(col(f"{p}_region"), rng.choice(("eq", "le", "ge")))(rng.randint(0, 4))
    if dim == "PART":
        return col("p_mfgr").le(rng.randint(0, 4))
    return col("ps_availqty").lt(rng.randint(1000, 10_000))


def _group(name, nullable=False):
    mn, card = GROUP_STATS[name]
    return Group(col(name), mn, card, nullable)


def harness_plan(rng: random.Random, rows: int, name: str = "fuzz", expanding_ok: bool = True):
    b = PlanBuilder(ssb_tables(rows, FACT_COLS), "LINEORDER", name=name)
    preds = [_cmp(rng, "lo_quantity", 1, 50) for _ in range(rng.randint(0, 2))]
    preds += [_cmp(rng, "lo_discount", 0, 10) for _ in range(rng.randint(0, 1))]
    if preds:
        b.filter(and_(*preds))
    dims = rng.sample(["DDATE", "CUSTOMER", "SUPPLIER", "PART"], rng.randint(0, 3))
    expanding = rng.choice((None, None, "or", "mht")) if expanding_ok else None
    if expanding == "mht" and "PART" not in dims:
        dims.append("PARTSUPP")
    if expanding == "or" and "DDATE" not in dims:
        dims.insert(rng.randint(0, len(dims)), "DDATE")
    groups = []
    for d in dims:
        fk = ("lo_orderdate", "lo_commitdate") if d == "DDATE" and expanding == "or" else FK[d]
        b.join(d, fk, where=_dim_filter(rng, d) if rng.random() < 0.8 else None)
        if len(groups) < 2 and rng.random() < 0.6:
            g = rng.choice(PAYLOADS[d])
            groups.append(_group(g))
    if not groups and rng.random() < 0.4:
        groups.append(_group(rng.choice(("lo_quantity", "lo_discount"))))
    aggs = [("count", star())] if rng.random() < 0.5 else []
    a, c2 = rng.choice(("lo_revenue", "lo_supplycost", "lo_quantity")), rng.choice(("lo_discount", "lo_quantity"))
    aggs.append(("sum", rng.choice((col(a), col(a) * col(c2), col(a) - col(c2)))))
    return b.aggregate(groups, aggs)


def engine_plan(rng: random.Random, rows: int, nullable: tuple[str, ...], name: str = "fuzz"):
    b = PlanBuilder(ssb_tables(rows, FACT_COLS), "LINEORDER", nullable=nullable, name=name)
    if rng.random() < 0.7:
        f = _cmp(rng, "lo_quantity", 1, 50)
        if rng.random() < 0.5:
            f = or_(f, col("lo_revenue").is_null())
        if rng.random() < 0.3:
            f = and_(f, not_(_cmp(rng, "lo_discount", 0, 10)))
        b.filter(f)
    dims = rng.sample(["DDATE", "CUSTOMER", "SUPPLIER", "PART"], rng.randint(0, 3))
    expanding = rng.choice((None, None, "or", "mht"))
    if expanding == "mht" and "PART" not in dims:
        dims.append("PARTSUPP")
    if expanding == "or" and "DDATE" not in dims:
        dims.insert(rng.randint(0, len(dims)), "DDATE")
    groups = []
    for d in dims:
        fk = ("lo_orderdate", "lo_commitdate") if d == "DDATE" and expanding == "or" else FK[d]
        b.join(d, fk, where=_dim_filter(rng, d) if rng.random() < 0.8 else None)
        if len(groups) < 2 and rng.random() < 0.6:
            g = rng.choice(PAYLOADS[d])
            groups.append(_group(g, g in nullable))
            if rng.random() < 0.3:
                b.filter(getattr(col(g), rng.choice(OPS))(GROUP_STATS[g][0] + rng.randint(0, 3)))
    if not groups and rng.random() < 0.4:
        groups.append(_group("lo_quantity", "lo_quantity" in nullable))
    pool = [("count", star()), ("count", col("lo_revenue")), ("sum", col("lo_revenue")),
            ("min", col("lo_revenue")), ("max", col("lo_supplycost") - col("lo_discount")),
            ("avg", col("lo_quantity")),
            ("sum", case(col("lo_discount").gt(5), col("lo_revenue"), lit(0)))]
    aggs = rng.sample(pool, rng.randint(1, 3))
    return b.aggregate(groups, aggs)
