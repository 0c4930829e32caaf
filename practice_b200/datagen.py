"""Seeded synthetic star-schema data (SSB-shaped), host and device.

The reference reads SSB dbgen output from disk (include/crystal/utils.h:10-26,
242-253); dbgen is not available, so tables are generated from a
counter-based hash instead.  Every value depends only on (seed, column stream,
row), so the device generator (``cx_gen_*`` in libcrystal_b200.so, cx_rng.h)
and the numpy restatement here produce identical columns, and any row range can
be regenerated on its own (the CPU baseline samples rows this way).

Domains follow the configured workloads: dimension keys 1..N (the PHT empty
sentinel is 0, include/crystal/join.h:140-141), dates yyyymmdd from 1992-01-01,
dense hierarchies (region 0..4, nation = region*5 + U5, city = nation*10 + U10;
mfgr 0..4, category = mfgr*5 + U5, brand = category*40 + U40) so the GROUP BY
perfect hash never folds groups (src/core/visitor.cpp:2056-2127).
"""
from __future__ import annotations

import datetime as _dt
from dataclasses import dataclass

import numpy as np

from .plan import Table

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
DATE_DAYS = 2556  # 1992-01-01 .. 1998-12-30

# Generator stream of every synthetic column (stable ids).
STREAMS = {
    "lo_orderdate": 1, "lo_custkey": 2, "lo_suppkey": 3, "lo_partkey": 4, "lo_quantity": 5,
    "lo_discount": 6, "lo_extendedprice": 7, "lo_revenue": 8, "lo_supplycost": 9, "lo_commitdate": 10,
    "c_region": 20, "c_nation": 21, "c_city": 22,
    "s_region": 30, "s_nation": 31, "s_city": 32,
    "p_mfgr": 40, "p_category": 41, "p_brand1": 42,
    "ps_partkey": 50, "ps_tier": 51, "ps_availqty": 52, "ps_supplycost": 53,
    "valid_lo_revenue": 100, "valid_c_city": 101, "valid_lo_quantity": 102, "valid_lo_discount": 103,
    "valid_ps_tier": 104, "valid_lo_commitdate": 105, "valid_c_nation": 106,
}

# Uniform fact columns: (lo, hi) inclusive.
FACT_UNIFORM = {
    "lo_quantity": (1, 50),
    "lo_discount": (0, 10),
    "lo_extendedprice": (90_000, 10_500_000),
    "lo_revenue": (100, 10_000_000),
    "lo_supplycost": (100, 10_000_000),
}

DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "PART": 200_000, "DDATE": DATE_DAYS, "PARTSUPP": 400_000}
COMMIT_LAG_DAYS = 91  # lo_commitdate = lo_orderdate + 0..90 days (may run past the date table)


def _splitmix64(z: np.ndarray) -> np.ndarray:
    z = z + np.uint64(GOLDEN)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _splitmix64_int(z: int) -> int:
    z = (z + GOLDEN) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def stream_key(seed: int, stream: int) -> int:
    return _splitmix64_int((seed & M64) ^ _splitmix64_int((stream * 0xD6E8FEB86659FD93 + 1) & M64))


def hashes(seed: int, stream: int, row0: int, rows: int) -> np.ndarray:
    key = np.uint64(stream_key(seed, stream))
    r = np.arange(row0, row0 + rows, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _splitmix64(key + r * np.uint64(GOLDEN))


def below(h: np.ndarray, n: int) -> np.ndarray:
    return ((h >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)


def uniform(seed: int, stream: int, lo: int, hi: int, row0: int, rows: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        return (np.int64(lo) + below(hashes(seed, stream, row0, rows), hi - lo + 1).astype(np.int64)).astype(np.int32)


_DATES = [(_dt.date(1992, 1, 1) + _dt.timedelta(days=d)) for d in range(DATE_DAYS)]
DATE_KEYS = np.array([d.year * 10000 + d.month * 100 + d.day for d in _DATES], dtype=np.int32)


def datekeys(seed: int, stream: int, row0: int, rows: int) -> np.ndarray:
    idx = below(hashes(seed, stream, row0, rows), DATE_DAYS).astype(np.int64)
    return DATE_KEYS[idx]


_EXT_DATES = [(_dt.date(1992, 1, 1) + _dt.timedelta(days=d)) for d in range(DATE_DAYS + COMMIT_LAG_DAYS)]
EXT_DATE_KEYS = np.array([d.year * 10000 + d.month * 100 + d.day for d in _EXT_DATES], dtype=np.int32)


def commitdates(seed: int, row0: int, rows: int) -> np.ndarray:
    """lo_commitdate: the row's order date plus 0..90 days, so about one row
    in 91 commits on its order date and the last 90 days of orders commit past
    the date dimension."""
    idx = below(hashes(seed, STREAMS["lo_orderdate"], row0, rows), DATE_DAYS).astype(np.int64)
    lag = below(hashes(seed, STREAMS["lo_commitdate"], row0, rows), COMMIT_LAG_DAYS).astype(np.int64)
    return EXT_DATE_KEYS[idx + lag]


def validity_words(seed: int, stream: int, rows: int, null_permille: int, row0: int = 0) -> np.ndarray:
    """uint64 words, bit r = 1 when row row0 + r is valid (the reference's
    .valid64); row0 > 0 gives the words of a row range on their own."""
    nulls = below(hashes(seed, stream, row0, rows), 1000) < np.uint64(null_permille)
    bits = np.zeros(((rows + 63) // 64) * 64, dtype=np.uint8)
    bits[:rows] = ~nulls
    return np.packbits(bits, bitorder="little").view("<u8").astype(np.uint64)


def fact_column(name: str, seed: int, row0: int, rows: int) -> np.ndarray:
    s = STREAMS[name]
    if name == "lo_orderdate":
        return datekeys(seed, s, row0, rows)
    if name == "lo_commitdate":
        return commitdates(seed, row0, rows)
    if name == "lo_custkey":
        return uniform(seed, s, 1, DIM_ROWS["CUSTOMER"], row0, rows)
    if name == "lo_suppkey":
        return uniform(seed, s, 1, DIM_ROWS["SUPPLIER"], row0, rows)
    if name == "lo_partkey":
        return uniform(seed, s, 1, DIM_ROWS["PART"], row0, rows)
    lo, hi = FACT_UNIFORM[name]
    return uniform(seed, s, lo, hi, row0, rows)


def fact_column_device(name: str, seed: int, rows: int, out_ptr: int, stream: int = 0, row0: int = 0) -> None:
    """Fills a device int32 buffer with the same values fact_column returns."""
    from ._lib import check, lib

    s = STREAMS[name]
    if name == "lo_commitdate":
        raise ValueError("lo_commitdate has no device generator; load fact_column() output")
    if name == "lo_orderdate":
        check(lib.cx_gen_datekey(s, seed, DATE_DAYS, row0, rows, out_ptr, stream or None), "cx_gen_datekey")
        return
    if name in ("lo_custkey", "lo_suppkey", "lo_partkey"):
        lo, hi = 1, DIM_ROWS[{"lo_custkey": "CUSTOMER", "lo_suppkey": "SUPPLIER", "lo_partkey": "PART"}[name]]
    else:
        lo, hi = FACT_UNIFORM[name]
    check(lib.cx_gen_uniform(s, seed, lo, hi, row0, rows, out_ptr, stream or None), "cx_gen_uniform")


def validity_device(name: str, seed: int, rows: int, permille: int, out_ptr: int, stream: int = 0) -> None:
    from ._lib import check, lib

    check(lib.cx_gen_validity(STREAMS["valid_" + name], seed, rows, permille, out_ptr, stream or None),
          "cx_gen_validity")


# ------------------------------------------------------------- dimensions


def dim_columns(table: str, seed: int) -> dict[str, np.ndarray]:
    n = DIM_ROWS[table]
    if table == "DDATE":
        return {
            "d_datekey": DATE_KEYS.copy(),
            "d_year": np.array([d.year for d in _DATES], dtype=np.int32),
            "d_month": np.array([d.month for d in _DATES], dtype=np.int32),
            "d_weeknum": np.array([(d.timetuple().tm_yday - 1) // 7 + 1 for d in _DATES], dtype=np.int32),
        }
    if table == "PARTSUPP":
        # Non-unique key: part keys drawn with replacement (0..several rows per
        # part, about 13.5% of parts have none).
        return {
            "ps_partkey": uniform(seed, STREAMS["ps_partkey"], 1, DIM_ROWS["PART"], 0, n),
            "ps_tier": uniform(seed, STREAMS["ps_tier"], 0, 4, 0, n),
            "ps_availqty": uniform(seed, STREAMS["ps_availqty"], 1, 9999, 0, n),
            "ps_supplycost": uniform(seed, STREAMS["ps_supplycost"], 1, 1000, 0, n),
        }
    p = {"CUSTOMER": "c", "SUPPLIER": "s", "PART": "p"}[table]
    key = np.arange(1, n + 1, dtype=np.int32)
    if table == "PART":
        mfgr = uniform(seed, STREAMS["p_mfgr"], 0, 4, 0, n)
        cat = mfgr * 5 + uniform(seed, STREAMS["p_category"], 0, 4, 0, n)
        brand = cat * 40 + uniform(seed, STREAMS["p_brand1"], 0, 39, 0, n)
        return {"p_partkey": key, "p_mfgr": mfgr, "p_category": cat, "p_brand1": brand}
    region = uniform(seed, STREAMS[f"{p}_region"], 0, 4, 0, n)
    nation = region * 5 + uniform(seed, STREAMS[f"{p}_nation"], 0, 4, 0, n)
    city = nation * 10 + uniform(seed, STREAMS[f"{p}_city"], 0, 9, 0, n)
    return {f"{p}_{'custkey' if p == 'c' else 'suppkey'}": key, f"{p}_region": region, f"{p}_nation": nation,
            f"{p}_city": city}


FACT_COLS = ["lo_orderdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_quantity", "lo_discount",
             "lo_extendedprice", "lo_revenue", "lo_supplycost"]


def ssb_tables(fact_rows: int, fact_cols: list[str] | None = None) -> dict[str, Table]:
    """Catalog entries (Table) of the synthetic SSB schema."""
    tables = _ssb_tables(fact_rows, fact_cols)
    for t in tables.values():
        t.stats = {c: GROUP_STATS[c] for c in t.cols if c in GROUP_STATS}
    return tables


def _ssb_tables(fact_rows: int, fact_cols: list[str] | None) -> dict[str, Table]:
    return {
        "LINEORDER": Table("LINEORDER", list(fact_cols or FACT_COLS), fact_rows, fact=True),
        "DDATE": Table("DDATE", ["d_datekey", "d_year", "d_month", "d_weeknum"], DATE_DAYS, key_col="d_datekey",
                       key_min=int(DATE_KEYS[0]), key_max=int(DATE_KEYS[-1])),
        "CUSTOMER": Table("CUSTOMER", ["c_custkey", "c_region", "c_nation", "c_city"], DIM_ROWS["CUSTOMER"],
                          key_col="c_custkey", key_min=1, key_max=DIM_ROWS["CUSTOMER"]),
        "SUPPLIER": Table("SUPPLIER", ["s_suppkey", "s_region", "s_nation", "s_city"], DIM_ROWS["SUPPLIER"],
                          key_col="s_suppkey", key_min=1, key_max=DIM_ROWS["SUPPLIER"]),
        "PART": Table("PART", ["p_partkey", "p_mfgr", "p_category", "p_brand1"], DIM_ROWS["PART"],
                      key_col="p_partkey", key_min=1, key_max=DIM_ROWS["PART"]),
        "PARTSUPP": Table("PARTSUPP", ["ps_partkey", "ps_tier", "ps_availqty", "ps_supplycost"],
                          DIM_ROWS["PARTSUPP"], key_col="ps_partkey", key_min=1, key_max=DIM_ROWS["PART"],
                          key_unique=False),
    }


# Catalog statistics of the group-by columns: (min, cardinality).
GROUP_STATS = {
    "d_year": (1992, 7), "d_month": (1, 12), "d_weeknum": (1, 53),
    "c_region": (0, 5), "c_nation": (0, 25), "c_city": (0, 250),
    "s_region": (0, 5), "s_nation": (0, 25), "s_city": (0, 250),
    "p_mfgr": (0, 5), "p_category": (0, 25), "p_brand1": (0, 1000),
    "lo_quantity": (1, 50), "lo_discount": (0, 11),
    "ps_tier": (0, 5),
}


def dim_of_column(c: str) -> str:
    if c.startswith("ps_"):
        return "PARTSUPP"
    return {"c": "CUSTOMER", "s": "SUPPLIER", "p": "PART", "d": "DDATE"}[c[0]]


@dataclass
class HostTables:
    """Host copies of a generated schema (used by the oracle and small tests)."""

    seed: int
    fact_rows: int
    columns: dict[str, np.ndarray]
    validity: dict[str, np.ndarray]


def host_tables(seed: int, fact_rows: int, fact_cols: list[str], nulls: dict[str, int] | None = None,
                dims: tuple[str, ...] = ("DDATE", "CUSTOMER", "SUPPLIER", "PART")) -> HostTables:
    cols: dict[str, np.ndarray] = {}
    for c in fact_cols:
        cols[c] = fact_column(c, seed, 0, fact_rows)
    for d in dims:
        cols.update(dim_columns(d, seed))
    validity: dict[str, np.ndarray] = {}
    for c, permille in (nulls or {}).items():
        rows = fact_rows if c.startswith("lo_") else DIM_ROWS[dim_of_column(c)]
        validity[c] = validity_words(seed, STREAMS["valid_" + c], rows, permille)
    return HostTables(seed, fact_rows, cols, validity)
