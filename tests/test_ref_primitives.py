"""The reference's own crystal primitives, compiled for the host by
`make -C oracle ref` (oracle/_ref), against the oracle restatement: the two
must agree bit-exactly on every supported query shape.  Skipped where the
reference sources were not available to build oracle/_ref."""
import random

import numpy as np
import pytest

import oracle
from oracle import refharness
from practice_b200 import datagen, queries

pytestmark = pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built (reference absent)")

DIMS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}


@pytest.fixture(scope="module")
def tables():
    n = 200_003
    return n, datagen.host_tables(21, n, queries.BATCH_COLS + ["lo_extendedprice"])


@pytest.mark.parametrize("t", [0, 1, 2, 3])
def test_templates_match_reference_primitives(tables, t):
    n, ht = tables
    rng = random.Random(50 + t)
    for _ in range(4):
        p = queries.template(t, rng, n)
        ref = refharness.run(p, ht.columns, DIMS, n)
        got = oracle.run_plan(p.text(), ht.columns, ht.validity, {"LINEORDER": n, **DIMS}, p.group_slots * p.storage_ts)
        np.testing.assert_array_equal(ref, got.words)


def test_q11_and_q31_match_reference_primitives(tables):
    n, ht = tables
    for p in (queries.ssb_q11(n), queries.ssb_q31(n, region=4)):
        ref = refharness.run(p, ht.columns, DIMS, n)
        got = oracle.run_plan(p.text(), ht.columns, ht.validity, {"LINEORDER": n, **DIMS}, p.group_slots * p.storage_ts)
        np.testing.assert_array_equal(ref, got.words)


@pytest.fixture(scope="module")
def expand_tables():
    n = 150_001
    cols = sorted(set(queries.OR_COLS + queries.MHT_COLS))
    return n, datagen.host_tables(22, n, cols, dims=("DDATE", "SUPPLIER", "PART", "PARTSUPP"))


@pytest.mark.parametrize("make", [lambda n: queries.or_join_year(n), lambda n: queries.or_join_year(n, (1994, 1998)),
                                  lambda n: queries.mht_year_tier(n), lambda n: queries.mht_year_tier(n, 300)])
def test_or_joins_and_mht_match_reference_primitives(expand_tables, make):
    """OR-join (two fact keys, duplicate keys skipped) and MHT row expansion:
    the oracle against the reference's own BlockBuildMHT_Count/Write,
    ProbeMultiHT and vector OR-join probes."""
    n, ht = expand_tables
    dims = {**DIMS, "PARTSUPP": datagen.DIM_ROWS["PARTSUPP"]}
    p = make(n)
    ref = refharness.run(p, ht.columns, dims, n)
    got = oracle.run_plan(p.text(), ht.columns, ht.validity, {"LINEORDER": n, **dims}, p.group_slots * p.storage_ts)
    np.testing.assert_array_equal(ref, got.words)
    assert ref.any()
