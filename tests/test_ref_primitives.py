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
