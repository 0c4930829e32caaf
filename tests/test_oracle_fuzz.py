"""Seeded random plans: the oracle restatement against the reference's own
crystal primitives (oracle/_ref) on shapes beyond the fixed workloads --
random fact filters, one to three joins in random order with and without
dimension filters, an OR over two date keys or a multi-value PARTSUPP join,
GROUP BY over payloads or fact columns, COUNT(*) and SUMs.  Bit-exact on every
aggregate word."""
import random

import numpy as np
import pytest

import oracle
from oracle import refharness
from practice_b200 import datagen

from randplans import FACT_COLS, harness_plan

pytestmark = pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built (reference absent)")

N = 60_013


@pytest.fixture(scope="module")
def tables():
    return datagen.host_tables(77, N, FACT_COLS, dims=("DDATE", "CUSTOMER", "SUPPLIER", "PART", "PARTSUPP"))


@pytest.mark.parametrize("seed", range(40))
def test_random_plan_matches_reference_primitives(tables, seed):
    plan = harness_plan(random.Random(seed), N, name=f"fuzz{seed}")
    dims = dict(datagen.DIM_ROWS)
    ref = refharness.run(plan, tables.columns, dims, N)
    got = oracle.run_plan(plan.text(), tables.columns, tables.validity, {"LINEORDER": N, **dims},
                          plan.group_slots * plan.storage_ts)
    np.testing.assert_array_equal(ref, got.words, err_msg=plan.text())
