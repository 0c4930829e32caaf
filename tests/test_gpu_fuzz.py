"""Seeded random plans through the CUDA path (C ABI) against the oracle, bit-
exact on every word of the raw aggregate buffer and its validity bitmap:
nullable fact and payload columns under three-valued logic, OR / NOT / IS NULL
filters, filters on join payloads, MIN / MAX / AVG / COUNT(column) / CASE
aggregates, one to three joins in random order, an OR over two date keys or a
multi-value PARTSUPP join -- at the default launch shape, at a TMA-staged
one and with warp-compacted rows (two tile shapes); random batches of shareable plans through one shared scan; and a random
mix through the request loop."""
import random

import numpy as np
import pytest

import oracle
from practice_b200 import _lib, datagen
from practice_b200.engine import make_tuning

from randplans import FACT_COLS, engine_plan, harness_plan

pytestmark = pytest.mark.gpu

N = 400_003
NULLABLE = ("lo_revenue", "c_nation")
TUNINGS = {"default": None, "tma": dict(block_threads=256, items_per_thread=4, stages=3, ctas_per_sm=2),
           "compact": dict(compact=1), "compact_ipt2": dict(block_threads=512, items_per_thread=2, compact=1),
           "compact_drain64": dict(compact=2)}


@pytest.fixture(scope="module")
def loaded():
    from practice_b200.engine import Database
    ht = datagen.host_tables(91, N, FACT_COLS, nulls={"lo_revenue": 80, "c_nation": 50},
                             dims=("DDATE", "CUSTOMER", "SUPPLIER", "PART", "PARTSUPP"))
    db = Database(0)
    db.load_host_tables(ht, datagen.ssb_tables(N, FACT_COLS))
    return db, ht


@pytest.mark.parametrize("shape", list(TUNINGS))
@pytest.mark.parametrize("seed", range(24))
def test_random_plan_matches_oracle(loaded, seed, shape):
    db, ht = loaded
    plan = engine_plan(random.Random(seed), N, NULLABLE, name=f"fuzz{seed}")
    ref = oracle.run_plan(plan.text(), ht.columns, ht.validity, {"LINEORDER": N, **datagen.DIM_ROWS},
                          plan.group_slots * plan.storage_ts)
    t = make_tuning(**TUNINGS[shape]) if TUNINGS[shape] else None
    got = db.execute(plan, t)
    assert got.kernel_error == 0, plan.text()
    fw = len(got.words)
    np.testing.assert_array_equal(got.words, ref.words[:fw], err_msg=plan.text())
    np.testing.assert_array_equal(got.validity, ref.validity[: (fw + 63) // 64], err_msg=plan.text())


@pytest.mark.parametrize("batch", range(6))
def test_random_shared_batch_matches_oracle_per_query(loaded, batch):
    """Eight random shareable plans (eight distinct shapes) answered by ONE
    shared scan: every query equals the oracle run on that query alone."""
    db, ht = loaded
    rng = random.Random(1000 + batch)
    plans = [harness_plan(rng, N, name=f"shared{batch}_{i}", expanding_ok=False) for i in range(8)]
    assert all(db.shareable(p) for p in plans)
    got = db.execute_shared(plans)
    assert got[0].kernel_error == 0
    for p, g in zip(plans, got):
        ref = oracle.run_plan(p.text(), ht.columns, ht.validity, {"LINEORDER": N, **datagen.DIM_ROWS},
                              p.group_slots * p.storage_ts)
        np.testing.assert_array_equal(g.words, ref.words, err_msg=p.text())
        np.testing.assert_array_equal(g.validity, ref.validity, err_msg=p.text())


def test_random_mix_through_the_request_loop(loaded):
    """Random shareable plans mixed with random plans the shared scan does not
    take (nullable columns, AVG / MIN / MAX, OR-joins, multi-value joins),
    submitted back to back to the request loop: every result equals the
    oracle's, whether it ran in a shared launch or alone."""
    db, ht = loaded
    rng = random.Random(777)
    plans = [harness_plan(rng, N, name=f"mix_h{i}", expanding_ok=False) for i in range(12)]
    plans += [engine_plan(rng, N, NULLABLE, name=f"mix_e{i}") for i in range(8)]
    rng.shuffle(plans)
    srv = _lib.Server(db.ctx, _lib.server_config(max_batch=16, slots=1, min_shared_batch=2))
    try:
        ids = [srv.submit(p.text()) for p in plans]
        for rid, p in zip(ids, plans):
            info = srv.wait(rid, 120_000)
            assert info.status == 0 and info.kernel_error == 0, (p.name, info.status, info.kernel_error)
            w, v = srv.fetch(rid, info)
            ref = oracle.run_plan(p.text(), ht.columns, ht.validity, {"LINEORDER": N, **datagen.DIM_ROWS},
                                  p.group_slots * p.storage_ts)
            np.testing.assert_array_equal(w, ref.words[: len(w)], err_msg=p.text())
            np.testing.assert_array_equal(v, ref.validity[: len(v)], err_msg=p.text())
            srv.release(rid)
        st = srv.stats()
        assert st.completed == len(plans) and st.rejected == 0
    finally:
        srv.close()
