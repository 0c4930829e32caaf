"""Bounded waits on the GPU: a wait that runs out returns an error status.

Every wait of a generated kernel on an mbarrier gives up after
`cx_tuning.wait_limit_us` microseconds and raises kernel error 1, which the
host reads as CX_E_KERNEL from cx_ctx_sync.  `cx_tuning.debug_stall` makes each
CTA wait first on a barrier that nothing completes (no copy in flight), so the
wait runs out for certain.  The tests check the status, that it comes back
within a short time, and that the context answers the same query correctly
afterwards.  No GPU fault, trap or hang is involved."""
import time

import numpy as np
import pytest

import oracle
from practice_b200 import _lib, datagen, queries
from practice_b200.engine import make_tuning

pytestmark = pytest.mark.gpu

DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}
LIMIT_US = 20_000


@pytest.fixture(scope="module")
def loaded():
    from practice_b200.engine import Database
    n = 100_003
    ht = datagen.host_tables(21, n, queries.BATCH_COLS)
    db = Database(0)
    db.load_host_tables(ht, datagen.ssb_tables(n, queries.BATCH_COLS))
    return db, ht, n


def _ref(plan, ht):
    rows = {"LINEORDER": ht.fact_rows, **DIM_ROWS}
    return oracle.run_plan(plan.text(), ht.columns, ht.validity, rows, plan.group_slots * plan.storage_ts)


@pytest.mark.parametrize("stages", [0, 3])
def test_plain_scan_wait_runs_out_and_context_recovers(loaded, stages):
    db, ht, n = loaded
    plan = queries.ssb_q31(n)
    stall = make_tuning(block_threads=256, items_per_thread=4, stages=stages, ctas_per_sm=2,
                        wait_limit_us=LIMIT_US, debug_stall=1)
    t0 = time.perf_counter()
    got = db.execute(plan, stall)
    elapsed = time.perf_counter() - t0
    assert got.kernel_error == 1, "the wait that ran out must raise kernel error 1"
    assert elapsed < 30.0  # includes the NVRTC compile; the wait itself is 20 ms
    # The same context answers correctly afterwards, at the stalled launch shape without the hook.
    ok = db.execute(plan, make_tuning(block_threads=256, items_per_thread=4, stages=stages, ctas_per_sm=2))
    assert ok.kernel_error == 0
    np.testing.assert_array_equal(ok.words, _ref(plan, ht).words[: len(ok.words)])


def test_kernel_error_is_reported_through_the_c_abi(loaded):
    db, _, n = loaded
    plan = queries.template(0, __import__("random").Random(4), n)
    m = db.compile(plan, make_tuning(wait_limit_us=LIMIT_US, debug_stall=1))
    res, val = db.alloc_result(m)
    for t, r in db.rows.items():
        db.ctx.set_rows(t, r)
    db.ctx.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
    db.ctx.execute(m, db.torch.cuda.current_stream().cuda_stream)
    with pytest.raises(_lib.CxError) as e:
        db.ctx.sync()
    assert e.value.code == -6  # CX_E_KERNEL
    assert db.ctx.kernel_error() == 1


def test_shared_scan_wait_runs_out_and_context_recovers(loaded):
    db, ht, n = loaded
    import random
    plans = [queries.template(t, random.Random(300 + t), n) for t in range(4)]
    stall = make_tuning(block_threads=1024, items_per_thread=1, stages=3, ctas_per_sm=1,
                        wait_limit_us=LIMIT_US, debug_stall=1, cube=0)  # the per-query path waits on mbarriers
    got = db.execute_shared(plans, stall)
    assert all(g.kernel_error == 1 for g in got)
    good = db.execute_shared(plans, make_tuning(block_threads=1024, items_per_thread=1, stages=3, ctas_per_sm=1, cube=0))
    for p, g in zip(plans, good):
        assert g.kernel_error == 0
        np.testing.assert_array_equal(g.words, _ref(p, ht).words[: len(g.words)])

