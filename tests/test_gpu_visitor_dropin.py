"""The reference's own code generator's programs on the GPU, bit-exact.

Each tests/golden/visitor/*.sycl program -- the SYCL text
JITOperatorVisitor::generateCode emits for the SSB Q1.1 and Q3.1 shapes and the
four batch templates -- is handed unchanged to cx_compile, run by cx_execute
over device-resident tables through an execution context bound by name, and
its raw result buffer compared word for word with the oracle evaluating the
same query (tests/visitor_plans.py).  The tables have the measured workloads'
sizes: 6,000,000 fact rows for Q1.1, 60,000,000 for the others."""
import os

import numpy as np
import pytest

from oracle import chunked
from practice_b200 import _lib, datagen

from visitor_plans import ALL_COLS, TRANSLATED, plan

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(__file__), "golden", "visitor")
DIM_ROWS = {"CUSTOMER": 300_000, "SUPPLIER": 20_000, "DDATE": 2556, "PART": 200_000}
SEED = 31


@pytest.fixture(scope="module")
def tables():
    from practice_b200.engine import Database
    out = {}
    for n in (6_000_000, 60_000_000):
        db = Database(0)
        db.generate_ssb(n, SEED, ALL_COLS)
        out[n] = db
    yield out
    for db in out.values():
        db.reset()


def run_visitor_program(db, name):
    src = open(os.path.join(FIX, f"{name}.sycl")).read()
    m = _lib.Module(src, key=f"gpu_visitor_{name}")
    res, val = db.alloc_result(m)
    c = _lib.ExecCtx()
    for col, t in db.cols.items():
        c.set_buffer("d_" + col, t.data_ptr(), t.numel())
    for t, n in db.rows.items():
        c.set_rows(t, n)
    c.set_result(res.data_ptr(), res.numel(), val.data_ptr(), val.numel())
    c.execute(m, db.torch.cuda.current_stream().cuda_stream)
    c.sync()
    timing = c.timing()
    c.close()
    fw = int(m.info.final_words)
    words = res.cpu().numpy().view(np.uint64)[:fw]
    validity = val.cpu().numpy().view(np.uint64)[: (fw + 63) // 64]
    return words, validity, timing


@pytest.mark.parametrize("name", TRANSLATED)
def test_reference_generated_program_is_bit_exact(tables, name):
    n = 6_000_000 if name == "q11" else 60_000_000
    db = tables[n]
    words, validity, timing = run_visitor_program(db, name)
    p = plan(name, n)
    dims = {}
    for t in ("DDATE", "CUSTOMER", "SUPPLIER", "PART"):
        dims.update(datagen.dim_columns(t, SEED))
    cols = [c for t in p.tables if t.fact for c in t.cols]  # the oracle binds every column the plan's table lists
    (acc,), _, _ = chunked.run_oracle([p], chunked.host_fetch(SEED, cols), n, dims, {}, DIM_ROWS,
                                      chunk_rows=10_000_000, threads=os.cpu_count())
    np.testing.assert_array_equal(words, acc.words[: len(words)])
    np.testing.assert_array_equal(validity, acc.validity[: len(validity)])
    assert np.any(words != 0)
    assert timing.gpu_launches >= 1 and timing.scan_ms > 0
