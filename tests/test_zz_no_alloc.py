"""The allocation-free compaction entry point (cx_compact_sparse_noalloc).

It serves callers that cannot let the library allocate device memory, such as
a serving loop that has reserved all of HBM for admitted queries.  Through the
C ABI, its output must equal cx_compact_sparse's, bit for bit (integer data),
on two calls in a row: the shared fixed scratch array keeps the previous
call's contents, and that must not leak into the next result.  This file is
collected last so a run that stops at the first failure has already run every
other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from practice_b200 import _lib

pytestmark = pytest.mark.gpu


def _compact(fn, torch, src, groups, ts):
    dst = torch.zeros_like(src)
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    _lib.check(fn(src.data_ptr(), groups, ts, dst.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    k = int(cnt.item())
    return k, dst.cpu().numpy()[: k * ts]


def test_noalloc_compaction_matches_allocating_entry_point_twice():
    import torch
    rng = np.random.default_rng(7)
    calls = []
    # Two different inputs in a row: the second call must not see the first's counts.
    for groups, ts, density in ((1_000_003, 3, 0.05), (70_001, 2, 0.5)):
        host = np.zeros(groups * ts, dtype=np.int64)
        present = rng.random(groups) < density
        vals = rng.integers(1, 1 << 40, size=groups * ts)
        host[np.repeat(present, ts)] = vals[np.repeat(present, ts)]
        src = torch.from_numpy(host).cuda()
        ref = _compact(_lib.lib.cx_compact_sparse, torch, src, groups, ts)
        got = _compact(_lib.lib.cx_compact_sparse_noalloc, torch, src, groups, ts)
        assert got[0] == ref[0] == int(present.sum())
        np.testing.assert_array_equal(got[1], ref[1])
        calls.append(got[0])
    assert calls[0] != calls[1]


def test_noalloc_compaction_rejects_oversized_input():
    import torch
    src = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = _lib.lib.cx_compact_sparse_noalloc(src.data_ptr(), 16384 * 2048 + 1, 1, src.data_ptr(), src.data_ptr(), None)
    assert rc == -5  # CX_E_CAPACITY, before any device work
