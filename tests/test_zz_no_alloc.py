"""The allocation-free compaction entry point (cx_compact_sparse_noalloc).

It serves callers that cannot let the library allocate device memory, such as
a serving loop that has reserved all of HBM for admitted queries.  Through the
C ABI, its output must equal cx_compact_sparse's, bit for bit (integer data),
on two calls in a row: the shared fixed scratch array keeps the previous
call's contents, and that must not leak into the next result.  The sizes run
from a few blocks of groups up to the documented maximum of 33,554,432 groups,
past the 1,024-block chunk of the one-CTA prefix scan.  The device's default
memory pool, which the allocating entry point draws on, must show no new use
across the allocation-free calls.  This file is collected last so a run that
stops at the first failure has already run every other test; it also passes
alone in a fresh process."""
import numpy as np
import pytest

from practice_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_GROUPS = 16384 * 2048  # the fixed scratch array's limit


def _compact(fn, torch, src, groups, ts):
    dst = torch.zeros_like(src)
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(fn(src.data_ptr(), groups, ts, dst.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    k = int(cnt.item())
    return k, dst[: k * ts].cpu().numpy()


def _source(torch, groups, ts, density, seed):
    """Group tuples on the device, a fraction `density` of them present."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    present = torch.rand(groups, generator=g, device="cuda") < density
    vals = torch.randint(1, 1 << 40, (groups, ts), generator=g, device="cuda", dtype=torch.int64)
    src = (vals * present.unsqueeze(1)).reshape(-1).contiguous()
    return src, int(present.sum().item())


class _Pool:
    """High-water marks of the current device's default memory pool."""

    def __init__(self):
        import torch
        from cuda.bindings import driver, runtime as rt

        self.rt = rt
        self.u64 = driver.cuuint64_t
        err, self.pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
        assert err == rt.cudaError_t.cudaSuccess

    def _attr(self, a):
        err, v = self.rt.cudaMemPoolGetAttribute(self.pool, a)
        assert err == self.rt.cudaError_t.cudaSuccess
        return int(v)

    def reset(self):
        A = self.rt.cudaMemPoolAttr
        for a in (A.cudaMemPoolAttrUsedMemHigh, A.cudaMemPoolAttrReservedMemHigh):
            (err,) = self.rt.cudaMemPoolSetAttribute(self.pool, a, self.u64(0))
            assert err == self.rt.cudaError_t.cudaSuccess

    def highs(self):
        A = self.rt.cudaMemPoolAttr
        return self._attr(A.cudaMemPoolAttrUsedMemHigh), self._attr(A.cudaMemPoolAttrReservedMemHigh)

    def used(self):
        return self._attr(self.rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)


@pytest.mark.parametrize("cases", [
    # Two different inputs in a row: the second call must not see the first's counts.
    ((1_000_003, 3, 0.05, 1), (70_001, 2, 0.5, 2)),
    # Just past one 1,024-block chunk of the prefix scan, then the maximum.
    ((2_097_153, 2, 0.3, 3), (MAX_GROUPS, 1, 0.01, 4)),
], ids=["small", "multi_chunk_and_maximum"])
def test_noalloc_compaction_matches_allocating_entry_point_twice(cases):
    import torch
    pool = _Pool()
    counts = []
    for groups, ts, density, seed in cases:
        src, present = _source(torch, groups, ts, density, seed)
        pool.reset()
        used0 = pool.used()
        ref = _compact(_lib.lib.cx_compact_sparse, torch, src, groups, ts)
        # Positive control: the allocating entry point's scratch shows up in the pool.
        assert pool.highs()[0] > used0
        pool.reset()
        highs = pool.highs()
        got = _compact(_lib.lib.cx_compact_sparse_noalloc, torch, src, groups, ts)
        assert pool.highs() == highs, "the allocation-free entry point drew on the memory pool"
        assert got[0] == ref[0] == present
        np.testing.assert_array_equal(got[1], ref[1])
        counts.append(got[0])
        del src
    assert counts[0] != counts[1]


def test_noalloc_compaction_rejects_oversized_input():
    import torch
    src = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = _lib.lib.cx_compact_sparse_noalloc(src.data_ptr(), MAX_GROUPS + 1, 1, src.data_ptr(), src.data_ptr(), None)
    assert rc == -5  # CX_E_CAPACITY, before any device work
    assert f"{MAX_GROUPS}" in _lib.lib.cx_last_error().decode()
