"""The allocation-free sort entry point (gpulsm_sort_pairs_noalloc).

Some callers may not allocate device memory at all - a process whose device
memory is owned by another allocator under a fixed budget, or a latency-
critical path that cannot risk an allocator call.  This entry point sorts
with a static device scratch array instead; its answers must equal those of
the allocating entry point (gpulsm_sort_pairs) exactly, call after call,
since every call reuses the same scratch.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test; it also passes when run alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    a = np.ascontiguousarray(a)
    view = np.int64 if a.dtype == np.uint64 else np.int32
    return torch.from_numpy(a.view(view)).cuda()


def _sort(lib, N, fn, k, v, bits, begin, end):
    import torch

    ko = torch.empty_like(k)
    vo = torch.empty_like(v) if v is not None else None
    N.check(fn(k.data_ptr(), v.data_ptr() if v is not None else None, ko.data_ptr(),
               vo.data_ptr() if vo is not None else None, k.numel(), bits, begin, end, None))
    torch.cuda.synchronize()
    return ko, vo


@pytest.mark.parametrize("bits,n,with_values", [(32, 1 << 20, True), (64, 300_001, True), (32, 77_777, False)])
def test_noalloc_sort_matches_allocating_sort_twice(gl, cuda, bits, n, with_values):
    import torch

    lib = gl.load()
    N = gl._native
    rng = np.random.default_rng(bits + n)
    end = 32 if bits == 32 else 44
    for call in range(2):  # two calls in a row: the shared scratch keeps the previous call's contents
        hi = 1 << (12 if call == 0 else end)  # many ties on the first call
        k = rng.integers(0, hi, n, dtype=np.uint64)
        k = k.astype(np.uint32) if bits == 32 else k
        kd = _dev(k)
        vd = _dev(np.arange(n, dtype=np.uint32) * 3 + call) if with_values else None
        ref_k, ref_v = _sort(lib, N, lib.gpulsm_sort_pairs, kd, vd, bits, 0, end)
        got_k, got_v = _sort(lib, N, lib.gpulsm_sort_pairs_noalloc, kd, vd, bits, 0, end)
        assert torch.equal(got_k, ref_k), f"keys differ on call {call}"
        if with_values:
            assert torch.equal(got_v, ref_v), f"values differ on call {call}"
        order = np.argsort(k, kind="stable")
        assert np.array_equal(got_k.cpu().numpy().view(k.dtype), k[order])


def test_noalloc_sort_rejects_counts_beyond_its_scratch(gl, cuda):
    import torch

    lib = gl.load()
    N = gl._native
    assert lib.gpulsm_sort_noalloc_scratch_bytes() > 0
    k = torch.zeros(8, dtype=torch.int32, device="cuda")
    # the count is checked before any pointer is dereferenced or work is enqueued
    with pytest.raises(gl.LengthError, match="at most"):
        N.check(lib.gpulsm_sort_pairs_noalloc(k.data_ptr(), None, k.data_ptr(), None, (1 << 20) + 1, 32, 0, 32,
                                              None))


@pytest.mark.parametrize("bits", [32, 64])
def test_noalloc_sort_partial_digit_range_and_in_place(gl, cuda, bits):
    """A bit range that is not a whole number of 8-bit digits ([3, 13) here) on
    full-width keys: both entries order by those 10 bits only, stably, like a
    stable argsort of (key >> 3) & 0x3ff; then the same sort in place (input
    buffers passed as outputs) gives the same result."""
    import torch

    lib = gl.load()
    N = gl._native
    rng = np.random.default_rng(bits)
    n = 200_003
    k = rng.integers(0, 1 << bits, n, dtype=np.uint64)
    k = k.astype(np.uint32) if bits == 32 else k
    v = np.arange(n, dtype=np.uint32)
    order = np.argsort((k >> k.dtype.type(3)) & k.dtype.type(0x3FF), kind="stable")
    for fn in (lib.gpulsm_sort_pairs, lib.gpulsm_sort_pairs_noalloc):
        for call in range(2):
            got_k, got_v = _sort(lib, N, fn, _dev(k), _dev(v), bits, 3, 13)
            assert np.array_equal(got_k.cpu().numpy().view(k.dtype), k[order]), f"{fn.__name__} call {call}"
            assert np.array_equal(got_v.cpu().numpy().view(np.uint32), v[order]), f"{fn.__name__} call {call}"
        kd, vd = _dev(k), _dev(v)
        N.check(fn(kd.data_ptr(), vd.data_ptr(), kd.data_ptr(), vd.data_ptr(), n, bits, 3, 13, None))
        torch.cuda.synchronize()
        assert np.array_equal(kd.cpu().numpy().view(k.dtype), k[order]), f"{fn.__name__} in place"
        assert np.array_equal(vd.cpu().numpy().view(np.uint32), v[order]), f"{fn.__name__} in place"
