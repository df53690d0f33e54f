"""FliX's own GPULSMOpt adapter (FliX/impl_gpulsmopt.cuh:137-311), built over
include/gpulsmopt_b200.cuh and libgpulsm.so (oracle/_ref), runs the FliX index
concept - build, insert, remove, lookup, range_lookup_sum, lookups_successor -
and every answer equals the oracle's: a reference-side caller works unchanged
through the C ABI."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import empty_u32, to_dev, to_host
from oracle import OracleLSM

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libflix_gpulsmopt_adapter.so")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter not built (oracle/Makefile)")]


def _lib(gl):
    gl.load()  # libgpulsm.so first, so the adapter's imports resolve to the in-tree library
    lib = C.CDLL(ADAPTER)
    vp, u64 = C.c_void_p, C.c_uint64
    for name, args in {"adapter_create": [C.POINTER(vp)], "adapter_destroy": [vp],
                       "adapter_build": [vp, vp, u64, u64], "adapter_insert": [vp, vp, vp, u64, vp],
                       "adapter_remove": [vp, vp, u64, vp], "adapter_lookup": [vp, vp, vp, u64, vp],
                       "adapter_range_lookup_sum": [vp, vp, vp, vp, u64, vp],
                       "adapter_lookups_successor": [vp, vp, vp, u64, vp]}.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = C.c_int
    lib.adapter_last_error.restype = C.c_char_p
    return lib


def test_flix_adapter_runs_over_the_c_abi(gl, cuda):
    import torch

    lib = _lib(gl)

    def ok(rc):
        assert rc == 0, lib.adapter_last_error().decode()

    rng = np.random.default_rng(9)
    n = 1 << 16
    keys = np.unique(rng.integers(0, 1 << 31, n + 4096, dtype=np.uint64))[:n].astype(np.uint32)
    keys = keys[rng.permutation(keys.size)]
    o = OracleLSM()
    o.bulk_build(keys, np.arange(keys.size, dtype=np.uint32))  # the adapter's build values: positions
    h = C.c_void_p()
    ok(lib.adapter_create(C.byref(h)))
    kd = to_dev(keys)
    ok(lib.adapter_build(h, kd.data_ptr(), keys.size, 4 * n))
    torch.cuda.synchronize()
    for step in range(3):  # inserts (updates and new keys), then a remove batch
        k = np.concatenate([keys[rng.integers(0, keys.size, 3000)],
                            rng.integers(0, 1 << 31, 3000, dtype=np.uint64).astype(np.uint32)])
        v = rng.integers(0, 1 << 32, k.size, dtype=np.uint64).astype(np.uint32)
        # device copies held by name for the duration of each call (a temporary
        # freed inside the argument list could be reused by the next copy)
        kd_, vd_ = to_dev(k), to_dev(v)
        ok(lib.adapter_insert(h, kd_.data_ptr(), vd_.data_ptr(), k.size, None))
        o.insert(k, v)
        e = keys[rng.integers(0, keys.size, 2000)]
        ed = to_dev(e)
        ok(lib.adapter_remove(h, ed.data_ptr(), e.size, None))
        o.erase(e)
    torch.cuda.synchronize()
    q = np.concatenate([keys[:5000], rng.integers(0, 1 << 32, 3000, dtype=np.uint64).astype(np.uint32)])
    qd = to_dev(q)
    out = empty_u32(q.size)
    ok(lib.adapter_lookup(h, qd.data_ptr(), out.data_ptr(), q.size, None))
    torch.cuda.synchronize()
    assert np.array_equal(to_host(out)[: q.size], o.lookup(q))
    lo = q[:2000]
    hi = (lo.astype(np.uint64) + rng.integers(0, 1 << 24, lo.size, dtype=np.uint64)).clip(0, 0xFFFFFFFF).astype(np.uint32)
    lod, hid = to_dev(lo), to_dev(hi)
    sums = empty_u32(lo.size)
    ok(lib.adapter_range_lookup_sum(h, lod.data_ptr(), hid.data_ptr(), sums.data_ptr(), lo.size, None))
    succ = empty_u32(q.size)
    ok(lib.adapter_lookups_successor(h, qd.data_ptr(), succ.data_ptr(), q.size, None))
    torch.cuda.synchronize()
    assert np.array_equal(to_host(sums)[: lo.size], o.range_sum(lo, hi))
    assert np.array_equal(to_host(succ)[: q.size], o.successor(q))
    ok(lib.adapter_destroy(h))
