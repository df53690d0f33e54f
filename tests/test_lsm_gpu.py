"""GPU parity of the LSM dictionary (GPULSMOpt semantics) against the CPU oracle.

Every answer is compared bit for bit: integer work, no tolerance.
"""
import numpy as np
import pytest

from conftest import empty_u32, to_dev, to_host
from oracle import OracleLSM
from scenarios import (NOT_FOUND, capacity_ops, forced_validation_steps, key_for_index, range_digest,
                       rollover_ops, sweep_lookup_queries, sweep_range_queries, validation_queries)

pytestmark = pytest.mark.gpu


class Twin:
    """Runs every operation on the GPU dictionary and on the oracle."""

    def __init__(self, gl, **cfg):
        self.d = gl.GPULSMOpt(gl.DictionaryConfig(**cfg))
        self.o = OracleLSM()

    def apply(self, op):
        if op[0] == "insert":
            self.d.insert(to_dev(op[1]), to_dev(op[2]))
            self.o.insert(op[1], op[2])
        else:
            self.d.erase(to_dev(op[1]))
            self.o.erase(op[1])

    def lookup(self, q, with_found=False):
        import torch

        out = empty_u32(q.size)
        found = torch.empty(max(q.size, 1), dtype=torch.uint8, device="cuda") if with_found else None
        self.d.lookup(to_dev(q), out, found, count=q.size)
        got = to_host(out)[: q.size]
        if with_found:
            want_v, want_f = self.o.lookup(q, with_found=True)
            assert np.array_equal(to_host(found, np.uint8)[: q.size], want_f)
            assert np.array_equal(got, want_v)
        else:
            assert np.array_equal(got, self.o.lookup(q))

    def ranges(self, lo, hi):
        out = empty_u32(lo.size)
        self.d.range(to_dev(lo), to_dev(hi), out, count=lo.size)
        assert np.array_equal(to_host(out)[: lo.size], self.o.range_sum(lo, hi))
        self.d.range_count(to_dev(lo), to_dev(hi), out, count=lo.size)
        assert np.array_equal(to_host(out)[: lo.size], self.o.range_count(lo, hi))
        off, k, v = self.d.range_query(to_dev(lo), to_dev(hi))
        o_off, o_k, o_v = self.o.range_pairs(lo, hi)
        assert np.array_equal(to_host(off, np.uint64), o_off)
        assert np.array_equal(to_host(k), o_k)
        assert np.array_equal(to_host(v), o_v)

    def successor(self, q):
        out = empty_u32(q.size)
        self.d.successor(to_dev(q), out, count=q.size)
        assert np.array_equal(to_host(out)[: q.size], self.o.successor(q))


def test_sort_pairs_stable(gl, cuda):
    import torch

    rng = np.random.default_rng(5)
    for n in (1, 100, 4096, 4097, 300_000):
        k = rng.integers(0, 1 << 12, n, dtype=np.uint64).astype(np.uint32)  # many ties
        v = np.arange(n, dtype=np.uint32)
        ko, vo = empty_u32(n), empty_u32(n)
        gl.sort_pairs(to_dev(k), to_dev(v), ko, vo)
        order = np.argsort(k, kind="stable")
        assert np.array_equal(to_host(ko)[:n], k[order])
        assert np.array_equal(to_host(vo)[:n], v[order])
    n = 200_000
    k64 = rng.integers(0, 1 << 40, n, dtype=np.uint64)
    ko = torch.empty(n, dtype=torch.int64, device="cuda")
    vo = empty_u32(n)
    gl.sort_pairs(to_dev(k64), to_dev(np.arange(n, dtype=np.uint32)), ko, vo, 0, 40)
    order = np.argsort(k64, kind="stable")
    assert np.array_equal(to_host(ko, np.uint64), k64[order])
    assert np.array_equal(to_host(vo)[:n], order.astype(np.uint32))


def test_forced_validation_scenarios(gl, cuda):
    t = Twin(gl, max_elements=1 << 20)
    for name, ops, expected, removed in forced_validation_steps():
        for op in ops:
            t.apply(op)
        q, want = validation_queries(expected, removed)
        out = empty_u32(q.size)
        t.d.lookup(to_dev(q), out, count=q.size)
        assert np.array_equal(to_host(out)[: q.size], want), name
        t.lookup(q, with_found=True)
    assert t.d.canonical_carry_status() == 0


def test_multilevel_rollover(gl, cuda):
    ops, q, expected = rollover_ops()
    t = Twin(gl, max_elements=512, batch_capacity=4, level_zero_capacity=64)
    for op in ops:
        t.apply(op)
    out = empty_u32(q.size)
    t.d.lookup(to_dev(q), out)
    assert np.array_equal(to_host(out), expected)
    assert t.d.canonical_carry_status() == 0
    t.successor(np.arange(0, 300, dtype=np.uint32))
    t.ranges(np.array([0, 10, 200], np.uint32), np.array([255, 20, 100], np.uint32))


def test_capacity_exhaustion_is_controlled(gl, cuda):
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1024, batch_capacity=4, level_zero_capacity=1024))
    o = OracleLSM()
    raised = None
    for op in capacity_ops():
        try:
            d.insert(to_dev(op[1]), to_dev(op[2]))
        except gl.CapacityError as e:
            raised = e
            break
        o.insert(op[1], op[2])
    if raised is None:  # the receipt of the last batch may still be in flight
        assert d.canonical_carry_status() & gl._native.STATUS_OUTPUT_OVERFLOW
        with pytest.raises(gl.CapacityError, match="capacity"):
            d.insert(to_dev(np.array([1], np.uint32)), to_dev(np.array([1], np.uint32)))
    assert "capacity" in str(raised or "capacity")
    assert d.canonical_carry_status() & gl._native.STATUS_OUTPUT_OVERFLOW
    # every accepted update stays readable
    q = np.arange(0, 17 * 16 * 4 + 8, dtype=np.uint32)
    out = empty_u32(q.size)
    d.lookup(to_dev(q), out)
    assert np.array_equal(to_host(out), o.lookup(q))


@pytest.mark.parametrize("batch_capacity,level_zero,fan_in", [(64, 0, 2), (256, 512, 4), (1024, 0, 8)])
def test_random_updates_match_oracle(gl, cuda, batch_capacity, level_zero, fan_in):
    rng = np.random.default_rng(batch_capacity + fan_in)
    t = Twin(gl, max_elements=1 << 16, batch_capacity=batch_capacity, level_zero_capacity=level_zero,
             fan_in=fan_in)
    universe = rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)
    universe[:6] = [0, 1, 2, 0xFFFFFFFF, 0xFFFFFFFE, 0x80000000]
    for step in range(60):
        n = int(rng.integers(0, 3 * batch_capacity))
        k = universe[rng.integers(0, universe.size, n)]
        if rng.random() < 0.3:
            t.apply(("erase", k))
        else:
            v = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            v[: min(n, 3)] = 0xFFFFFFFF  # real values equal to the tombstone sentinel
            t.apply(("insert", k, v))
        if step % 10 == 9:
            q = np.concatenate([universe, rng.integers(0, 1 << 32, 500, dtype=np.uint64).astype(np.uint32)])
            t.lookup(q)
            t.lookup(q, with_found=True)
            lo = universe[rng.integers(0, universe.size, 300)]
            hi = (lo.astype(np.uint64) + rng.integers(0, 1 << 28, 300, dtype=np.uint64)).clip(0, 0xFFFFFFFF)
            lo[:3] = [5, 0, 0xFFFFFFFF]
            hi = hi.astype(np.uint32)
            hi[:3] = [4, 0xFFFFFFFF, 0xFFFFFFFF]  # lo > hi, full range, single key
            t.ranges(lo, hi)
            t.successor(q)
    assert t.d.canonical_carry_status() == 0


@pytest.mark.parametrize("batch_capacity,level_zero,fan_in", [(256, 512, 4), (1 << 20, 0, 4)])
def test_mixed_update_batches_match_oracle(gl, cuda, batch_capacity, level_zero, fan_in):
    """gpulsm_dict_update: inserts and erases in one batch, the last row of a
    key winning, equal to the oracle applying the rows one at a time; mixed
    with insert-only and erase-only batches, through level cascades, with
    inserted values equal to the tombstone sentinel and keys inserted, erased
    and re-inserted inside one batch (also across a tile boundary of the
    batch capacity)."""
    rng = np.random.default_rng(batch_capacity + 5)
    t = Twin(gl, max_elements=1 << 21, batch_capacity=batch_capacity, level_zero_capacity=level_zero,
             fan_in=fan_in)
    universe = rng.integers(0, 1 << 32, 20000, dtype=np.uint64).astype(np.uint32)
    universe[:6] = [0, 1, 2, 0xFFFFFFFF, 0xFFFFFFFE, 0x80000000]
    import torch
    for step in range(30):
        n = int(rng.choice([1, 2, 100, 4095, 4097, 70000, 300000]))
        k = universe[rng.integers(0, universe.size, n)]
        v = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        v[rng.random(n) < 0.05] = 0xFFFFFFFF  # real values equal to the tombstone sentinel
        e = (rng.random(n) < rng.choice([0.0, 0.3, 1.0] if step % 4 == 0 else [0.5])).astype(np.uint8)
        if n >= 3:  # insert, erase, insert the same key inside the batch; and the reverse
            k[:3] = k[0]
            e[:3] = [0, 1, 0]
            k[-2:] = k[-1]
            e[-2:] = [0, 1]
        t.d.update(to_dev(k), to_dev(v), torch.from_numpy(e).cuda())
        t.o.update(k, v, e)
        if step % 6 == 5:
            q = np.concatenate([universe, rng.integers(0, 1 << 32, 500, dtype=np.uint64).astype(np.uint32)])
            t.lookup(q, with_found=True)
            lo = universe[rng.integers(0, universe.size, 300)]
            hi = (lo.astype(np.uint64) + rng.integers(0, 1 << 28, 300, dtype=np.uint64)).clip(0, 0xFFFFFFFF)
            t.ranges(lo, hi.astype(np.uint32))
            t.successor(q[rng.integers(0, q.size, 3000)])
        if step % 5 == 2:  # plain batches between mixed ones
            t.apply(("erase", universe[rng.integers(0, universe.size, 3000)]))
            kk = universe[rng.integers(0, universe.size, 3000)]
            t.apply(("insert", kk, rng.integers(0, 1 << 32, kk.size, dtype=np.uint64).astype(np.uint32)))
    assert t.d.canonical_carry_status() == 0
    z = torch.empty(0, dtype=torch.int32, device="cuda")
    t.d.update(z, z, torch.empty(0, dtype=torch.uint8, device="cuda"))  # empty: a no-op
    kd = to_dev(universe)
    with pytest.raises(gl.InvalidArgument):  # values and erase marks are required
        gl._native.check(t.d._lib.gpulsm_dict_update(t.d._h, kd.data_ptr(), None, None, 5, None))


def skewed_batches(rng):
    """Update batches shaped to exercise every admission route: batch sizes
    around the 4096-row bucket limit, all-equal keys, few distinct keys
    repeated (buckets of one key larger than shared memory), a dense cluster
    inside a wide range (one bucket sorted through global memory) and a
    normal distribution (uneven buckets)."""
    u32 = lambda a: np.asarray(a, np.uint64).astype(np.uint32)
    full = lambda n: u32(rng.integers(0, 1 << 32, n, dtype=np.uint64))
    yield "sizes", [full(n) for n in (1, 2, 3, 4095, 4096, 4097, 3 * 2048 + 1, 100_000)]
    yield "all_equal", [np.full(1 << 20, 0x9E3779B9, np.uint32), np.full(5000, 0, np.uint32)]
    yield "few_keys", [u32(rng.integers(0, 100, 1 << 20)), u32(rng.integers(0, 1000, 300_000))]
    cluster = u32(rng.integers(500_000_000, 500_000_000 + (1 << 14), 1 << 19))
    yield "cluster", [rng.permutation(np.concatenate([cluster, full(1 << 19)]))]
    normal = rng.normal(2.0 ** 31, 2.0 ** 26, 1 << 20).clip(0, 2.0 ** 32 - 1)
    yield "normal", [u32(normal)]
    yield "top_bits", [u32(rng.integers(0, 1 << 8, 200_000)) << np.uint32(24),
                       full(50_000) | np.uint32(0xFFFF0000)]


def test_admission_skewed_batches(gl, cuda):
    rng = np.random.default_rng(77)
    for name, batches in skewed_batches(rng):
        t = Twin(gl, max_elements=1 << 23)
        seen = []
        for i, k in enumerate(batches):
            v = rng.integers(0, 1 << 32, k.size, dtype=np.uint64).astype(np.uint32)
            t.apply(("insert", k, v))
            seen.append(k)
            if i % 2 == 1:  # erase a skewed sample of what is there
                t.apply(("erase", k[rng.integers(0, k.size, max(1, k.size // 3))]))
        keys = np.unique(np.concatenate(seen))
        probe = np.concatenate([keys, rng.integers(0, 1 << 32, 2000, dtype=np.uint64).astype(np.uint32)])
        t.lookup(probe, with_found=True)
        t.successor(probe[rng.integers(0, probe.size, 5000)])
        lo = probe[rng.integers(0, probe.size, 500)]
        hi = (lo.astype(np.uint64) + rng.integers(0, 1 << 26, 500, dtype=np.uint64)).clip(0, 0xFFFFFFFF)
        t.ranges(lo, hi.astype(np.uint32))
        assert t.d.canonical_carry_status() == 0, name


def test_empty_and_edge_inputs(gl, cuda):
    import torch

    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 12))
    q = np.array([0, 1, 0xFFFFFFFF], np.uint32)
    out = empty_u32(3)
    d.lookup(to_dev(q), out)
    assert to_host(out).tolist() == [NOT_FOUND] * 3
    d.successor(to_dev(q), out)
    assert to_host(out).tolist() == [NOT_FOUND] * 3
    d.range(to_dev(q), to_dev(q), out)
    assert to_host(out).tolist() == [0, 0, 0]
    z = torch.empty(0, dtype=torch.int32, device="cuda")
    d.insert(z, z)  # empty batches are no-ops
    d.erase(z)
    d.lookup(z, z)
    with pytest.raises(gl.InvalidArgument):
        gl._native.check(d._lib.gpulsm_dict_insert(d._h, None, None, 5, None))
    with pytest.raises(ValueError):
        gl._native.check(d._lib.gpulsm_dict_lookup(d._h, None, 4, None, None, None))
    # pointers the GPU cannot dereference are refused before any kernel runs
    host_buf = np.zeros(16, np.uint32)
    qd = to_dev(q)
    with pytest.raises(gl.InvalidArgument, match="device-accessible|CUDA pointer"):
        gl._native.check(d._lib.gpulsm_dict_lookup(d._h, qd.data_ptr(), 3, host_buf.ctypes.data, None, None))
    with pytest.raises(gl.InvalidArgument):
        gl._native.check(d._lib.gpulsm_dict_lookup(d._h, qd.data_ptr(), 3, out.data_ptr(), 1 << 24, None))
    with pytest.raises(ValueError):
        gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 33))
    d.insert(to_dev(np.array([0xFFFFFFFF, 0], np.uint32)), to_dev(np.array([7, 0xFFFFFFFF], np.uint32)))
    d.lookup(to_dev(q), out)
    assert to_host(out).tolist() == [0xFFFFFFFF, NOT_FOUND, 7]
    d.successor(to_dev(np.array([1, 0xFFFFFFFF], np.uint32)), out, count=2)
    assert to_host(out)[:2].tolist() == [0xFFFFFFFF, 0xFFFFFFFF]


def test_bulk_build_then_updates(gl, cuda):
    rng = np.random.default_rng(3)
    t = Twin(gl, max_elements=1 << 18, batch_capacity=1 << 12)
    k = rng.integers(0, 1 << 20, 100_000, dtype=np.uint64).astype(np.uint32)
    v = np.arange(k.size, dtype=np.uint32)
    t.d.bulk_build(to_dev(k), to_dev(v))
    t.o.bulk_build(k, v)
    t.lookup(np.arange(0, 1 << 20, 7, dtype=np.uint32))
    for i in range(10):
        kk = rng.integers(0, 1 << 20, 5000, dtype=np.uint64).astype(np.uint32)
        t.apply(("erase", kk) if i % 3 == 2 else ("insert", kk, rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)))
    t.lookup(np.arange(0, 1 << 20, 3, dtype=np.uint32), with_found=True)
    t.successor(rng.integers(0, 1 << 21, 10000, dtype=np.uint64).astype(np.uint32))
    lo = rng.integers(0, 1 << 20, 2000, dtype=np.uint64).astype(np.uint32)
    t.ranges(lo, lo + np.uint32(500))


def test_streams_are_ordered(gl, cuda):
    import torch

    t = Twin(gl, max_elements=1 << 16, batch_capacity=1 << 10)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    rng = np.random.default_rng(9)
    k = rng.integers(0, 1 << 32, 20000, dtype=np.uint64).astype(np.uint32)
    v = rng.integers(0, 1 << 32, 20000, dtype=np.uint64).astype(np.uint32)
    kd, vd = to_dev(k), to_dev(v)
    torch.cuda.synchronize()
    t.d.insert(kd, vd, stream=s1)
    t.o.insert(k, v)
    out = empty_u32(k.size)
    t.d.lookup(kd, out, stream=s2)
    s2.synchronize()
    assert np.array_equal(to_host(out), t.o.lookup(k))


def test_updates_overlap_merges_and_release_their_input(gl, cuda):
    """insert/erase return once the batch is admitted (its merges run on the
    dictionary's stream, overlapping the next admission): the caller may
    overwrite the batch in stream order right away, and a read on any stream
    sees every merge."""
    import torch

    t = Twin(gl, max_elements=1 << 18, batch_capacity=1 << 12, level_zero_capacity=1 << 13)
    rng = np.random.default_rng(21)
    s = torch.cuda.Stream()
    kbuf = torch.empty(1 << 12, dtype=torch.int32, device="cuda")
    vbuf = torch.empty(1 << 12, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(s):
        for i in range(40):  # one staging buffer, refilled in stream order after every update
            k = rng.integers(0, 1 << 16, 1 << 12, dtype=np.uint64).astype(np.uint32)
            v = rng.integers(0, 1 << 32, 1 << 12, dtype=np.uint64).astype(np.uint32)
            kbuf.copy_(to_dev(k), non_blocking=True)
            if i % 5 == 4:
                t.d.erase(kbuf, stream=s)
                t.o.erase(k)
            else:
                vbuf.copy_(to_dev(v), non_blocking=True)
                t.d.insert(kbuf, vbuf, stream=s)
                t.o.insert(k, v)
            kbuf.fill_(-1)  # the batch was read before this runs
            vbuf.fill_(-1)
        t.d.join(stream=s)
    s.synchronize()
    probe = np.arange(1 << 16, dtype=np.uint32)
    out = empty_u32(probe.size)
    t.d.lookup(to_dev(probe), out)  # another stream: the read joins the merges itself
    torch.cuda.synchronize()
    assert np.array_equal(to_host(out), t.o.lookup(probe))
    assert t.d.canonical_carry_status() == 0


def test_lsm_small_configuration(gl, cuda, workloads):
    w = workloads.lsm_small()
    t = Twin(gl, max_elements=1 << 20, batch_capacity=1 << 16)
    for op in w.ops:
        t.apply(op)
    t.lookup(w.lookups)
    t.lookup(w.lookups, with_found=True)
    out = empty_u32(w.range_lo.size)
    t.d.range_count(to_dev(w.range_lo), to_dev(w.range_hi), out)
    assert np.array_equal(to_host(out), t.o.range_count(w.range_lo, w.range_hi))
    t.ranges(w.range_lo[:4096], w.range_hi[:4096])
    t.successor(w.lookups[:100_000])


def test_paper_sweep_protocol(gl, cuda):
    n = 1 << 20
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=n))
    keys = key_for_index(np.arange(n))
    ones = to_dev(np.ones(1 << 16, np.uint32))
    for b in range(0, n, 1 << 16):
        d.insert(to_dev(keys[b:b + (1 << 16)]), ones)
    out = empty_u32(1 << 18)
    d.lookup(to_dev(sweep_lookup_queries(1 << 18, n, True, 3)), out)
    assert (to_host(out) == 1).all()
    d.lookup(to_dev(sweep_lookup_queries(1 << 18, n, False, 4)), out)
    assert (to_host(out) == NOT_FOUND).all()
    o = OracleLSM()
    o.insert(keys, np.ones(n, np.uint32))
    for expected_hits in (8, 1024):
        lo, hi = sweep_range_queries(1 << 16, n, expected_hits, 5)
        r = empty_u32(lo.size)
        d.range(to_dev(lo), to_dev(hi), r)
        assert range_digest(to_host(r)) == range_digest(o.range_sum(lo, hi))


def test_lsm_scale_reduced(gl, cuda, workloads):
    """The at-scale configuration's shape at 1/16 size, exact against the oracle."""
    w = workloads.lsm_scale(scale=4)
    t = Twin(gl, max_elements=(1 << 22) + (1 << 18), batch_capacity=1 << 16)
    for op in w.ops:
        t.apply(op)
    t.lookup(w.lookups)
    t.ranges(w.range_lo, w.range_hi)
    t.successor(w.lookups[:200_000])
    assert t.d.canonical_carry_status() == 0


@pytest.mark.slow
def test_lsm_scale_full_size_properties(gl, cuda, workloads):
    """Full 2^26-key configuration: lookups exact; ranges through per-query
    counts, sums and a digest of every returned pair."""
    import torch

    w = workloads.lsm_scale(scale=0)
    t = Twin(gl, max_elements=(1 << 26) + (1 << 22))
    for op in w.ops:
        t.apply(op)
    t.lookup(w.lookups)
    lo, hi = w.range_lo, w.range_hi
    off, k, v = t.d.range_query(to_dev(lo), to_dev(hi))
    counts = (off[1:] - off[:-1]).to(torch.int64)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint32), t.o.range_count(lo, hi))
    seg = torch.repeat_interleave(torch.arange(lo.size, device="cuda"), counts)
    sums = torch.zeros(lo.size, dtype=torch.int64, device="cuda")
    sums.index_add_(0, seg, v.to(torch.int64) & 0xFFFFFFFF)
    assert np.array_equal((sums.cpu().numpy() & 0xFFFFFFFF).astype(np.uint32), t.o.range_sum(lo, hi))
    keys_sorted = bool(((k[1:].to(torch.int64) & 0xFFFFFFFF) > (k[:-1].to(torch.int64) & 0xFFFFFFFF))
                       .logical_or(seg[1:] != seg[:-1]).all())
    assert keys_sorted
    sample = np.arange(0, lo.size, 997)
    o_off, o_k, o_v = t.o.range_pairs(lo[sample], hi[sample])
    got_k = np.concatenate([to_host(k[int(off[i]):int(off[i + 1])]) for i in sample])
    assert np.array_equal(got_k, o_k)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_search_modes_match_oracle(gl, cuda, mode):
    """Radix directory (0), learned position model per level (1) and plain
    binary search (2) must give identical, exact answers; the levels here are
    large enough (>= 2^22 rows) for the learned mode to fit its models."""
    rng = np.random.default_rng(40 + mode)
    t = Twin(gl, max_elements=1 << 23, batch_capacity=1 << 16, search_mode=mode)
    base = rng.integers(0, 1 << 32, 1 << 22, dtype=np.uint64).astype(np.uint32)
    base[:3] = [0, 1, 0xFFFFFFFF]
    t.d.bulk_build(to_dev(base), to_dev(np.arange(base.size, dtype=np.uint32)))
    t.o.bulk_build(base, np.arange(base.size, dtype=np.uint32))
    for i in range(12):
        k = np.concatenate([base[rng.integers(0, base.size, 1 << 14)],
                            rng.integers(0, 1 << 32, 1 << 15, dtype=np.uint64).astype(np.uint32)])
        if i % 4 == 3:
            t.apply(("erase", k))
        else:
            t.apply(("insert", k, rng.integers(0, 1 << 32, k.size, dtype=np.uint64).astype(np.uint32)))
    q = np.concatenate([base[rng.integers(0, base.size, 50_000)],
                        rng.integers(0, 1 << 32, 50_000, dtype=np.uint64).astype(np.uint32),
                        np.array([0, 1, 2, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32)])
    t.lookup(q, with_found=True)
    t.successor(q[:20_000])
    lo = q[:3000]
    hi = (lo.astype(np.uint64) + rng.integers(0, 1 << 24, lo.size, dtype=np.uint64)).clip(0, 0xFFFFFFFF)
    t.ranges(lo, hi.astype(np.uint32))
    assert t.d.canonical_carry_status() == 0


def test_merge_timing_hook_counts_rows(gl, cuda):
    """The measurement hook brackets every merge launch: launch count, positive
    device time, and algorithmic bytes equal to 9 B per row read and written
    plus 4 B per directory entry (so at least 18 B per merged output row)."""
    rng = np.random.default_rng(21)
    t = Twin(gl, max_elements=1 << 16, batch_capacity=1 << 10)
    t.d.kernel_timing(True)
    t.d.kernel_timing_read()
    for _ in range(12):
        k = rng.integers(0, 1 << 32, 1 << 10, dtype=np.uint64).astype(np.uint32)
        t.apply(("insert", k, np.arange(k.size, dtype=np.uint32)))
    got = t.d.kernel_timing_read()
    t.d.kernel_timing(False)
    assert got["launches"] > 0 and got["ms"] > 0
    rows_out_min = 2 * (1 << 10) * got["launches"] / 2  # every merge reads and writes at least one batch
    assert got["bytes"] >= 18 * rows_out_min
    assert t.d.kernel_timing_read()["launches"] == 0  # a read resets the record
    q = rng.integers(0, 1 << 32, 4096, dtype=np.uint64).astype(np.uint32)
    t.lookup(q)


def test_paper_sweep_runner_writes_reference_csvs(gl, cuda, tmp_path):
    """The sweep runner (gpu-lsm-tree_b200/sweep.py) on a reduced protocol:
    the reference's three CSV files with its columns, every lookup validated,
    range sums equal to range counts (all values are 1) and digests equal to
    the oracle's."""
    import csv
    import importlib

    sw = importlib.import_module("gpu-lsm-tree_b200.sweep")
    rc = sw.main(["--out", str(tmp_path), "--batch-logs", "16", "--insert-limit-log", "19",
                  "--query-limit-log", "18", "--range-chunk-log", "16", "--include-count"])
    assert rc == 0
    ins = list(csv.DictReader(open(tmp_path / "insertion_b16.csv")))
    look = list(csv.DictReader(open(tmp_path / "lookup_b16.csv")))
    rng = list(csv.DictReader(open(tmp_path / "count_range_b16.csv")))
    assert len(ins) == 8 and [int(r["resident_elements"]) for r in ins] == [(i + 1) << 16 for i in range(8)]
    assert {r["scenario"] for r in look} == {"all_existing", "none_existing"} and len(look) == 2 * 4
    assert len(rng) == 4 * 2 * 2  # 4 steps under the query limit, 8 and 1024 hits, count + range
    # digests against the oracle for the first step
    o = OracleLSM()
    o.insert(key_for_index(np.arange(1 << 16)), np.ones(1 << 16, np.uint32))
    for expected in (8, 1024):
        lo, hi = sw.range_queries(1 << 16, 1 << 16, expected, 0x30000 + 1 + expected)
        want = range_digest(o.range_sum(lo, hi))
        row = [r for r in rng if r["r"] == "1" and r["operation"] == "range" and r["expected_hits"] == str(expected)]
        assert (int(row[0]["checksum_sum"]), int(row[0]["checksum_xor"])) == want


@pytest.mark.parametrize("index,key_bits", [("flix", 64), ("flix", 32), ("gpulsmopt", 32)])
def test_updates_runner_writes_reference_result_file(gl, cuda, tmp_path, index, key_bits):
    """The updates runner (gpu-lsm-tree_b200/updates_runner.py) on a reduced
    protocol: every probe, miss and successor validated on the host, and the
    result file in the reference's long form with its record names."""
    import csv
    import importlib

    ur = importlib.import_module("gpu-lsm-tree_b200.updates_runner")
    out = tmp_path / "updates.csv"
    assert ur.main(["--out", str(out), "--index", index, "--key-bits", str(key_bits), "--build-size-log", "16",
                    "--probe-size-log", "14", "--batch-count", "2", "--rebuild"]) == 0
    rows = list(csv.reader(open(out), skipinitialspace=True))
    header = rows[0]
    assert header[:5] == ["EXPERIMENT", "index_type", "index_parameters", "index_id", "run"]
    assert header[-2:] == ["DESCRIPTION", "VALUE"] and "after_update_size" in header
    body = [dict(zip(header, r)) for r in rows[1:]]
    steps = {r["step"] for r in body}
    assert steps == {str(s) for s in range(5)}
    assert {r["DESCRIPTION"] for r in body} >= {"insert_or_delete_time_ms", "probe_time_ms", "probe_miss_time_ms",
                                                "before_update_bytes", "after_update_bytes"}
    sizes = {int(r["step"]): (int(r["before_update_size"]), int(r["after_update_size"])) for r in body}
    assert sizes[0] == (1 << 16, 1 << 16) and sizes[2][1] == 1 << 17 and sizes[4][1] == 1 << 16


def test_cleanup_keeps_answers_and_leaves_one_level(gl, cuda):
    """LSMu's cleanup (FliX/impl_lsm_tree.cuh:1256-1400): after inserts, upserts
    and erases spread over several levels, cleanup returns the live key count,
    leaves one level, and every lookup, range sum, range count and successor
    answer stays the oracle's; updates after it land as usual."""
    import torch

    rng = np.random.default_rng(77)
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 18, batch_capacity=4096, level_zero_capacity=4096,
                                         fan_in=2))
    o = OracleLSM()
    universe = rng.integers(0, 1 << 32, 40000, dtype=np.uint64).astype(np.uint32)
    for step in range(30):
        k = universe[rng.integers(0, universe.size, 3000)]
        if step % 3 == 2:
            d.erase(to_dev(k))
            o.erase(k)
        else:
            v = rng.integers(0, 1 << 32, k.size, dtype=np.uint64).astype(np.uint32)
            d.insert(to_dev(k), to_dev(v))
            o.insert(k, v)
    rows_before, levels_before = d.size()
    assert levels_before > 1 or rows_before > len(o)  # there is something to clean up
    assert d.cleanup() == len(o)
    rows, levels = d.size()
    assert (rows, levels) == (len(o), 1)
    q = np.concatenate([universe[:8000], rng.integers(0, 1 << 32, 2000, dtype=np.uint64).astype(np.uint32)])
    out = empty_u32(q.size)
    d.lookup(to_dev(q), out)
    assert np.array_equal(to_host(out)[: q.size], o.lookup(q))
    lo = q[:1000]
    hi = (lo.astype(np.uint64) + (1 << 26)).clip(0, 0xFFFFFFFF).astype(np.uint32)
    s = empty_u32(lo.size)
    d.range(to_dev(lo), to_dev(hi), s)
    assert np.array_equal(to_host(s)[: lo.size], o.range_sum(lo, hi))
    c = empty_u32(lo.size)
    d.range_count(to_dev(lo), to_dev(hi), c)
    assert np.array_equal(to_host(c)[: lo.size], o.range_count(lo, hi))
    d.successor(to_dev(q), out)
    assert np.array_equal(to_host(out)[: q.size], o.successor(q))
    k = universe[:5000]
    v = np.arange(k.size, dtype=np.uint32)
    d.insert(to_dev(k), to_dev(v))
    o.insert(k, v)
    d.lookup(to_dev(q), out)
    torch.cuda.synchronize()
    assert np.array_equal(to_host(out)[: q.size], o.lookup(q))
    assert d.cleanup() == len(o)


def test_single_level_range_pairs_edges(gl, cuda):
    """The one-level range-pairs copy (warps take 32-query groups from a
    counter, slices of up to 8 rows are copied per lane and longer ones by the
    warp) against the oracle: inverted and empty ranges, single keys present
    and absent, slices around the 8-row per-lane limit, whole-key-space
    ranges, the key-space ends, and query counts that are not multiples of
    the 32-query group."""
    rng = np.random.default_rng(11)
    t = Twin(gl, max_elements=1 << 18, batch_capacity=1 << 14)
    keys = np.unique(rng.integers(0, 1 << 20, 60000, dtype=np.uint64).astype(np.uint32))
    keys = np.concatenate([keys, np.array([0, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32)])
    vals = rng.integers(0, 1 << 32, keys.size, dtype=np.uint64).astype(np.uint32)
    t.apply(("insert", keys, vals))
    t.apply(("erase", keys[rng.integers(0, keys.size, 3000)]))
    t.d.cleanup()  # one tombstone-free level: every range read takes the one-level path
    assert t.d.size()[1] == 1
    lo, hi = [], []
    for w in (0, 1, 2, 50, 100, 130, 140, 150, 160, 300, 5000, 1 << 16):  # ~0..3700 rows
        a = rng.integers(0, 1 << 20, 64, dtype=np.uint64)
        lo.append(a)
        hi.append(a + w)
    present = keys[rng.integers(0, keys.size, 64)].astype(np.uint64)
    lo += [present, present + 1, np.array([0, 0, 5, 0xFFFFFF00, 0xFFFFFFFF, 0xFFFFFFFF, 100, 1 << 21], np.uint64)]
    hi += [present, present + 1, np.array([0xFFFFFFFF, 0, 0, 0xFFFFFFFF, 0xFFFFFFFF, 0, 99, 1 << 22], np.uint64)]
    lo = np.concatenate(lo).clip(0, 0xFFFFFFFF).astype(np.uint32)
    hi = np.concatenate(hi).clip(0, 0xFFFFFFFF).astype(np.uint32)
    perm = rng.permutation(lo.size)
    lo, hi = lo[perm], hi[perm]
    for n in (1, 31, 33, 100, lo.size):
        t.ranges(lo[:n], hi[:n])
