"""GPU parity of the FliX bucket layer against the CPU oracle (bit exact)."""
import numpy as np
import pytest

from conftest import empty_u32, to_dev, to_host
from oracle import OracleFlix

pytestmark = pytest.mark.gpu


def keys_t(a, bits):
    return to_dev(np.ascontiguousarray(a, dtype=np.uint64 if bits == 64 else np.uint32))


def empty_keys(n, bits):
    import torch

    return torch.empty(max(n, 1), dtype=torch.int64 if bits == 64 else torch.int32, device="cuda")


def host_keys(t, bits, n):
    return to_host(t, np.uint64 if bits == 64 else np.uint32)[:n].astype(np.uint64)


class FlixTwin:
    def __init__(self, gl, bits, **kw):
        self.bits = bits
        self.f = gl.FlixIndex(key_bits=bits, **kw)
        self.o = OracleFlix(bits)

    def build(self, keys, values=None):
        self.f.build_bucket_layer_only(keys_t(keys, self.bits), keys.size,
                                       values=None if values is None else to_dev(values))
        self.o.build(keys, values)

    def insert(self, k, v):
        self.f.insert(keys_t(k, self.bits), to_dev(v), k.size)
        self.o.insert(k, v)

    def remove(self, k):
        self.f.remove(keys_t(k, self.bits), k.size)
        self.o.remove(k)

    def check(self, probes):
        n = probes.size
        out = empty_u32(n)
        self.f.lookup(keys_t(probes, self.bits), out, n)
        assert np.array_equal(to_host(out)[:n], self.o.lookup(probes))
        sk = empty_keys(n, self.bits)
        self.f.successor(keys_t(probes, self.bits), sk, n)
        assert np.array_equal(host_keys(sk, self.bits, n), self.o.successor(probes))
        # unsorted batches up to 2^20 probes take the fence tree, larger ones are sorted first
        big = np.tile(probes, (1 << 20) // max(n, 1) + 2)
        nb = big.size
        outb, skb = empty_u32(nb), empty_keys(nb, self.bits)
        self.f.lookup(keys_t(big, self.bits), outb, nb)
        assert np.array_equal(to_host(outb)[:nb], self.o.lookup(big))
        self.f.successor(keys_t(big, self.bits), skb, nb)
        assert np.array_equal(host_keys(skb, self.bits, nb), self.o.successor(big))
        sp = np.sort(probes)
        self.f.lookups_ordered(keys_t(sp, self.bits), out, n)
        assert np.array_equal(to_host(out)[:n], self.o.lookup(sp))
        self.f.lookups_successor(keys_t(sp, self.bits), sk, n)
        assert np.array_equal(host_keys(sk, self.bits, n), self.o.successor(sp))
        assert self.f.size() == len(self.o)
        assert self.f.status() == 0


@pytest.mark.parametrize("bits,mode", [(32, 0), (64, 0), (64, 1)])
def test_build_lookup_successor(gl, cuda, bits, mode):
    rng = np.random.default_rng(bits)
    keys = np.unique(rng.integers(2, 1 << (bits - 2), 50_000, dtype=np.uint64))
    t = FlixTwin(gl, bits, search_mode=mode)
    t.build(keys)  # sorted unique, values = input index
    probes = np.concatenate([keys[::3], rng.integers(0, 1 << (bits - 2), 20_000, dtype=np.uint64),
                             np.array([0, 1, 2, keys[-1], keys[-1] + 1], np.uint64)])
    t.check(probes)


@pytest.mark.parametrize("bits", [32, 64])
def test_unsorted_build_keeps_first_duplicate(gl, cuda, bits):
    rng = np.random.default_rng(7)
    keys = rng.integers(2, 5000, 20_000, dtype=np.uint64)
    t = FlixTwin(gl, bits)
    t.build(keys)
    t.check(np.arange(0, 5100, dtype=np.uint64))


@pytest.mark.parametrize("bits,mode", [(32, 0), (64, 0), (32, 1), (64, 1)])
def test_insert_delete_rounds(gl, cuda, bits, mode):
    rng = np.random.default_rng(11 + bits)
    hi = (1 << 31) if bits == 32 else (1 << 40)
    keys = np.unique(rng.integers(2, hi, 100_000, dtype=np.uint64))
    t = FlixTwin(gl, bits, max_elements=400_000, search_mode=mode)
    t.build(keys)
    hot = rng.integers(2, hi - 100_000, 16, dtype=np.uint64)
    for r in range(8):
        uni = rng.integers(2, hi, 10_000, dtype=np.uint64)
        clustered = hot[rng.integers(0, 16, 10_000)] + rng.integers(0, 5000, 10_000, dtype=np.uint64)
        ins = np.concatenate([uni, clustered])  # unsorted, duplicates, some present already
        vals = rng.integers(0, 1 << 32, ins.size, dtype=np.uint64).astype(np.uint32)
        t.insert(ins, vals)
        live = t.o.dump()[0]
        dels = np.concatenate([live[rng.choice(live.size, 5000, replace=False)],
                               rng.integers(2, hi, 500, dtype=np.uint64)])
        t.remove(dels)
        if r % 2 == 1:
            probes = np.concatenate([live[::7], rng.integers(0, hi, 5000, dtype=np.uint64), dels[:1000]])
            t.check(probes)
    t.f.rebuild_bucket_layer_only()
    t.check(np.concatenate([t.o.dump()[0][::5], rng.integers(0, hi, 5000, dtype=np.uint64)]))


def test_delete_everything_then_successor_walks_buckets(gl, cuda):
    keys = np.arange(2, 20_002, dtype=np.uint64) * 3
    t = FlixTwin(gl, 64)
    t.build(keys)
    t.remove(keys[: keys.size - 10])  # empties every bucket but the last
    t.check(np.array([0, 5, 3000, int(keys[-11]), int(keys[-10]), int(keys[-1]) + 1], np.uint64))
    t.remove(keys)
    t.check(np.array([0, 7, int(keys[-1])], np.uint64))
    t.insert(np.array([100, 50, 100], np.uint64), np.array([1, 2, 3], np.uint32))
    t.check(np.array([0, 50, 51, 100, 101], np.uint64))


@pytest.mark.parametrize("mode", [0, 1])
def test_flix_workload_shape_small(gl, cuda, workloads, mode):
    w = workloads.flix(scale=10, rounds=4)
    t = FlixTwin(gl, 64, max_elements=w.build_keys.size * 2, search_mode=mode)
    t.build(w.build_keys)
    for ins, vals, dels, probes in w.rounds:
        t.insert(ins, vals)
        t.remove(dels)
        n = probes.size
        sk = empty_keys(n, 64)
        t.f.successor(keys_t(probes, 64), sk, n)
        assert np.array_equal(host_keys(sk, 64, n), t.o.successor(probes))
    assert t.f.size() == len(t.o)


@pytest.mark.slow
def test_flix_configuration_at_size_after_32_rounds(gl, cuda, workloads):
    """The updatable-index configuration at its stated size: bulk build of 2^28
    sorted u64 keys (geometric gaps, mean 16), 32 rounds of 2^22 inserts (half
    in 1024 hot ranges), 2^21 deletes and 2^24 unsorted successor probes.  Every
    round: status clean and the key count exact.  After round 32: 2^20 uniform
    probes, 2^18 sampled live keys and 2^16 deleted keys checked bit-exact for
    successor and lookup against the std::map answers (the live set and its
    values rebuilt from the generator's record), both through the unsorted
    entry points (sorted inside) and the ordered ones."""
    import torch

    w = workloads.flix_fast(0, rounds=32)
    n0 = w.build_keys.size
    cap = n0 + sum(r[0].size for r in w.rounds)
    f = gl.FlixIndex(key_bits=64, max_elements=cap)
    f.build_bucket_layer_only(keys_t(w.build_keys, 64), n0, max_size=cap)
    expect = n0
    out = empty_keys(w.rounds[0][3].size, 64)
    for r, (ins, vals, dels, probes) in enumerate(w.rounds):
        f.insert(keys_t(ins, 64), to_dev(vals), ins.size)
        f.remove(keys_t(dels, 64), dels.size)
        f.successor(keys_t(probes, 64), out, probes.size)  # the round's probes (timed in bench.py)
        expect += ins.size - dels.size
        assert f.status() == 0, f"round {r}"
        assert f.size() == expect, f"round {r}"
    torch.cuda.synchronize()
    # the exact live set after the last round, with values
    live_b = ~w.build_deleted
    bk = w.build_keys[live_b]
    bv = np.flatnonzero(live_b).astype(np.uint32)  # build values are input positions
    ik = np.concatenate([r[0] for r in w.rounds])
    iv = np.concatenate([r[1] for r in w.rounds])
    o = np.argsort(ik)
    ik, iv = ik[o], iv[o]
    pos = np.searchsorted(bk, ik)
    live_k = np.insert(bk, pos, ik)
    live_v = np.insert(bv, pos, iv)
    assert live_k.size == expect
    rng = np.random.default_rng(32)
    lo, hi = w.span
    dead = w.build_keys[w.build_deleted]
    probes = np.concatenate([rng.integers(lo, hi + 2, 1 << 20, dtype=np.uint64),
                             live_k[rng.integers(0, live_k.size, 1 << 18)],
                             dead[rng.integers(0, dead.size, 1 << 16)]])
    p = np.searchsorted(live_k, probes)
    inb = p < live_k.size
    exact_succ = np.where(inb, live_k[np.minimum(p, live_k.size - 1)], np.uint64(0xFFFFFFFF))
    hit = inb & (live_k[np.minimum(p, live_k.size - 1)] == probes)
    exact_val = np.where(hit, live_v[np.minimum(p, live_v.size - 1)], np.uint32(0xFFFFFFFF)).astype(np.uint32)
    n = probes.size
    sk, lv = empty_keys(n, 64), empty_u32(n)
    f.successor(keys_t(probes, 64), sk, n)
    f.lookup(keys_t(probes, 64), lv, n)
    assert np.array_equal(host_keys(sk, 64, n), exact_succ)
    assert np.array_equal(to_host(lv)[:n], exact_val)
    sp = np.unique(probes)
    q = np.searchsorted(live_k, sp)
    qb = q < live_k.size
    f.lookups_successor(keys_t(sp, 64), sk, sp.size)
    assert np.array_equal(host_keys(sk, 64, sp.size),
                          np.where(qb, live_k[np.minimum(q, live_k.size - 1)], np.uint64(0xFFFFFFFF)))
    assert f.status() == 0
    f.close()
