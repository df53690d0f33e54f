"""Seeded synthetic workloads with the shapes of the dictionary configurations.

No public dataset is involved; these generators restate the configured sizes
and distributions (numpy PCG64, seed 0x5EED + config id):

  lsm_small  2^20 u32 keys uniform on [0, 2^32-2] (duplicates allowed), values
             = global insertion counter, 16 insert batches of 2^16; 2^20
             lookups (50% inserted keys, 50% uniform); 2^14 range counts,
             lo uniform, width uniform on [1, 2^16].
  lsm_scale  64 insert batches of 2^20; after every 4th insert batch a delete
             batch of 2^18 keys drawn from the keys inserted so far; 2^24
             lookups (70% Zipf s=0.99 over the inserted keys, 30% uniform);
             2^20 range queries returning pairs, width log-uniform on [1, 2^20].
  flix       bulk build of sorted unique u64 keys with geometric gaps (mean 16,
             first key >= 2, never 0xffffffff); rounds of an insert batch (50%
             uniform over the span, 50% in 1024 hot ranges, unique, absent),
             a delete batch of live keys and successor probes uniform over the span.

`scale` divides every size by 2^scale so tests can run the same shapes small.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

KEY_MAX = 0xFFFFFFFE  # keys uniform on [0, 2^32 - 2]


def rng_for(config_id: int, salt: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(0x5EED + config_id + 1000003 * salt))


def zipf_ranks(rng: np.random.Generator, n_items: int, size: int, s: float = 0.99) -> np.ndarray:
    """Zipf-distributed ranks in [0, n_items) by inverting the continuous power law
    (approximates the discrete Zipf(s) for large n_items)."""
    u = rng.random(size)
    if abs(s - 1.0) < 1e-9:
        r = np.exp(u * np.log(n_items + 1.0)) - 1.0
    else:
        a = 1.0 - s
        r = ((n_items + 1.0) ** a - 1.0) * u + 1.0
        r = r ** (1.0 / a) - 1.0
    return np.minimum(r.astype(np.int64), n_items - 1)


@dataclass
class LsmWorkload:
    name: str
    ops: list = field(default_factory=list)  # ("insert", keys, values) | ("erase", keys)
    lookups: np.ndarray | None = None
    range_lo: np.ndarray | None = None
    range_hi: np.ndarray | None = None
    range_kind: str = "count"

    @property
    def inserted_keys(self) -> int:
        return sum(op[1].size for op in self.ops if op[0] == "insert")

    @property
    def erased_keys(self) -> int:
        return sum(op[1].size for op in self.ops if op[0] == "erase")


def lsm_small(scale: int = 0) -> LsmWorkload:
    rng = rng_for(1)
    batch = 1 << (16 - scale)
    w = LsmWorkload("lsm_small: 2^20 u32 keys in 16 batches of 2^16, 2^20 lookups, 2^14 range counts")
    counter = 0
    all_keys = []
    for _ in range(16):
        k = rng.integers(0, KEY_MAX + 1, batch, dtype=np.uint32)
        v = np.arange(counter, counter + batch, dtype=np.uint32)
        counter += batch
        w.ops.append(("insert", k, v))
        all_keys.append(k)
    inserted = np.concatenate(all_keys)
    nq = 1 << (20 - scale)
    hits = inserted[rng.integers(0, inserted.size, nq // 2)]
    misses = rng.integers(0, KEY_MAX + 1, nq - nq // 2, dtype=np.uint32)
    q = np.concatenate([hits, misses])
    rng.shuffle(q)
    w.lookups = q
    nr = 1 << (14 - min(scale, 6))
    lo = rng.integers(0, KEY_MAX + 1, nr, dtype=np.uint64)
    width = rng.integers(1, (1 << 16) + 1, nr, dtype=np.uint64)
    hi = np.minimum(lo + width - 1, 0xFFFFFFFF)
    w.range_lo = lo.astype(np.uint32)
    w.range_hi = hi.astype(np.uint32)
    w.range_kind = "count"
    return w


def lsm_scale(scale: int = 0, insert_batches: int = 64) -> LsmWorkload:
    rng = rng_for(2)
    batch = 1 << (20 - scale)
    del_batch = 1 << (18 - scale)
    w = LsmWorkload("lsm_scale: 2^26 u32 pairs in 64 batches of 2^20 + 16 delete batches of 2^18, "
                    "2^24 lookups, 2^20 range-pair queries")
    counter = 0
    inserted = []
    for b in range(insert_batches):
        k = rng.integers(0, KEY_MAX + 1, batch, dtype=np.uint32)
        v = np.arange(counter, counter + batch, dtype=np.uint32)
        counter += batch
        w.ops.append(("insert", k, v))
        inserted.append(k)
        if (b + 1) % 4 == 0:
            # draw uniformly from every key inserted so far without concatenating
            sizes = np.array([x.size for x in inserted])
            pick = rng.integers(0, sizes.sum(), del_batch)
            which = np.searchsorted(np.cumsum(sizes), pick, side="right")
            offs = pick - np.concatenate([[0], np.cumsum(sizes)[:-1]])[which]
            dk = np.empty(del_batch, np.uint32)
            for j in np.unique(which):
                m = which == j
                dk[m] = inserted[j][offs[m]]
            w.ops.append(("erase", dk))
    all_ins = np.concatenate(inserted)
    nq = 1 << (24 - scale)
    n_hit = int(nq * 0.7)
    ranks = zipf_ranks(rng, all_ins.size, n_hit, 0.99)
    hits = all_ins[ranks]
    misses = rng.integers(0, KEY_MAX + 1, nq - n_hit, dtype=np.uint32)
    q = np.concatenate([hits, misses])
    rng.shuffle(q)
    w.lookups = q
    nr = 1 << (20 - scale)
    lo = rng.integers(0, KEY_MAX + 1, nr, dtype=np.uint64)
    width = np.floor(np.exp(rng.random(nr) * np.log(float(1 << 20)))).astype(np.uint64)
    width = np.clip(width, 1, 1 << 20)
    hi = np.minimum(lo + width - 1, 0xFFFFFFFF)
    w.range_lo = lo.astype(np.uint32)
    w.range_hi = hi.astype(np.uint32)
    w.range_kind = "pairs"
    return w


@dataclass
class FlixWorkload:
    name: str
    build_keys: np.ndarray
    rounds: list  # (insert_keys, insert_values, delete_keys, successor_probes)
    span: tuple
    # flix_fast only: which build keys the rounds deleted (the live set after
    # the last round is build_keys[~build_deleted] plus every round's inserts)
    build_deleted: np.ndarray | None = None


def flix(scale: int = 0, rounds: int = 32, key_bits: int = 64) -> FlixWorkload:
    """Bulk build 2^28 sorted keys (gaps geometric, mean 16) then rounds of
    2^22 inserts / 2^21 deletes / 2^24 successor probes (sizes / 2^scale)."""
    rng = rng_for(3)
    n = 1 << (28 - scale)
    gaps = rng.geometric(1.0 / 16.0, n).astype(np.uint64)
    keys = np.cumsum(gaps, dtype=np.uint64) + np.uint64(1)  # first key >= 2
    if key_bits == 32:
        keys = keys[keys < 0xFFFFFFFE]
    keys = keys[keys != 0xFFFFFFFF]
    lo_span, hi_span = int(keys[0]), int(keys[-1])
    w = FlixWorkload("flix: bulk build of 2^28 sorted u64 keys, rounds of 2^22 inserts, 2^21 deletes, "
                     "2^24 successor probes", keys, [], (lo_span, hi_span))
    n_ins = 1 << (22 - scale)
    n_del = 1 << (21 - scale)
    n_succ = 1 << (24 - scale)
    hot_starts = rng.integers(lo_span, hi_span - (1 << 17), 1024, dtype=np.uint64)
    # live set kept as a sorted array (updated per round)
    live_keys = keys.copy()
    for _ in range(rounds):
        want = n_ins
        cand_u = rng.integers(lo_span, hi_span, want, dtype=np.uint64)
        hr = rng.integers(0, 1024, want - want // 2)
        cand_h = hot_starts[hr] + rng.integers(0, 1 << 17, hr.size, dtype=np.uint64)
        cand = np.concatenate([cand_u[: want // 2], cand_h])
        cand = cand[(cand >= 2) & (cand != 0xFFFFFFFF)]
        cand = np.unique(cand)
        pos = np.searchsorted(live_keys, cand)
        present = (pos < live_keys.size) & (live_keys[np.minimum(pos, live_keys.size - 1)] == cand)
        ins = cand[~present]
        rng.shuffle(ins)
        ins = ins[:want]
        ins_vals = rng.integers(0, 1 << 32, ins.size, dtype=np.uint64).astype(np.uint32)
        live_keys = np.union1d(live_keys, ins)
        dels = live_keys[rng.choice(live_keys.size, n_del, replace=False)]
        live_keys = np.setdiff1d(live_keys, dels, assume_unique=True)
        probes = rng.integers(lo_span, hi_span + 2, n_succ, dtype=np.uint64)
        w.rounds.append((ins, ins_vals, dels, probes))
    return w


def _bitmap_set(bm: np.ndarray, sorted_unique: np.ndarray) -> None:
    """Sets the bits of sorted unique keys in a byte bitmap (vectorised: the
    bits of keys sharing a byte are OR-reduced first)."""
    if not sorted_unique.size:
        return
    byte = sorted_unique >> np.uint64(3)
    bit = (np.uint8(1) << (sorted_unique & np.uint64(7)).astype(np.uint8)).astype(np.uint8)
    starts = np.flatnonzero(np.concatenate([[True], byte[1:] != byte[:-1]]))
    bm[byte[starts]] |= np.bitwise_or.reduceat(bit, starts)


def _bitmap_has(bm: np.ndarray, keys: np.ndarray) -> np.ndarray:
    return ((bm[keys >> np.uint64(3)] >> (keys & np.uint64(7)).astype(np.uint8)) & np.uint8(1)).astype(bool)


def flix_fast(scale: int = 0, rounds: int = 4, key_bits: int = 64) -> FlixWorkload:
    """The FliX configuration's shapes without re-sorting the whole live set
    every round (fast enough for all 32 rounds at full size): 2^28 sorted keys
    with geometric gaps (mean 16), then per round 2^22 unique keys absent from
    the index so far (half uniform over the span, half in 1024 hot ranges of
    2^17 key units; presence is read from a bitmap of every key ever stored), a
    2^21-key delete batch drawn from the build keys not yet deleted (all live),
    and 2^24 uniform successor probes (sizes / 2^scale)."""
    rng = rng_for(3)
    n = 1 << (28 - scale)
    keys = np.cumsum(rng.geometric(1.0 / 16.0, n).astype(np.uint64), dtype=np.uint64) + np.uint64(1)
    if key_bits == 32:
        keys = keys[keys < 0xFFFFFFFE]
    keys = keys[keys != 0xFFFFFFFF]
    n = keys.size
    lo_span, hi_span = int(keys[0]), int(keys[-1])
    w = FlixWorkload("flix: bulk build of 2^28 sorted u64 keys, rounds of 2^22 inserts, 2^21 deletes, "
                     "2^24 successor probes", keys, [], (lo_span, hi_span))
    n_ins, n_del, n_succ = 1 << (22 - scale), 1 << (21 - scale), 1 << (24 - scale)
    hot_starts = rng.integers(lo_span, hi_span - (1 << 17), 1024, dtype=np.uint64)
    bm = np.zeros((hi_span >> 3) + 2, np.uint8)  # every key ever stored (hot ranges end below hi_span)
    _bitmap_set(bm, keys)
    deleted = np.zeros(n, bool)
    for _ in range(rounds):
        cand_u = rng.integers(lo_span, hi_span, n_ins, dtype=np.uint64)
        hr = rng.integers(0, 1024, n_ins)
        cand_h = hot_starts[hr] + rng.integers(0, 1 << 17, n_ins, dtype=np.uint64)
        cand = np.concatenate([cand_u, cand_h])
        cand.sort()
        keep = np.empty(cand.size, bool)
        keep[0] = True
        np.not_equal(cand[1:], cand[:-1], out=keep[1:])
        cand = cand[keep & (cand >= 2) & (cand != 0xFFFFFFFF)]
        ins = cand[~_bitmap_has(bm, cand)]
        ins = ins[rng.permutation(ins.size)[:n_ins]]
        _bitmap_set(bm, np.sort(ins))
        ins_vals = rng.integers(0, 1 << 32, ins.size, dtype=np.uint64).astype(np.uint32)
        pick = rng.integers(0, n, 2 * n_del)
        pick.sort()
        first = np.empty(pick.size, bool)
        first[0] = True
        np.not_equal(pick[1:], pick[:-1], out=first[1:])
        pick = pick[first & ~deleted[pick]]
        pick = pick[rng.permutation(pick.size)[:n_del]]
        deleted[pick] = True
        dels = keys[pick]
        probes = rng.integers(lo_span, hi_span + 2, n_succ, dtype=np.uint64)
        w.rounds.append((ins, ins_vals, dels, probes))
    w.build_deleted = deleted
    return w
