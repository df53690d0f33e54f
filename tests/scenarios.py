"""Known-answer scenarios restated from the reference's own validation code.

These are the reference's test expectations re-expressed as data generators
(no reference code is copied):

  * forced unified validation, FliX/paper_lsmu_sweep.cu:441-700:
    sparse_unique (:524-539), dense_unique (:541-556),
    duplicate_newest_wins (:558-574), tombstone_visibility (:576-589),
    multi-level rollover (:593-641), capacity exhaustion (:646-695);
    misses are probed in quotient 25000 (:485-494).
  * paper-sweep protocol, FliX/paper_lsmu_sweep.cu:64-227: keys
    key_for_index(i) = (i * 747796405 + 289133645) mod 2^30, inserted value 1,
    hit/miss probes through mix32, range bounds for an expected hit count,
    and the range digest (sum + xor of splitmix over (query << 32 | result)).
"""
from __future__ import annotations

import numpy as np

NOT_FOUND = 0xFFFFFFFF
KEY_DOMAIN = 1 << 30
PAPER_INSERT_LIMIT = 1 << 27


def sparse_validation_key(q):
    q = np.asarray(q, dtype=np.uint64)
    return ((q << np.uint64(16)) | ((q * np.uint64(40503) + np.uint64(17)) & np.uint64(0xFFFF))).astype(np.uint32)


def forced_validation_steps():
    """Yields (name, ops, expected_dict_after, removed_keys) for the four cumulative
    scenarios that share one dictionary (max 2^20, default batch capacity)."""
    expected: dict[int, int] = {}
    removed: list[int] = []
    steps = []
    # sparse_unique: one key in each of 32768 quotients
    ops = []
    for batch in range(16):
        q = np.arange(batch * 2048, (batch + 1) * 2048, dtype=np.uint32)
        k = sparse_validation_key(q)
        v = (0x01000000 + q).astype(np.uint32)
        ops.append(("insert", k, v))
        expected.update(zip(k.tolist(), v.tolist()))
    steps.append(("sparse_unique", ops, dict(expected), list(removed)))
    # dense_unique: every suffix of quotient 30000
    ops = []
    for batch in range(16):
        s = np.arange(batch * 4096, (batch + 1) * 4096, dtype=np.uint32)
        k = ((np.uint32(30000) << np.uint32(16)) | s).astype(np.uint32)
        v = (0x02000000 + s).astype(np.uint32)
        ops.append(("insert", k, v))
        expected.update(zip(k.tolist(), v.tolist()))
    steps.append(("dense_unique", ops, dict(expected), list(removed)))
    # duplicate_newest_wins: 4 copies per key per batch, last position of the newest batch wins
    ops = []
    for batch in range(16):
        i = np.arange(4096, dtype=np.uint32)
        k = sparse_validation_key(i % 1024)
        v = (0x10000000 + batch * 4096 + i).astype(np.uint32)
        ops.append(("insert", k, v))
        for kk, vv in zip(k.tolist(), v.tolist()):
            expected[kk] = vv
    steps.append(("duplicate_newest_wins", ops, dict(expected), list(removed)))
    # tombstone_visibility: 16 repeated deletes of 1024 keys
    k = sparse_validation_key(np.arange(1024, dtype=np.uint32))
    ops = [("erase", k) for _ in range(16)]
    for kk in k.tolist():
        expected.pop(kk, None)
        removed.append(kk)
    steps.append(("tombstone_visibility", ops, dict(expected), list(removed)))
    return steps


def validation_queries(expected: dict, removed: list):
    """Query list of the reference's validate(): live keys, removed keys, then
    4096 absent keys of quotient 25000 (FliX/paper_lsmu_sweep.cu:472-494)."""
    keys = list(expected.keys())
    vals = list(expected.values())
    keys += removed
    vals += [NOT_FOUND] * len(removed)
    target = len(keys) + 4096
    suffix = 0
    while len(keys) < target:
        key = (25000 << 16) | (suffix & 0xFFFF)
        suffix += 1
        if key in expected:
            continue
        keys.append(key)
        vals.append(NOT_FOUND)
    return np.array(keys, dtype=np.uint32), np.array(vals, dtype=np.uint32)


def rollover_ops():
    """CANONICAL_MULTILEVEL_ROLLOVER_VALIDATION: config max 512, batch 4, level
    zero 64; 512 batches of 4 updates over 256 keys (:593-641)."""
    ops = []
    expected = np.zeros(256, dtype=np.uint32)
    for batch in range(32 * 16):
        ordinal = np.arange(batch * 4, batch * 4 + 4, dtype=np.uint32)
        k = (ordinal % 256).astype(np.uint32)
        v = (0x28000000 + ordinal).astype(np.uint32)
        expected[k] = v
        ops.append(("insert", k, v))
    return ops, np.arange(256, dtype=np.uint32), expected


def capacity_ops():
    """CANONICAL_CAPACITY_VALIDATION: config max 1024, batch 4, level zero 1024;
    17*16 batches of 4 unique keys exceed the capacity (:646-695)."""
    ops = []
    for batch in range(17 * 16):
        k = np.arange(batch * 4, batch * 4 + 4, dtype=np.uint32)
        ops.append(("insert", k, (0x30000000 + k).astype(np.uint32)))
    return ops


# ---- paper-sweep protocol -------------------------------------------------
def key_for_index(i):
    i = np.asarray(i, dtype=np.uint64)
    return ((i * np.uint64(747796405) + np.uint64(289133645)) & np.uint64(KEY_DOMAIN - 1)).astype(np.uint32)


def mix32(v):
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(16)
    v = (v * np.uint64(0x7FEB352D)) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(15)
    v = (v * np.uint64(0x846CA68B)) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(16)
    return v.astype(np.uint32)


def sweep_lookup_queries(count: int, resident: int, hits: bool, seed: int):
    tid = np.arange(count, dtype=np.uint64)
    r = mix32(tid + np.uint64(seed)).astype(np.uint64)
    if hits:
        return key_for_index(r % np.uint64(resident))
    miss_begin = max(resident, PAPER_INSERT_LIMIT)
    return key_for_index(np.uint64(miss_begin) + r % np.uint64(KEY_DOMAIN - miss_begin))


def sweep_range_queries(count: int, resident: int, expected_hits: int, seed: int):
    tid = np.arange(count, dtype=np.uint64)
    width = (expected_hits * KEY_DOMAIN + resident - 1) // resident
    width = min(max(width, 1), KEY_DOMAIN)
    starts = KEY_DOMAIN - width + 1
    first = mix32(tid + np.uint64(seed)).astype(np.uint64) % np.uint64(starts)
    return first.astype(np.uint32), (first + np.uint64(width - 1)).astype(np.uint32)


def range_digest(results, query_offset: int = 0):
    """(sum, xor) digest of range results as digest_range_results computes it."""
    r = np.asarray(results, dtype=np.uint64)
    q = np.arange(r.size, dtype=np.uint64) + np.uint64(query_offset)
    v = (q << np.uint64(32)) | r
    with np.errstate(over="ignore"):
        v = v + np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    return int(r.sum(dtype=np.uint64)), int(np.bitwise_xor.reduce(v)) if v.size else 0


def bulk_build_stages(seed: int = 21):
    """Stages for the bulk-build fixture (GPULSMOpt.cuh:5738-5834: reset, stable
    radix sort of the pairs, keep the LAST duplicate, mark_last_key_kernel
    :2633-2638).  Yields (op, probe_queries, lo, hi) where op is
    ("bulk", keys, values) | ("insert", keys, values) | ("erase", keys).
    Keys repeat heavily and include 0, 1 and 0xffffffff; the third bulk build
    replaces a dictionary that already holds updates, and the last one is
    empty (the reference returns after the reset, leaving no keys)."""
    rng = np.random.default_rng(seed)
    universe = rng.integers(0, 1 << 32, 1 << 13, dtype=np.uint64).astype(np.uint32)
    universe[:4] = [0, 1, 0xFFFFFFFF, 0xFFFFFFFE]

    def vals(n):
        return rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)

    def probes():
        q = np.concatenate([universe, rng.integers(0, 1 << 32, 2048, dtype=np.uint64).astype(np.uint32)])
        lo = universe[rng.integers(0, universe.size, 512)]
        hi = np.minimum(lo.astype(np.uint64) + rng.integers(0, 1 << 28, 512, dtype=np.uint64),
                        0xFFFFFFFF).astype(np.uint32)
        lo[:2] = [7, 0]
        hi[:2] = [3, 0xFFFFFFFF]
        return q, lo, hi

    stages = []
    k = universe[rng.integers(0, universe.size, 1 << 16)]
    stages.append((("bulk", k, vals(k.size)),) + probes())
    k = universe[rng.integers(0, universe.size, 3000)]
    stages.append((("insert", k, vals(k.size)),) + probes())
    k = universe[rng.integers(0, universe.size, 1500)]
    stages.append((("erase", k),) + probes())
    k = universe[rng.integers(0, universe.size // 2, 20000)]
    stages.append((("bulk", k, vals(k.size)),) + probes())
    stages.append((("bulk", np.zeros(0, np.uint32), np.zeros(0, np.uint32)),) + probes())
    return stages
