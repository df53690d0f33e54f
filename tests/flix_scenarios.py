"""Seeded FliX bucket-layer scenarios shared by the fixture generator
(tests/golden/make_golden.py, which runs the reference's own FliX kernels) and
the tests that replay them (tests/golden_cases.py).

Every scenario keeps to the contract of the reference's FliX interface
(FliX/impl_cg_rtx_index_updates.cuh:1711-2677 as driven by
FliX/benchmarks_updates.cuh:252-360,1700-1935):
  - usable keys are >= 2 (0 marks an empty slot, 1 a tombstone:
    FliX/definitions.cuh:86-98, FliX/definitions_updates.cuh:259-261);
  - 64-bit scenarios never store 0xffffffff, the widened not_found sentinel
    (FliX/coarse_granular_lookups_tile_bulk.cuh:672);
  - build keys are unique, insert and remove batches sorted and unique, probes
    of the ordered lookups sorted;
  - values stay below 0xffffffff (the lookup miss value).
Scenarios:
  flix32_main   the reference driver's protocol with 32-bit keys (the
                published configuration): new keys only, live deletes only, a
                rebuild between rounds; every answer is pinned bit-exact.
  flix64_insert 64-bit keys: build, insert rounds (half the keys in hot ranges)
                and successor probes up to past the top key.  The reference's
                64-bit ordered lookup and tiled delete read node values at the
                4-byte-key position (extract_offset_node<smallsize>,
                FliX/coarse_granular_lookups_tile_bulk.cuh:403,
                FliX/coarse_granular_deletes_tiles.cuh:1201), so only the
                operations that never read a value are pinned for 64-bit keys.
  flix32_edge   inputs the driver never sends but the interface admits:
                inserts of keys already present (insert if absent), deletes of
                absent keys, a contiguous delete that empties whole buckets
                with successor probes inside the gap, a rebuild after it, and
                finally the whole index deleted.  The reference deviates from
                the std::map answers in two documented ways here (a successor
                probe inside emptied buckets can read 0, the quirk its own
                driver check skips at FliX/benchmarks_updates.cuh:160-162; a
                rebuild after emptied buckets can lose keys); the tests allow
                exactly those classes and nothing else.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NOT_FOUND = 0xFFFFFFFF


@dataclass
class FlixStage:
    kind: str  # "insert" | "remove" | "rebuild" | "probe"
    keys: np.ndarray | None = None
    values: np.ndarray | None = None
    lookup_probes: np.ndarray | None = None
    successor_probes: np.ndarray | None = None
    # documented reference deviations this probe stage may show (see allowed())
    quirks: tuple = ()


@dataclass
class FlixScenario:
    name: str
    key_bits: int
    build_keys: np.ndarray
    max_size: int
    stages: list = field(default_factory=list)


def _kdtype(key_bits):
    return np.uint32 if key_bits == 32 else np.uint64


def _draw_new(rng, live_sorted, count, lo, hi, key_bits, hot_ranges):
    """`count` sorted unique keys absent from `live_sorted`: half uniform over
    [lo, hi], half clustered in `hot_ranges` narrow intervals around live keys."""
    dt = _kdtype(key_bits)
    out = np.zeros(0, dt)
    centres = live_sorted[rng.integers(0, live_sorted.size, hot_ranges)].astype(np.uint64)
    width = np.uint64(max(64, int((hi - lo) // max(live_sorted.size, 1)) * 8))
    while out.size < count:
        m = 2 * (count - out.size) + 64
        uni = rng.integers(lo, hi + 1, m // 2, dtype=np.uint64)
        c = centres[rng.integers(0, hot_ranges, m - m // 2)]
        off = rng.integers(0, int(width), m - m // 2, dtype=np.uint64)
        hot = np.clip(c + off, lo, hi)
        cand = np.concatenate([uni, hot]).astype(dt)
        cand = cand[(cand >= 2)]
        if key_bits == 64:
            cand = cand[cand != np.uint64(NOT_FOUND)]
        cand = np.setdiff1d(cand, live_sorted)
        out = np.union1d(out, cand)
    sel = np.sort(rng.choice(out.size, count, replace=False))
    return out[sel]


def _values(rng, n):
    return rng.integers(0, NOT_FOUND, n, dtype=np.uint64).astype(np.uint32)


def _probes(rng, live, deleted, lo, hi, key_bits, n_lookup, n_succ, extra_succ=()):
    dt = _kdtype(key_bits)
    parts = [live[rng.integers(0, live.size, n_lookup // 2)] if live.size else np.zeros(0, dt),
             deleted[rng.integers(0, deleted.size, n_lookup // 4)] if deleted.size else np.zeros(0, dt),
             rng.integers(lo, hi + 1, n_lookup // 4, dtype=np.uint64).astype(dt)]
    lp = np.unique(np.concatenate(parts).astype(dt))
    sp = [rng.integers(lo, hi + 1, n_succ, dtype=np.uint64).astype(dt)]
    if live.size:
        top = np.uint64(live[-1])
        sp.append(np.array([live[0], live[-1], max(int(live[0]) - 1, 2)], dtype=dt))
        above = top + np.arange(1, 33, dtype=np.uint64)
        if key_bits == 32:
            above = above[above <= np.uint64(NOT_FOUND - 3)]
        sp.append(above.astype(dt))
    sp.extend(np.asarray(e, dtype=dt) for e in extra_succ)
    s = np.unique(np.concatenate(sp).astype(dt))
    s = s[s >= 2]
    if key_bits == 64:
        s = s[s != np.uint64(NOT_FOUND)]
    return lp[lp >= 2], s


def _build_keys(rng, key_bits, n0):
    if key_bits == 32:
        lo, hi = 2, NOT_FOUND - 3
        keys = np.unique(rng.integers(lo, hi + 1, n0 + n0 // 8, dtype=np.uint64))
    else:
        lo = 2
        gaps = rng.geometric(1.0 / (1 << 20), n0 + n0 // 8).astype(np.uint64)
        keys = np.unique(np.uint64(2) + np.cumsum(gaps))
        keys = keys[keys != np.uint64(NOT_FOUND)]
        hi = int(keys[-1]) + (1 << 24)
    keys = keys[rng.permutation(keys.size)[:n0]].astype(_kdtype(key_bits))  # unique, input order shuffled
    return keys, lo, hi


def main_scenario(seed: int = 101, n0: int = 1 << 14, rounds: int = 4, insert_n: int = 1 << 12,
                  delete_n: int = 1 << 11) -> FlixScenario:
    """32-bit keys: build, then `rounds` of (insert new keys, delete live keys,
    probe lookups and successors), with a rebuild after round 1."""
    rng = np.random.default_rng(seed)
    keys, lo, hi = _build_keys(rng, 32, n0)
    sc = FlixScenario("flix32_main", 32, keys, max_size=8 * (n0 + rounds * insert_n))
    live = np.sort(keys)
    for r in range(rounds):
        ins = _draw_new(rng, live, insert_n, lo, hi, 32, hot_ranges=8)
        sc.stages.append(FlixStage("insert", ins, _values(rng, ins.size)))
        live = np.union1d(live, ins)
        dels = live[np.sort(rng.choice(live.size, delete_n, replace=False))]
        sc.stages.append(FlixStage("remove", dels))
        live = np.setdiff1d(live, dels)
        lp, spr = _probes(rng, live, dels, lo, hi, 32, 1 << 12, 1 << 12)
        sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr))
        if r == 1:
            sc.stages.append(FlixStage("rebuild"))
            sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr))
    return sc


def insert64_scenario(seed: int = 102, n0: int = 1 << 14, rounds: int = 4,
                      insert_n: int = 1 << 12) -> FlixScenario:
    """64-bit keys spanning past 2^32: build, then rounds of new-key inserts
    (half in hot ranges, so nodes split and chains grow) with successor probes
    over the span and past the top key (the widened not_found sentinel)."""
    rng = np.random.default_rng(seed)
    keys, lo, hi = _build_keys(rng, 64, n0)
    sc = FlixScenario("flix64_insert", 64, keys, max_size=8 * (n0 + rounds * insert_n))
    live = np.sort(keys)
    for r in range(rounds):
        ins = _draw_new(rng, live, insert_n, lo, hi, 64, hot_ranges=8)
        sc.stages.append(FlixStage("insert", ins, _values(rng, ins.size)))
        live = np.union1d(live, ins)
        _, spr = _probes(rng, live, np.zeros(0, np.uint64), lo, hi, 64, 4, 1 << 12,
                         (ins[:: max(1, ins.size // 64)],))
        sc.stages.append(FlixStage("probe", successor_probes=spr))
    return sc


def edge_scenario(seed: int = 103, n0: int = 1 << 12) -> FlixScenario:
    """32-bit keys, inputs outside the driver's protocol (see the module doc)."""
    rng = np.random.default_rng(seed)
    span = 1 << 30
    keys = np.unique(rng.integers(2, span, n0 + 64, dtype=np.uint64))
    keys = keys[rng.permutation(keys.size)[:n0]].astype(np.uint32)
    sc = FlixScenario("flix32_edge", 32, keys, max_size=8 * n0)
    live = np.sort(keys)
    new = _draw_new(rng, live, n0 // 4, 2, span - 1, 32, hot_ranges=4)
    present = live[rng.choice(live.size, n0 // 32, replace=False)]
    ins = np.union1d(new, present).astype(np.uint32)
    sc.stages.append(FlixStage("insert", ins, _values(rng, ins.size)))
    live = np.union1d(live, new)
    absent = _draw_new(rng, live, n0 // 32, 2, span - 1, 32, hot_ranges=2)
    dels = np.union1d(live[rng.choice(live.size, n0 // 4, replace=False)], absent).astype(np.uint32)
    sc.stages.append(FlixStage("remove", dels))
    live = np.setdiff1d(live, dels)
    lp, spr = _probes(rng, live, dels, 2, span - 1, 32, 1 << 11, 1 << 11)
    sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr))
    # a contiguous block of live keys deleted: whole buckets become empty
    start = int(rng.integers(live.size // 4, live.size // 2))
    block = live[start:start + 200]
    sc.stages.append(FlixStage("remove", block.astype(np.uint32)))
    live = np.setdiff1d(live, block)
    gap = rng.integers(int(block[0]), int(block[-1]) + 1, 128, dtype=np.uint64)
    lp, spr = _probes(rng, live, block, 2, span - 1, 32, 1 << 11, 1 << 11, (gap,))
    zero = ("zero_successor",)
    lost = ("zero_successor", "lost_in_rebuild")
    sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr, quirks=zero))
    sc.stages.append(FlixStage("rebuild"))
    sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr, quirks=lost))
    sc.stages.append(FlixStage("remove", live.astype(np.uint32)))
    sc.stages.append(FlixStage("probe", lookup_probes=lp, successor_probes=spr, quirks=lost))
    return sc


def allowed(stage: FlixStage, name: str, exact, ref):
    """Mask of the positions where the reference's answer may differ from the
    exact (std::map) answer in this probe stage, by documented class only:
      zero_successor   a successor probe inside emptied buckets reads 0 in the
                       reference (its own driver check skips a 0 result,
                       FliX/benchmarks_updates.cuh:160-162);
      lost_in_rebuild  after a rebuild that followed emptied buckets, the
                       reference misses keys that are live (lookup reads
                       not_found)."""
    exact, ref = np.asarray(exact), np.asarray(ref)
    mask = np.zeros(exact.shape, bool)
    if name == "successor" and "zero_successor" in stage.quirks:
        mask |= (ref == 0) & (exact != 0)
    if name == "lookup" and "lost_in_rebuild" in stage.quirks:
        mask |= (ref == NOT_FOUND) & (exact != NOT_FOUND)
    return mask


def scenarios() -> list[FlixScenario]:
    return [main_scenario(), insert64_scenario(), edge_scenario()]


def digest(sc: FlixScenario) -> str:
    """sha256 of every input array of the scenario, in order: a fixture records
    it so that a replay on another numpy build fails loudly if the seeded
    inputs ever come out different."""
    import hashlib

    h = hashlib.sha256()
    h.update(np.ascontiguousarray(sc.build_keys).tobytes())
    for st in sc.stages:
        h.update(st.kind.encode())
        for a in (st.keys, st.values, st.lookup_probes, st.successor_probes):
            if a is not None:
                h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()
