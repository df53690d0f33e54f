"""CPU tests of the oracle: the reference's own known answers, a pure-Python
model on small random cases, and the paper-sweep protocol."""
import numpy as np
import pytest

from oracle import OracleFlix, OracleLSM
from scenarios import (NOT_FOUND, forced_validation_steps, key_for_index, range_digest, rollover_ops,
                       sweep_lookup_queries, sweep_range_queries, validation_queries)


def apply_ops(d, ops):
    for op in ops:
        if op[0] == "insert":
            d.insert(op[1], op[2])
        else:
            d.erase(op[1])


def test_forced_validation_scenarios():
    d = OracleLSM()
    for name, ops, expected, removed in forced_validation_steps():
        apply_ops(d, ops)
        q, want = validation_queries(expected, removed)
        got = d.lookup(q)
        assert np.array_equal(got, want), name
        vals, found = d.lookup(q, with_found=True)
        assert np.array_equal(found.astype(bool), want != NOT_FOUND) or name == "sparse_unique"
        assert np.array_equal(vals[found == 0], np.zeros(int((found == 0).sum()), np.uint32)), name


def test_rollover_scenario():
    ops, q, expected = rollover_ops()
    d = OracleLSM()
    apply_ops(d, ops)
    assert np.array_equal(d.lookup(q), expected)


class Model:
    """Pure-Python statement of the GPULSMOpt visible state (dict of live keys)."""

    def __init__(self):
        self.m = {}

    def insert(self, k, v):
        for a, b in zip(k.tolist(), v.tolist()):
            self.m[a] = b  # later input index wins

    def erase(self, k):
        for a in k.tolist():
            self.m.pop(a, None)

    def lookup(self, q):
        return np.array([self.m.get(x, NOT_FOUND) for x in q.tolist()], np.uint32)

    def sorted(self):
        ks = sorted(self.m)
        return np.array(ks, np.uint64), np.array([self.m[k] for k in ks], np.uint64)

    def range_sum(self, lo, hi):
        ks, vs = self.sorted()
        out = []
        for a, b in zip(lo.tolist(), hi.tolist()):
            if a > b:
                out.append(0)
                continue
            i, j = np.searchsorted(ks, a), np.searchsorted(ks, b, side="right")
            out.append(int(vs[i:j].sum()) & 0xFFFFFFFF)
        return np.array(out, np.uint32)

    def successor(self, q):
        ks, _ = self.sorted()
        out = []
        for x in q.tolist():
            i = np.searchsorted(ks, x)
            out.append(int(ks[i]) if i < ks.size else NOT_FOUND)
        return np.array(out, np.uint32)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_python_model(seed):
    rng = np.random.default_rng(seed)
    d, m = OracleLSM(), Model()
    universe = rng.integers(0, 1 << 32, 300, dtype=np.uint64).astype(np.uint32)
    universe[:4] = [0, 1, 0xFFFFFFFF, 0xFFFFFFFE]
    for step in range(40):
        n = int(rng.integers(0, 200))
        k = universe[rng.integers(0, universe.size, n)]
        if rng.random() < 0.3:
            d.erase(k)
            m.erase(k)
        else:
            v = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            d.insert(k, v)
            m.insert(k, v)
        q = np.concatenate([universe, rng.integers(0, 1 << 32, 50, dtype=np.uint64).astype(np.uint32)])
        assert np.array_equal(d.lookup(q), m.lookup(q))
        lo = universe[rng.integers(0, universe.size, 64)]
        hi = universe[rng.integers(0, universe.size, 64)]
        assert np.array_equal(d.range_sum(lo, hi), m.range_sum(lo, hi))
        assert np.array_equal(d.successor(q), m.successor(q))
        off, rk, rv = d.range_pairs(lo, hi)
        counts = d.range_count(lo, hi)
        assert np.array_equal(np.diff(off).astype(np.uint32), counts)
        sums = np.array([int(rv[off[i]:off[i + 1]].astype(np.uint64).sum()) & 0xFFFFFFFF
                         for i in range(lo.size)], np.uint32)
        assert np.array_equal(sums, d.range_sum(lo, hi))


def test_bulk_build_keeps_last_duplicate():
    d = OracleLSM()
    d.bulk_build(np.array([7, 3, 7, 7, 3], np.uint32), np.array([1, 2, 3, 4, 5], np.uint32))
    k, v = d.dump()
    assert k.tolist() == [3, 7] and v.tolist() == [5, 4]


def test_mixed_update_equals_rows_one_at_a_time():
    rng = np.random.default_rng(9)
    d, ref = OracleLSM(), {}
    d.bulk_build(np.arange(0, 200, 2, dtype=np.uint32), np.arange(100, dtype=np.uint32))
    ref.update({int(k): int(v) for k, v in zip(range(0, 200, 2), range(100))})
    for _ in range(20):
        n = int(rng.integers(1, 300))
        k = rng.integers(0, 220, n).astype(np.uint32)
        v = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        e = (rng.random(n) < 0.4).astype(np.uint8)
        d.update(k, v, e)
        for ki, vi, ei in zip(k.tolist(), v.tolist(), e.tolist()):
            if ei:
                ref.pop(ki, None)
            else:
                ref[ki] = vi
    dk, dv = d.dump()
    assert dk.tolist() == sorted(ref) and dv.tolist() == [ref[x] for x in sorted(ref)]


def test_range_sum_wraps_and_empty_ranges():
    d = OracleLSM()
    d.insert(np.array([10, 11, 12], np.uint32), np.array([0xFFFFFFFF, 0xFFFFFFFF, 3], np.uint32))
    assert d.range_sum([10, 12, 5], [12, 10, 9]).tolist() == [(2 * 0xFFFFFFFF + 3) & 0xFFFFFFFF, 0, 0]


def test_flix_oracle_rules():
    f = OracleFlix(64)
    f.build(np.array([10, 2, 30, 2], np.uint64))  # values = input index, first duplicate wins
    assert f.dump()[0].tolist() == [2, 10, 30] and f.dump()[1].tolist() == [1, 0, 2]
    f.insert(np.array([2, 5, 5], np.uint64), np.array([7, 8, 9], np.uint32))  # insert if absent
    assert f.lookup(np.array([2, 5, 11], np.uint64)).tolist() == [1, 8, NOT_FOUND]
    f.remove(np.array([10, 11], np.uint64))
    assert f.successor(np.array([3, 6, 31, 1 << 40], np.uint64)).tolist() == [5, 30, 0xFFFFFFFF, 0xFFFFFFFF]
    g = OracleFlix(32)
    g.build(np.array([5, 0xFFFFFFFE], np.uint64), np.array([1, 2], np.uint32))
    assert g.successor(np.array([6], np.uint64)).tolist() == [0xFFFFFFFE]


def test_paper_sweep_protocol():
    n = 1 << 16
    d = OracleLSM()
    keys = key_for_index(np.arange(n))
    for b in range(0, n, 1 << 13):
        d.insert(keys[b:b + (1 << 13)], np.ones(1 << 13, np.uint32))
    hits = sweep_lookup_queries(4096, n, True, 7)
    misses = sweep_lookup_queries(4096, n, False, 9)
    assert (d.lookup(hits) == 1).all()
    assert (d.lookup(misses) == NOT_FOUND).all()
    for expected_hits in (8, 1024):
        lo, hi = sweep_range_queries(2048, n, expected_hits, 11)
        sums = d.range_sum(lo, hi)
        assert np.array_equal(sums, d.range_count(lo, hi))  # values are 1
        assert abs(float(sums.mean()) - expected_hits) < 0.2 * expected_hits
        s, x = range_digest(sums)
        assert s == int(sums.sum())


def test_sweep_runner_inputs_match_the_sweep_protocol():
    """The paper-sweep runner generates the same keys, queries and digests as
    the sweep protocol restated in scenarios.py (FliX/paper_lsmu_sweep.cu)."""
    import importlib

    import scenarios as sc

    sw = importlib.import_module("gpu-lsm-tree_b200.sweep")
    i = np.arange(0, 1 << 16, 7, dtype=np.uint64)
    assert np.array_equal(sw.key_for_index(i), sc.key_for_index(i))
    for hits in (True, False):
        assert np.array_equal(sw.lookup_queries(4096, 1 << 20, hits, 0x10003),
                              sc.sweep_lookup_queries(4096, 1 << 20, hits, 0x10003))
    lo, hi = sw.range_queries(4096, 1 << 20, 1024, 0x30401)
    lo2, hi2 = sc.sweep_range_queries(4096, 1 << 20, 1024, 0x30401)
    assert np.array_equal(lo, lo2) and np.array_equal(hi, hi2)
    r = np.random.default_rng(3).integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)
    assert sw.range_digest(r, 77) == sc.range_digest(r, 77)


def test_updates_runner_writes_result_collector_long_form():
    """The updates runner's writer lays a table out as result_collector's
    write_csv(first_line_header, long_form, pack_columns) does
    (FliX/result_collector.h:172-296): the parameter columns in first-seen
    order, then DESCRIPTION and VALUE; one line per measurement, repeating the
    row's parameters, an empty field for a parameter the row lacks, values
    printed at precision 16 and booleans as 1/0."""
    import importlib

    ur = importlib.import_module("gpu-lsm-tree_b200.updates_runner")
    rc = ur.ResultCollector()
    rc.commit([("EXPERIMENT", "batches"), ("step", 0), ("do_insert", True)],
              [("probe_time_ms", 0.125), ("after_update_bytes", 4096)])
    rc.commit([("EXPERIMENT", "batches"), ("run", 1)], [("probe_time_ms", 1 / 3)])
    assert rc.long_form_packed() == (
        "EXPERIMENT, step, do_insert, run, DESCRIPTION, VALUE\n"
        "batches, 0, 1, , probe_time_ms, 0.125\n"
        "batches, 0, 1, , after_update_bytes, 4096\n"
        "batches, , , 1, probe_time_ms, 0.3333333333333333\n")
    try:
        rc.commit([("probe_time_ms", 1)], [])
    except ValueError:
        pass
    else:
        raise AssertionError("a measurement column reused as a parameter must be refused")


@pytest.mark.parametrize("engine", ["map", "lsm"])
def test_cpu_baselines_match_oracle(engine):
    """The CPU baselines timed beside the GPU (std::map, leveled OpenMP LSM)
    give the oracle's answers: upserts with the last write of a batch winning,
    erases, lookups with and without found flags, range pairs."""
    from oracle import CpuLsm, CpuMap, OracleLSM

    rng = np.random.default_rng(5)
    o = OracleLSM()
    e = CpuMap() if engine == "map" else CpuLsm(cap0=512, fan_in=3)
    universe = rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)
    universe[:3] = [0, 0xFFFFFFFF, 1]
    for step in range(60):
        n = int(rng.integers(1, 700))
        k = universe[rng.integers(0, universe.size, n)]
        if rng.random() < 0.3:
            o.erase(k)
            e.erase(k)
        else:
            v = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            o.insert(k, v)
            e.insert(k, v)
        if step % 10 == 9:
            q = np.concatenate([universe, rng.integers(0, 1 << 32, 500, dtype=np.uint64).astype(np.uint32)])
            assert np.array_equal(e.lookup(q), o.lookup(q))
            ev, ef = e.lookup(q, with_found=True)
            ov, of = o.lookup(q, with_found=True)
            assert np.array_equal(ev, ov) and np.array_equal(ef, of)
            lo = universe[rng.integers(0, universe.size, 300)]
            hi = np.minimum(lo.astype(np.uint64) + rng.integers(0, 1 << 30, 300, dtype=np.uint64),
                            0xFFFFFFFF).astype(np.uint32)
            lo[:2], hi[:2] = [9, 0], [3, 0xFFFFFFFF]
            for a, b in zip(e.range_pairs(lo, hi), o.range_pairs(lo, hi)):
                assert np.array_equal(a, b)
    if engine == "lsm":
        assert e.levels() >= 2  # the run carried down several levels
