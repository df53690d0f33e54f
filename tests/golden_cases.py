"""Loads the reference-generated golden fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py from the reference's own GPULSMOpt engine and
FliX bucket layer) as replayable cases: the update operations, the
configuration, the queries and the reference's answers."""
from __future__ import annotations

import importlib
import os
from dataclasses import dataclass, field

import numpy as np

import flix_scenarios as FS
from scenarios import bulk_build_stages, forced_validation_steps, key_for_index, rollover_ops, capacity_ops, \
    sweep_lookup_queries, sweep_range_queries, validation_queries

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@dataclass
class Probe:
    queries: np.ndarray
    expect: dict  # answer name -> reference output
    lo: np.ndarray | None = None
    hi: np.ndarray | None = None


@dataclass
class Case:
    name: str
    config: dict
    stages: list = field(default_factory=list)  # (ops, Probe | None)


def available() -> bool:
    return os.path.exists(os.path.join(GOLDEN, "forced_validation.npz"))


def _load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def _ops_from(z):
    ops, pos = [], 0
    for kind, size in zip(z["op_kind"], z["op_size"]):
        size = int(size)
        k = z["op_keys"][pos:pos + size]
        v = z["op_vals"][pos:pos + size]
        pos += size
        ops.append(("insert", k, v) if kind == 0 else ("erase", k))
    return ops


def cases():
    out = []
    z = _load("forced_validation.npz")
    c = Case("forced_validation", {"max_elements": 1 << 20})
    for name, ops, expected, removed in forced_validation_steps():
        q, _ = validation_queries(expected, removed)
        assert np.array_equal(q, z[f"{name}_queries"])
        c.stages.append((ops, Probe(q, {k: z[f"{name}_{k}"] for k in
                                        ("lookup", "lookup_found_values", "lookup_found", "successor")})))
    out.append(c)

    z = _load("rollover.npz")
    ops, q, _ = rollover_ops()
    out.append(Case("rollover", {"max_elements": 512, "batch_capacity": 4, "level_zero_capacity": 64},
                    [(ops, Probe(q, {k: z[k] for k in ("lookup", "lookup_found_values", "lookup_found",
                                                        "successor", "range_sum")},
                                 np.array([0, 10, 200], np.uint32), np.array([255, 20, 100], np.uint32)))]))

    for seed in (11, 12, 13):
        z = _load(f"random_s{seed}.npz")
        out.append(Case(f"random_s{seed}", {"max_elements": 1 << 16, "batch_capacity": int(z["batch_capacity"][0])},
                        [(_ops_from(z), Probe(z["queries"], {k: z[k] for k in (
                            "lookup", "lookup_found_values", "lookup_found", "successor", "range_sum")},
                            z["lo"], z["hi"]))]))

    z = _load("paper_sweep.npz")
    n = int(z["n"][0])
    keys = key_for_index(np.arange(n))
    ops = [("insert", keys[b:b + (1 << 16)], np.ones(1 << 16, np.uint32)) for b in range(0, n, 1 << 16)]
    c = Case("paper_sweep", {"max_elements": n})
    hits = sweep_lookup_queries(1 << 14, n, True, 3)
    misses = sweep_lookup_queries(1 << 14, n, False, 4)
    lo8, hi8 = sweep_range_queries(1 << 13, n, 8, 5)
    lo1k, hi1k = sweep_range_queries(1 << 12, n, 1024, 6)
    c.stages.append((ops, Probe(hits, {"lookup": z["lookup_hits"]})))
    c.stages.append(([], Probe(misses, {"lookup": z["lookup_misses"]})))
    c.stages.append(([], Probe(np.zeros(0, np.uint32), {"range_sum": z["range_r8"]}, lo8, hi8)))
    c.stages.append(([], Probe(np.zeros(0, np.uint32), {"range_sum": z["range_r1024"]}, lo1k, hi1k)))
    out.append(c)

    z = _load("lsm_small_scale2.npz")
    W = importlib.import_module("gpu-lsm-tree_b200.workloads")
    w = W.lsm_small(scale=2)
    out.append(Case("lsm_small_scale2", {"max_elements": 1 << 18, "batch_capacity": 1 << 14},
                    [(w.ops, Probe(w.lookups, {"lookup": z["lookup"]})),
                     ([], Probe(np.zeros(0, np.uint32), {"range_sum": z["range_sum"]}, w.range_lo, w.range_hi))]))
    return out


def capacity_case():
    z = _load("capacity.npz")
    return {"accepted": int(z["accepted"][0]), "status": int(z["status"][0]),
            "loop_error": str(z["loop_error"][0]), "after_error": str(z["after_error"][0]),
            "queries": z["queries"], "lookup": z["lookup"], "ops": capacity_ops()}


def bulk_available() -> bool:
    return os.path.exists(os.path.join(GOLDEN, "bulk_build.npz"))


def bulk_case():
    """[(op, Probe)] for the bulk-build fixture; op is ("bulk"|"insert", keys,
    values) or ("erase", keys)."""
    z = _load("bulk_build.npz")
    out = []
    for i, (op, q, lo, hi) in enumerate(bulk_build_stages()):
        out.append((op, Probe(q, {k: z[f"s{i}_{k}"] for k in ("lookup", "lookup_found_values", "lookup_found",
                                                                "successor", "range_sum")}, lo, hi)))
    return out


def flix_available() -> bool:
    return all(os.path.exists(os.path.join(GOLDEN, f"{sc}.npz"))
               for sc in ("flix32_main", "flix64_insert", "flix32_edge"))


def flix_cases():
    """[(FlixScenario, {answer name: reference output})]; the recorded input
    digest must match the regenerated scenario."""
    out = []
    for sc in FS.scenarios():
        z = _load(f"{sc.name}.npz")
        assert str(z["digest"][0]) == FS.digest(sc), f"{sc.name}: regenerated inputs differ from the fixture's"
        out.append((sc, {k: z[k] for k in z.files}))
    return out
