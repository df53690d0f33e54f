"""Generates the golden fixtures in this folder by running the REFERENCE's own
engines on a CUDA GPU: GPULSMOpt (oracle/_ref/libref_gpulsmopt.so, compiled
from the reference header GPULSMOpt.cuh) and FliX's bucket layer
(oracle/_ref/libref_flix.so, compiled from FliX/impl_cg_rtx_index_updates.cuh).

    python tests/golden/make_golden.py [--out DIR] [--only lsm,bulk,flix]

Each fixture stores the scenario's inputs (or the seed that regenerates them)
and the reference's outputs.  tests/test_golden.py checks the CPU oracle
against them (pinning the oracle to the reference) and tests/test_golden_gpu.py
checks our engine against them.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.refgpu import RefError, RefFlix, RefGPULSMOpt  # noqa: E402
from scenarios import (bulk_build_stages, capacity_ops, forced_validation_steps, key_for_index,  # noqa: E402
                       rollover_ops, sweep_lookup_queries, sweep_range_queries, validation_queries)
import flix_scenarios as FS  # noqa: E402

W = importlib.import_module("gpu-lsm-tree_b200.workloads")


def dev(a):
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()


def host(t, dtype=np.uint32):
    return t.cpu().numpy().view(dtype)


def run_ops(ref, ops):
    for op in ops:
        if op[0] == "insert":
            ref.insert(dev(op[1]), dev(op[2]))
        else:
            ref.erase(dev(op[1]))


def queries(ref, q, lo=None, hi=None):
    out = {}
    v = torch.empty(max(q.size, 1), dtype=torch.int32, device="cuda")
    f = torch.empty(max(q.size, 1), dtype=torch.uint8, device="cuda")
    ref.lookup(dev(q), v)
    out["lookup"] = host(v)[: q.size].copy()
    ref.lookup(dev(q), v, f)
    out["lookup_found_values"] = host(v)[: q.size].copy()
    out["lookup_found"] = host(f, np.uint8)[: q.size].copy()
    ref.successor(dev(q), v)
    out["successor"] = host(v)[: q.size].copy()
    if lo is not None:
        s = torch.empty(max(lo.size, 1), dtype=torch.int32, device="cuda")
        ref.range(dev(lo), dev(hi), s)
        out["range_sum"] = host(s)[: lo.size].copy()
    return out


def flatten_ops(ops):
    kinds = np.array([0 if o[0] == "insert" else 1 for o in ops], np.uint8)
    sizes = np.array([o[1].size for o in ops], np.uint64)
    keys = np.concatenate([o[1] for o in ops]) if ops else np.zeros(0, np.uint32)
    vals = np.concatenate([o[2] if o[0] == "insert" else np.zeros(o[1].size, np.uint32) for o in ops])
    return dict(op_kind=kinds, op_size=sizes, op_keys=keys, op_vals=vals)


def random_ops(seed, batch_capacity, steps=40):
    rng = np.random.default_rng(seed)
    universe = rng.integers(0, 1 << 32, 3000, dtype=np.uint64).astype(np.uint32)
    universe[:6] = [0, 1, 2, 0xFFFFFFFF, 0xFFFFFFFE, 0x80000000]
    ops = []
    for _ in range(steps):
        n = int(rng.integers(1, 3 * batch_capacity))
        k = universe[rng.integers(0, universe.size, n)]
        if rng.random() < 0.3:
            ops.append(("erase", k))
        else:
            ops.append(("insert", k, rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)))
    q = np.concatenate([universe, rng.integers(0, 1 << 32, 1000, dtype=np.uint64).astype(np.uint32)])
    lo = universe[rng.integers(0, universe.size, 500)]
    hi = np.minimum(lo.astype(np.uint64) + rng.integers(0, 1 << 28, 500, dtype=np.uint64), 0xFFFFFFFF).astype(np.uint32)
    lo[:2] = [5, 0]
    hi[:2] = [4, 0xFFFFFFFF]
    return ops, q, lo, hi


def dev_keys(a):
    a = np.ascontiguousarray(a)
    view = {np.dtype(np.uint32): np.int32, np.dtype(np.uint64): np.int64}[a.dtype]
    return torch.from_numpy(a.view(view)).cuda()


def make_bulk():
    """GPULSMOpt bulk_build with duplicate keys, updates after it, a bulk build
    over a dictionary holding updates, and an empty bulk build."""
    ref = RefGPULSMOpt(1 << 17, 1 << 12)
    data = {}
    for i, (op, q, lo, hi) in enumerate(bulk_build_stages()):
        if op[0] == "bulk":
            ref.bulk_build(dev(op[1]), dev(op[2]))
        elif op[0] == "insert":
            ref.insert(dev(op[1]), dev(op[2]))
        else:
            ref.erase(dev(op[1]))
        for k2, v2 in queries(ref, q, lo, hi).items():
            data[f"s{i}_{k2}"] = v2
    data["status"] = np.array([ref.status()], np.uint32)
    np.savez_compressed(os.path.join(HERE, "bulk_build.npz"), **data)
    ref.close()


def make_flix():
    """FliX bucket-layer scenarios (tests/flix_scenarios.py) through the
    reference's own FliX kernels: every probe stage records the ordered lookup
    and successor answers and the key count the reference reports."""
    for sc in FS.scenarios():
        kdt = np.uint32 if sc.key_bits == 32 else np.uint64
        tdt = torch.int32 if sc.key_bits == 32 else torch.int64
        ref = RefFlix(sc.key_bits)
        ref.build_bucket_layer_only(dev_keys(sc.build_keys), sc.max_size)
        torch.cuda.synchronize()
        data = {"digest": np.array([FS.digest(sc)]), "build_total_keys": np.array([ref.total_keys()], np.uint64)}
        p = 0
        for st in sc.stages:
            if st.kind == "insert":
                ref.insert(dev_keys(st.keys), dev(st.values))
            elif st.kind == "remove":
                ref.remove(dev_keys(st.keys))
            elif st.kind == "rebuild":
                ref.rebuild_bucket_layer_only()
            else:
                if st.lookup_probes is not None:
                    probes = st.lookup_probes
                    out = torch.empty(max(probes.size, 1), dtype=torch.int32, device="cuda")
                    ref.lookups_ordered(dev_keys(probes), out)
                    data[f"p{p}_lookup"] = host(out)[: probes.size].copy()
                probes = st.successor_probes
                out = torch.empty(max(probes.size, 1), dtype=tdt, device="cuda")
                ref.lookups_successor(dev_keys(probes), out)
                data[f"p{p}_successor"] = host(out, kdt)[: probes.size].copy()
                torch.cuda.synchronize()
                data[f"p{p}_total_keys"] = np.array([ref.total_keys()], np.uint64)
                p += 1
        torch.cuda.synchronize()
        data["allocation_state"] = np.array(ref.allocation_state(), np.uint64)
        np.savez_compressed(os.path.join(HERE, f"{sc.name}.npz"), **data)
        ref.close()


def main():
    global HERE
    if "--out" in sys.argv:
        HERE = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(HERE, exist_ok=True)
    only = set(sys.argv[sys.argv.index("--only") + 1].split(",")) if "--only" in sys.argv else {"lsm", "bulk", "flix"}
    torch.cuda.init()
    if "bulk" in only:
        make_bulk()
    if "flix" in only:
        make_flix()
    if "lsm" not in only:
        torch.cuda.synchronize()
        print("golden fixtures written to", HERE)
        return
    # 1. forced validation (cumulative, one dictionary)
    ref = RefGPULSMOpt(1 << 20)
    data = {}
    for i, (name, ops, expected, removed) in enumerate(forced_validation_steps()):
        run_ops(ref, ops)
        q, _ = validation_queries(expected, removed)
        res = queries(ref, q)
        data[f"{name}_queries"] = q
        for k2, v2 in res.items():
            data[f"{name}_{k2}"] = v2
    data["status"] = np.array([ref.status()], np.uint32)
    np.savez_compressed(os.path.join(HERE, "forced_validation.npz"), **data)
    ref.close()

    # 2. multi-level rollover
    ops, q, _ = rollover_ops()
    ref = RefGPULSMOpt(512, 4, 64)
    run_ops(ref, ops)
    res = queries(ref, q, np.array([0, 10, 200], np.uint32), np.array([255, 20, 100], np.uint32))
    np.savez_compressed(os.path.join(HERE, "rollover.npz"), queries=q, status=np.array([ref.status()], np.uint32),
                        **res)
    ref.close()

    # 3. capacity exhaustion behaviour
    ref = RefGPULSMOpt(1024, 4, 1024)
    accepted = 0
    loop_error = ""
    for op in capacity_ops():
        try:
            ref.insert(dev(op[1]), dev(op[2]))
            accepted += 1
        except RefError as e:
            loop_error = str(e)
            break
    status = ref.status()
    after = ""
    try:
        ref.insert(dev(np.array([1], np.uint32)), dev(np.array([1], np.uint32)))
    except RefError as e:
        after = str(e)
    q = np.arange(0, accepted * 4 + 8, dtype=np.uint32)
    res = queries(ref, q)
    np.savez_compressed(os.path.join(HERE, "capacity.npz"), accepted=np.array([accepted]),
                        status=np.array([status], np.uint32), loop_error=np.array([loop_error]),
                        after_error=np.array([after]), queries=q, **res)
    ref.close()

    # 4. random small scenarios with several batch capacities
    for seed, bc, lz in ((11, 64, 0), (12, 256, 0), (13, 4096, 0)):
        ops, q, lo, hi = random_ops(seed, bc)
        ref = RefGPULSMOpt(1 << 16, bc, lz)
        run_ops(ref, ops)
        res = queries(ref, q, lo, hi)
        np.savez_compressed(os.path.join(HERE, f"random_s{seed}.npz"), batch_capacity=np.array([bc]),
                            level_zero=np.array([lz]), queries=q, lo=lo, hi=hi,
                            status=np.array([ref.status()], np.uint32), **flatten_ops(ops), **res)
        ref.close()

    # 5. paper-sweep protocol (values 1: range sum == range count)
    n = 1 << 18
    ref = RefGPULSMOpt(n)
    keys = key_for_index(np.arange(n))
    for b in range(0, n, 1 << 16):
        ref.insert(dev(keys[b:b + (1 << 16)]), dev(np.ones(1 << 16, np.uint32)))
    hits = sweep_lookup_queries(1 << 14, n, True, 3)
    misses = sweep_lookup_queries(1 << 14, n, False, 4)
    lo8, hi8 = sweep_range_queries(1 << 13, n, 8, 5)
    lo1k, hi1k = sweep_range_queries(1 << 12, n, 1024, 6)
    out = {}
    for nm, qq in (("hits", hits), ("misses", misses)):
        v = torch.empty(qq.size, dtype=torch.int32, device="cuda")
        ref.lookup(dev(qq), v)
        out[f"lookup_{nm}"] = host(v).copy()
    for nm, (a, b) in (("r8", (lo8, hi8)), ("r1024", (lo1k, hi1k))):
        s = torch.empty(a.size, dtype=torch.int32, device="cuda")
        ref.range(dev(a), dev(b), s)
        out[f"range_{nm}"] = host(s).copy()
    np.savez_compressed(os.path.join(HERE, "paper_sweep.npz"), n=np.array([n]), **out)
    ref.close()

    # 6. small configuration shape at 1/4 size: lookups and range sums
    w = W.lsm_small(scale=2)
    ref = RefGPULSMOpt(1 << 18, 1 << 14)
    run_ops(ref, w.ops)
    v = torch.empty(w.lookups.size, dtype=torch.int32, device="cuda")
    ref.lookup(dev(w.lookups), v)
    s = torch.empty(w.range_lo.size, dtype=torch.int32, device="cuda")
    ref.range(dev(w.range_lo), dev(w.range_hi), s)
    np.savez_compressed(os.path.join(HERE, "lsm_small_scale2.npz"), lookup=host(v).copy(),
                        range_sum=host(s).copy())
    ref.close()
    torch.cuda.synchronize()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
