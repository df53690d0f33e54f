"""Times the reference's own GPULSMOpt kernels (oracle/_ref, compiled from the
reference header) and this library on the same workload and the same GPU.

    python tests/bench_vs_reference.py [--scale S] [--out FILE]

Workload: the at-scale LSM configuration (64 insert batches of 2^20 with a
2^18-key delete batch after every 4th, 2^24 lookups, 2^20 range sums, 2^20
successor queries), sizes divided by 2^S.  Both engines get the same device
buffers; every phase is timed with CUDA events on the launching stream, best
of three repetitions, and all answers are compared for equality.
Test infrastructure: it loads oracle/_ref, so it lives under tests/.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle.refgpu import RefGPULSMOpt  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def timed(fn, reps=3):
    best = float("inf")
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=0)
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    gl = importlib.import_module("gpu-lsm-tree_b200")
    W = importlib.import_module("gpu-lsm-tree_b200.workloads")
    w = W.lsm_scale(args.scale)
    ops = [(o[0], dev(o[1]), dev(o[2]) if o[0] == "insert" else None) for o in w.ops]
    q = dev(w.lookups)
    lo, hi = dev(w.range_lo), dev(w.range_hi)
    nq, nr = w.lookups.size, w.range_lo.size
    max_el = w.inserted_keys + w.erased_keys
    results = {"workload": w.name, "scale": args.scale}
    outs = {}
    batch = 1 << (20 - args.scale)
    engines = {
        # the reference adapter's configuration: batch capacity = the batch,
        # level zero = one 16-batch epoch (FliX/impl_gpulsmopt.cuh:37-70)
        "reference": lambda: RefGPULSMOpt(max_el, batch, batch * 16),
        "ours": lambda: gl.GPULSMOpt(gl.DictionaryConfig(max_elements=max_el)),
    }
    for name, make in engines.items():
        d = make()
        upd_keys = w.inserted_keys + w.erased_keys

        def updates():
            d.clear()
            for kind, k, v in ops:
                d.insert(k, v) if kind == "insert" else d.erase(k)
            if hasattr(d, "join"):  # ours: the last batches' merges complete
                d.join()

        t_upd = timed(updates)
        ov = torch.empty(nq, dtype=torch.int32, device="cuda")
        of = torch.empty(nq, dtype=torch.uint8, device="cuda")
        t_look = timed(lambda: d.lookup(q, ov, of))
        sums = torch.empty(nr, dtype=torch.int32, device="cuda")
        t_range = timed(lambda: d.range(lo, hi, sums))
        nsucc = min(nq, 1 << (20 - args.scale))
        sq = q[:nsucc]
        so = torch.empty(nsucc, dtype=torch.int32, device="cuda")
        t_succ = timed(lambda: d.successor(sq, so), reps=1)
        torch.cuda.synchronize()
        outs[name] = (ov.cpu().numpy(), of.cpu().numpy(), sums.cpu().numpy(), so.cpu().numpy())
        results[name] = {
            "update_ms": round(t_upd, 3), "insert_mkeys_s": round(upd_keys / t_upd / 1e3, 1),
            "lookup_ms": round(t_look, 3), "lookup_mops_s": round(nq / t_look / 1e3, 1),
            "range_sum_ms": round(t_range, 3), "range_mqueries_s": round(nr / t_range / 1e3, 2),
            "successor_ms": round(t_succ, 3), "successor_mops_s": round(nsucc / t_succ / 1e3, 2),
        }
        del d
        torch.cuda.empty_cache()
    same = all(np.array_equal(a, b) for a, b in zip(outs["reference"], outs["ours"]))
    results["answers_identical"] = bool(same)
    results["speedup"] = {k: round(results["reference"][k.replace("_x", "_ms")] / results["ours"][k.replace("_x", "_ms")], 2)
                          for k in ("update_x", "lookup_x", "range_sum_x", "successor_x")}
    line = json.dumps(results)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    if not same:
        sys.exit(1)


if __name__ == "__main__":
    main()
