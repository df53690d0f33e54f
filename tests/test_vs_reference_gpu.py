"""This library against the reference's own GPU kernels on the same B200, the
same inputs and the same device buffers: every answer identical, and the
headline speed-ups measured with CUDA events (best of three).

  * GPULSMOpt (oracle/_ref/libref_gpulsmopt.so, compiled from GPULSMOpt.cuh):
    the at-scale LSM configuration at full size - 64 insert batches of 2^20
    keys with a 2^18-key erase batch after every 4th (2^26 + 2^22 updates),
    2^24 Zipf lookups, 2^20 range sums, 2^20 successor queries.  The target
    holds as assertions: inserted keys/s and lookups/s at least 1.5x the
    reference's insert (GPULSMOpt.cuh:5836) and lookup (:5850).
  * FliX (oracle/_ref/libref_flix.so, compiled from
    FliX/impl_cg_rtx_index_updates.cuh): the updatable-index configuration's
    shapes at 1/16 of its size with 32-bit keys - bulk build of 2^24 sorted
    keys (geometric gaps, mean 16), then 4 rounds of a 2^18-key insert batch
    (half in 1024 hot ranges), a 2^17-key delete batch and 2^20 sorted
    successor probes plus 2^20 ordered lookups, every answer compared; the
    ratios are recorded.  32-bit keys because the reference's 64-bit ordered
    lookup and tiled delete read values at the 4-byte-key position
    (extract_offset_node<smallsize>, FliX/coarse_granular_lookups_tile_bulk.cuh:403,
    FliX/coarse_granular_deletes_tiles.cuh:1201) and so return wrong values.

The measured figures go to the test log and, when GPULSM_REPORT_DIR names a
folder, to vs_reference_gpulsmopt.json / vs_reference_flix.json there.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from oracle import refgpu

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _timed(fn, reps=3):
    import torch

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


def _report(name, results):
    line = json.dumps(results)
    print(line)
    out = os.environ.get("GPULSM_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"vs_reference_{name}.json"), "w") as f:
            f.write(line + "\n")


@pytest.mark.skipif(not refgpu.available(), reason="reference GPULSMOpt engine not built (oracle/_ref)")
def test_gpulsmopt_at_scale_same_answers_and_target_speedups(gl, cuda, workloads):
    import torch

    w = workloads.lsm_scale(0)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    ops = [(o[0], dev(o[1]), dev(o[2]) if o[0] == "insert" else None) for o in w.ops]
    q = dev(w.lookups)
    lo, hi = dev(w.range_lo), dev(w.range_hi)
    nq, nr = w.lookups.size, w.range_lo.size
    nsucc = 1 << 20
    max_el = w.inserted_keys + w.erased_keys
    batch = 1 << 20
    engines = {
        # the reference adapter's configuration: batch capacity = the batch,
        # level zero = one 16-batch epoch (FliX/impl_gpulsmopt.cuh:37-70)
        "reference": lambda: refgpu.RefGPULSMOpt(max_el, batch, batch * 16),
        "ours": lambda: gl.GPULSMOpt(gl.DictionaryConfig(max_elements=max_el)),
    }
    results = {"workload": w.name, "device": torch.cuda.get_device_name(0)}
    outs = {}
    for name, make in engines.items():
        d = make()

        def updates():
            d.clear()
            for kind, k, v in ops:
                d.insert(k, v) if kind == "insert" else d.erase(k)
            if hasattr(d, "join"):  # ours: the last batches' merges complete
                d.join()

        t_upd = _timed(updates)
        ov = torch.empty(nq, dtype=torch.int32, device="cuda")
        of = torch.empty(nq, dtype=torch.uint8, device="cuda")
        t_look = _timed(lambda: d.lookup(q, ov, of))
        sums = torch.empty(nr, dtype=torch.int32, device="cuda")
        t_range = _timed(lambda: d.range(lo, hi, sums))
        sq = q[:nsucc]
        so = torch.empty(nsucc, dtype=torch.int32, device="cuda")
        t_succ = _timed(lambda: d.successor(sq, so))
        torch.cuda.synchronize()
        outs[name] = (ov.cpu().numpy(), of.cpu().numpy(), sums.cpu().numpy(), so.cpu().numpy())
        results[name] = {
            "update_ms": round(t_upd, 3),
            "update_mkeys_s": round((w.inserted_keys + w.erased_keys) / t_upd / 1e3, 1),
            "inserted_mkeys_s": round(w.inserted_keys / t_upd / 1e3, 1),
            "lookup_ms": round(t_look, 3), "lookup_mops_s": round(nq / t_look / 1e3, 1),
            "range_sum_ms": round(t_range, 3), "range_mqueries_s": round(nr / t_range / 1e3, 2),
            "successor_ms": round(t_succ, 3), "successor_mops_s": round(nsucc / t_succ / 1e3, 1),
        }
        del d
        torch.cuda.empty_cache()
    names = ("lookup values", "lookup found flags", "range sums", "successors")
    same = {n: bool(np.array_equal(a, b)) for n, a, b in zip(names, outs["reference"], outs["ours"])}
    results["answers_identical"] = same
    results["speedup"] = {k: round(results["reference"][f"{k}_ms"] / results["ours"][f"{k}_ms"], 2)
                          for k in ("update", "lookup", "range_sum", "successor")}
    _report("gpulsmopt", results)
    assert all(same.values()), same
    assert results["speedup"]["update"] >= 1.5, results
    assert results["speedup"]["lookup"] >= 1.5, results


@pytest.mark.skipif(not refgpu.flix_available(), reason="reference FliX bucket layer not built (oracle/_ref)")
def test_flix_same_answers_as_reference_kernels(gl, cuda, workloads):
    import torch

    w = workloads.flix_fast(scale=4, rounds=4, key_bits=32)
    n0 = w.build_keys.size
    max_size = 2 * (n0 + sum(r[0].size for r in w.rounds))

    def dk(a):  # 32-bit keys
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()

    def d32(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()

    # the reference's interface takes sorted unique batches and sorted probes
    rounds, host_rounds = [], []
    for ins, vals, dels, probes in w.rounds:
        o = np.argsort(ins, kind="stable")
        sp = np.unique(probes[probes < np.uint64(0xFFFFFFFC)])
        rounds.append((dk(ins[o]), d32(vals[o]), dk(np.sort(dels)), dk(sp), sp.size))
        host_rounds.append((ins, dels, sp))
    live = np.sort(w.build_keys)
    keys = dk(w.build_keys)
    # warm-up on separate small indexes: an insert and a remove are timed once
    # per round (they change the index), so each engine's first-call costs
    # (kernel loading, first stream-ordered allocations) are paid here
    # (a round-0-sized insert and remove, so that their workspaces reach full size)
    warm_keys = np.sort(w.build_keys[: 1 << 18])
    for eng in (refgpu.RefFlix(32), gl.FlixIndex(key_bits=32, max_elements=1 << 21)):
        wk = dk(warm_keys)
        eng.build_bucket_layer_only(wk, 1 << 21) if isinstance(eng, refgpu.RefFlix) else \
            eng.build_bucket_layer_only(wk, max_size=1 << 21)
        eng.insert(rounds[0][0], rounds[0][1])
        eng.remove(dk(warm_keys[::2]))
        torch.cuda.synchronize()
    ref = refgpu.RefFlix(32)
    ours = gl.FlixIndex(key_bits=32, max_elements=max_size)
    t = {"reference": {"insert_ms": 0.0, "remove_ms": 0.0, "successor_ms": 0.0, "lookup_ms": 0.0},
         "ours": {"insert_ms": 0.0, "remove_ms": 0.0, "successor_ms": 0.0, "lookup_ms": 0.0}}
    ref.build_bucket_layer_only(keys, max_size)
    ours.build_bucket_layer_only(keys, max_size=max_size)
    torch.cuda.synchronize()
    mismatches, reference_quirks = [], []
    n_ins = n_del = n_probe = 0
    for r, (ins, vals, dels, probes, n) in enumerate(rounds):
        n_ins += ins.numel()
        n_del += dels.numel()
        n_probe += n
        for name, eng in (("reference", ref), ("ours", ours)):
            t[name]["insert_ms"] += _timed(lambda: eng.insert(ins, vals), reps=1)
            t[name]["remove_ms"] += _timed(lambda: eng.remove(dels), reps=1)
        outs = {}
        for name, eng in (("reference", ref), ("ours", ours)):
            so = torch.empty(n, dtype=torch.int32, device="cuda")
            lo = torch.empty(n, dtype=torch.int32, device="cuda")
            t[name]["successor_ms"] += _timed(lambda: eng.lookups_successor(probes, so))
            t[name]["lookup_ms"] += _timed(lambda: eng.lookups_ordered(probes, lo))
            outs[name] = (so.cpu().numpy(), lo.cpu().numpy())
        # the exact successors (std::map answers) from the live set kept on the host
        h_ins, h_dels, h_sp = host_rounds[r]
        live = np.setdiff1d(np.union1d(live, h_ins), h_dels, assume_unique=True)
        pos = np.searchsorted(live, h_sp)
        exact = np.where(pos < live.size, live[np.minimum(pos, live.size - 1)], 0xFFFFFFFF).astype(np.uint32)
        ours_s = outs["ours"][0].view(np.uint32)
        ref_s = outs["reference"][0].view(np.uint32)
        assert np.array_equal(ours_s, exact), f"round {r}: our successors differ from the exact answers"
        for what, a, b in zip(("successor", "lookup"), outs["reference"], outs["ours"]):
            bad = np.flatnonzero(a != b)
            if what == "successor" and bad.size:
                # ours equals the exact answer everywhere (asserted above), so every
                # disagreement is the reference's; recorded with an example, by
                # class: a successor read as 0 (the quirk its own driver check skips,
                # FliX/benchmarks_updates.cuh:160-162) or another wrong key
                ex = ref_s[bad]
                for cls, sel in (("zero_successor", ex == 0), ("wrong_successor", ex != 0)):
                    if sel.any():
                        j = bad[sel][0]
                        reference_quirks.append({"round": r, "class": cls, "count": int(sel.sum()),
                                                 "probe": int(h_sp[j]), "reference": int(ref_s[j]),
                                                 "exact": int(exact[j])})
                bad = bad[:0]
            if bad.size:
                mismatches.append((r, what, int(bad.size)))
    total_ref, total_ours = ref.total_keys(), ours.size()
    results = {"workload": "flix: bulk build of 2^24 sorted u32 keys, 4 rounds of 2^18 inserts (half in 1024 hot "
                           "ranges), 2^17 deletes, 2^20 sorted successor probes and ordered lookups",
               "device": torch.cuda.get_device_name(0), "mismatches": mismatches,
               "reference_quirks": reference_quirks,
               "total_keys": {"reference": total_ref, "ours": total_ours}}
    for name in t:
        results[name] = {k: round(v, 3) for k, v in t[name].items()}
        results[name].update(insert_gkeys_s=round(n_ins / t[name]["insert_ms"] / 1e6, 2),
                             remove_gkeys_s=round(n_del / t[name]["remove_ms"] / 1e6, 2),
                             successor_gops_s=round(n_probe / t[name]["successor_ms"] / 1e6, 2),
                             lookup_gops_s=round(n_probe / t[name]["lookup_ms"] / 1e6, 2))
    results["speedup"] = {k: round(t["reference"][f"{k}_ms"] / t["ours"][f"{k}_ms"], 2)
                          for k in ("insert", "remove", "successor", "lookup")}
    _report("flix", results)
    ref.close()
    assert not mismatches, mismatches
    assert total_ref == total_ours
