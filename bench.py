"""Benchmark of the GPU dictionary hot path (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload lsm_scale|lsm_small] [--no-e2e] [--no-cpu]

A step is one pass of the at-scale LSM workload over a fresh dictionary:
64 insert batches of 2^20 u32 (key, value) pairs with a 2^18-key delete batch
after every 4th insert batch (2^26 + 2^22 updates), then 2^24 point lookups
(70% Zipf s=0.99 over inserted keys, 30% uniform) and 2^20 range queries that
return (key, value) pairs (offsets pass + pairs pass).  value = all operations
of the step (updated keys + lookups + range queries) / step time, in M ops/s;
per-phase rates (inserted keys/s, lookups/s, range queries/s) and per-batch
p50/p99 latencies ride along.  Inputs live in HBM before the timed region;
together they exceed the 126 MB L2, so no flush is needed between steps.

--impl reference times a CPU implementation of the path (the reference has no
CPU engine of its own): a multi-threaded leveled LSM with the path's semantics
on every host thread, on the same workload at the same size.  Under torchrun (N > 1) each rank runs
an independent dictionary on its own seeded data (replicas: the path has no
exchange step), rank 0 prints the aggregate.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "M lookups/s & M inserted keys/s at 2^26 keys vs plain form; p50/p99 request latency"
# DRAM bytes (read + write) of merge_kernel per algorithmic byte, from an ncu
# capture of `bench.py --case merge` (one 17.8M-row merge: 161.1 MB read,
# 128.0 MB written against 328.6 MB algorithmic; the rest of the writes were
# still in L2 when the kernel ended)
MERGE_TRAFFIC_RATIO = 0.880
LOOKUP_BYTES = 41  # algorithmic bytes per u32 point lookup (query + value + found + one row sector)
INSERT_BYTES = 16  # per inserted (key, value): read 8 + write 8 into the structure
DELETE_BYTES = 12
RANGE_BYTES = 76   # per range query (lo, hi, count + two boundary sectors) + 16 per returned pair


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="lsm_scale", choices=["lsm_scale", "lsm_small"])
    p.add_argument("--scale", type=int, default=0, help="divide sizes by 2^scale (development only)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-tenants", action="store_true")
    p.add_argument("--no-flix", action="store_true")
    p.add_argument("--flix-rounds", type=int, default=32)
    p.add_argument("--tenant-rounds", type=int, default=4)
    p.add_argument("--serving-seconds", type=float, default=2.0)
    p.add_argument("--case", default=None, choices=["merge", "admit", "serving-mix", "flix", "lookup"],
                   help="run one small profiling case instead of the benchmark (see profile_case)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(
        os.environ.get("LOCAL_RANK", 0))


def make_workload(W, name, scale, rank):
    if name == "lsm_small":
        w = W.lsm_small(scale)
    else:
        w = W.lsm_scale(scale)
    if rank:
        # replicas: each rank draws its own keys (same shapes, different seed stream)
        rng = np.random.default_rng(0x5EED + 7919 * rank)
        perm = rng.integers(0, 1 << 32, 1, dtype=np.uint64).astype(np.uint32)[0]
        w.ops = [(o[0], o[1] ^ perm, *o[2:]) for o in w.ops]
        w.lookups = w.lookups ^ perm
    return w


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def step_config(args, w, world):
    """The workload description both arms print (the same dict for the GPU arm
    and the CPU reference arm on the same configuration)."""
    return {"workload": w.name, "global_batch": (w.inserted_keys + w.erased_keys) * world,
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (no flush)",
            "value_definition": "(updated keys + lookups + range queries) per step / step time",
            "scale": args.scale}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    gl = importlib.import_module("gpu-lsm-tree_b200")
    W = importlib.import_module("gpu-lsm-tree_b200.workloads")
    lib = gl.load()
    w = make_workload(W, args.workload, args.scale, rank)

    def to_dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)

    ops_dev = [(o[0], to_dev(o[1]), to_dev(o[2]) if o[0] == "insert" else None) for o in w.ops]
    q = to_dev(w.lookups)
    lo, hi = to_dev(w.range_lo), to_dev(w.range_hi)
    nq, nr = w.lookups.size, w.range_lo.size
    out_v = torch.empty(nq, dtype=torch.int32, device=dev)
    out_f = torch.empty(nq, dtype=torch.uint8, device=dev)
    offsets = torch.empty(nr + 1, dtype=torch.int64, device=dev)
    max_el = w.inserted_keys + w.erased_keys
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=max_el))
    stream = torch.cuda.current_stream(dev)
    pairs = [None, None]

    def step(ev=None, batch_ev=None):
        d.clear()
        if ev is not None:
            ev["start"].record(stream)
        if batch_ev is not None:
            batch_ev[0].record(stream)
        for i, (kind, k, v) in enumerate(ops_dev):
            if kind == "insert":
                d.insert(k, v)
            else:
                d.erase(k)
            if batch_ev is not None:  # latency of one batch alone: admission and merges
                d.join()
                batch_ev[i + 1].record(stream)
        # updates return once admitted (their merges overlap the next batch's
        # admission); the update phase ends when every merge has completed
        d.join()
        if ev is not None:
            ev["update"].record(stream)
        d.lookup(q, out_v, out_f)
        if ev is not None:
            ev["lookup"].record(stream)
        d.range_offsets(lo, hi, offsets)
        d.range_pairs(lo, hi, offsets, pairs[0], pairs[1])
        if ev is not None:
            ev["range"].record(stream)

    # size the range output from one untimed pass
    d.clear()
    for kind, k, v in ops_dev:
        d.insert(k, v) if kind == "insert" else d.erase(k)
    d.range_offsets(lo, hi, offsets)
    total_pairs = int(offsets[nr].item())
    pairs[0] = torch.empty(max(total_pairs, 1), dtype=torch.int32, device=dev)
    pairs[1] = torch.empty(max(total_pairs, 1), dtype=torch.int32, device=dev)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    def new_events():
        mk = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        return {"start": mk(), "update": mk(), "lookup": mk(), "range": mk()}

    events = [new_events() for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = lib.gpulsm_launch_count()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for s in range(args.steps):
            step(events[s])
        t1.record(stream)
        torch.cuda.synchronize(dev)
    launches = lib.gpulsm_launch_count() - launches0
    # One more step of the same workload with every batch joined before the
    # next (no overlap of its merges with the next admission): per-batch
    # latency, and the dominant kernel (merge_kernel) timed alone, every merge
    # launch bracketed by CUDA events on the dictionary's merge stream (events
    # between chained launches would slow the timed steps, so they stay out)
    batch_ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(ops_dev) + 1)]
    d.kernel_timing(True)
    d.kernel_timing_read()
    step(batch_ev=batch_ev)
    merge_timing = d.kernel_timing_read()
    d.kernel_timing(False)
    torch.cuda.synchronize(dev)
    total_ms = t0.elapsed_time(t1)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()

    # per-phase times (device events on the launching stream)
    upd_ms, look_ms, range_ms = [], [], []
    for ev in events:
        upd_ms.append(ev["start"].elapsed_time(ev["update"]))
        look_ms.append(ev["update"].elapsed_time(ev["lookup"]))
        range_ms.append(ev["lookup"].elapsed_time(ev["range"]))
    batch_ms = [(ops_dev[i][0], batch_ev[i].elapsed_time(batch_ev[i + 1])) for i in range(len(ops_dev))]
    ms_per_step = total_ms / args.steps
    upd_keys = w.inserted_keys + w.erased_keys
    ops_per_step = upd_keys + nq + nr
    value = ops_per_step * world / (ms_per_step * 1e-3) / 1e6
    ins_lat = [b for k, b in batch_ms if k == "insert"]
    upd = float(np.median(upd_ms))
    look = float(np.median(look_ms))
    rng_ms = float(np.median(range_ms))
    peak, peak_kind = peaks()
    lookup_gbs = nq * LOOKUP_BYTES / (look * 1e-3) / 1e9
    range_gbs = (nr * RANGE_BYTES + total_pairs * 16) / (rng_ms * 1e-3) / 1e9
    update_gbs = (w.inserted_keys * INSERT_BYTES + w.erased_keys * DELETE_BYTES) / (upd * 1e-3) / 1e9
    phases = {"update": (upd, update_gbs), "lookup": (look, lookup_gbs), "range": (rng_ms, range_gbs)}
    ml = max(merge_timing["launches"], 1)
    merge_gbs = merge_timing["bytes"] / max(merge_timing["ms"], 1e-9) / 1e6
    roofline = {"bound": "hbm", "kernel": "lsm::merge_kernel",
                "measured": "one extra step with every batch joined, CUDA events per launch",
                "achieved": round(merge_gbs, 1), "peak": peak,
                "unit": "GB/s", "frac": round(merge_gbs / peak, 4), "peak_source": peak_kind,
                "traffic": None if MERGE_TRAFFIC_RATIO is None else
                round(MERGE_TRAFFIC_RATIO * merge_timing["bytes"] / ml),
                "launches": merge_timing["launches"],
                "ms_per_launch": round(merge_timing["ms"] / ml, 4),
                "algorithmic_bytes_per_launch": round(merge_timing["bytes"] / ml),
                "share_of_update_ms": round(merge_timing["ms"] / upd, 3),
                "phases_gbs": {k: round(v[1], 1) for k, v in phases.items()}}

    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "M ops/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded PCG64; shapes of the at-scale LSM configuration)",
        "config": step_config(args, w, world),
        "parts": {
            "update_mkeys_s": round(upd_keys / (upd * 1e-3) / 1e6, 1),
            "inserted_mkeys_s": round(w.inserted_keys / (upd * 1e-3) / 1e6, 1),
            "lookup_mops_s": round(nq / (look * 1e-3) / 1e6, 1),
            "range_mqueries_s": round(nr / (rng_ms * 1e-3) / 1e6, 2),
            "range_pairs_per_step": total_pairs,
            "update_ms": round(upd, 3), "lookup_ms": round(look, 3), "range_ms": round(rng_ms, 3),
            "insert_batch_ms_p50": round(float(np.percentile(ins_lat, 50)), 4),
            "insert_batch_ms_p99": round(float(np.percentile(ins_lat, 99)), 4),
        },
        "roofline": roofline,
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }

    result["lookup_modes"] = lookup_modes(gl, ops_dev, q, out_v, out_f, max_el, look, stream)
    if not args.no_e2e:
        result["e2e"] = e2e_ours(args, gl, w, dev, total_pairs, max_el)
    if not args.no_tenants:
        result["tenants"] = tenants_leg(args, gl, dev)
    if not args.no_flix:
        result["flix"] = flix_leg(args, gl, W, dev)
    if not args.no_serving:
        del d, ops_dev, q, lo, hi, out_v, out_f, offsets, pairs
        torch.cuda.empty_cache()
        result["serving"] = serving_leg(args, gl, w, dev)
    if rank == 0 and not args.no_cpu:
        result["cpu_baseline"] = cpu_baseline(args, W, w)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def lookup_modes(gl, ops_dev, q, out_v, out_f, max_el, directory_ms, stream):
    """The step's 2^24 lookups over the same final dictionary in each search
    mode: radix directory (the plain form), learned position models (levels of
    >= 2^22 rows), plain binary search.  Each mode: the step's updates, then
    four lookup launches, best of them (the first also builds what its reads
    need: directories, models), CUDA events on the launching stream; answers
    compared with the step's.  `step_directory_ms` is the step's own lookup
    phase (its first read: directory builds included)."""
    import torch

    res = {"step_directory_ms": round(directory_ms, 4)}
    ref_v, ref_f = out_v.clone(), out_f.clone()
    for name, mode in (("directory", 0), ("learned", 1), ("binary", 2)):
        d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=max_el, search_mode=mode))
        for kind, k, v in ops_dev:
            d.insert(k, v) if kind == "insert" else d.erase(k)
        d.join()
        best = float("inf")
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            d.lookup(q, out_v, out_f)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        res[f"{name}_ms"] = round(best, 4)
        res[f"{name}_same_answers"] = bool(torch.equal(out_v, ref_v) and torch.equal(out_f, ref_f))
        d.close()
    directory_ms = res["directory_ms"]
    res["learned_speedup_vs_directory"] = round(directory_ms / res["learned_ms"], 3)
    res["learned_speedup_vs_binary"] = round(res["binary_ms"] / res["learned_ms"], 3)
    return res


def flix_leg(args, gl, W, dev):
    """FliX-style updatable sorted index at its configured size: bulk build of
    2^28 sorted u64 keys (geometric gaps, mean 16), then 32 rounds of 2^22
    inserts (half uniform, half in 1024 hot ranges), 2^21 deletes and 2^24
    uniform successor probes, after one untimed warm-up round; bucket routing
    by binary search over the bucket maxima (plain) against the learned
    piecewise-linear model with 4096 segments (learned).  Every round is timed
    with CUDA events; the allocation region's use is read after each round."""
    import torch

    w = W.flix_fast(0, rounds=args.flix_rounds + 1)
    u64 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(dev)  # noqa: E731
    u32 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)  # noqa: E731
    keys = u64(w.build_keys)
    # the reference's interface takes sorted batches (its driver sorts before
    # the timed calls); probes are timed both pre-sorted (ordered lookups, as
    # the published numbers) and unsorted (sort inside the call)
    rounds = []
    for i, v, d, p in w.rounds:
        o = np.argsort(i, kind="stable")
        rounds.append((u64(i[o]), u32(v[o]), u64(np.sort(d)), u64(np.sort(p)), u64(p)))
    n_build = w.build_keys.size
    cap = n_build + len(w.rounds) * rounds[0][0].numel()
    out = torch.empty(rounds[0][3].numel(), dtype=torch.int64, device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    res = {"rounds_timed": args.flix_rounds, "build_keys": int(n_build)}
    warm = gl.FlixIndex(key_bits=64, max_elements=1 << 20)
    warm.build(keys[: 1 << 20])
    torch.cuda.synchronize()
    warm.close()
    for name, mode in (("plain", 0), ("learned", 1)):
        idx = gl.FlixIndex(key_bits=64, search_mode=mode, max_elements=cap)
        idx.build(keys, max_size=cap)  # first build maps the index's device memory; time a rebuild from keys
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        idx.build(keys, max_size=cap)
        e1.record()
        torch.cuda.synchronize()
        build_ms = e0.elapsed_time(e1)
        per = {"insert_ms": [], "delete_ms": [], "ordered_successor_ms": [], "unsorted_successor_ms": [],
               "region_used_nodes": []}
        n_ins = n_del = n_suc = 0
        for r, (ins, vals, dels, sprobes, probes) in enumerate(rounds):
            a, b, c, d, e = ev(), ev(), ev(), ev(), ev()
            a.record()
            idx.insert(ins, vals)
            b.record()
            idx.remove(dels)
            c.record()
            idx.lookups_successor(sprobes, out)
            d.record()
            idx.successor(probes, out)
            e.record()
            torch.cuda.synchronize()
            if r == 0:
                continue
            per["insert_ms"].append(a.elapsed_time(b))
            per["delete_ms"].append(b.elapsed_time(c))
            per["ordered_successor_ms"].append(c.elapsed_time(d))
            per["unsorted_successor_ms"].append(d.elapsed_time(e))
            per["region_used_nodes"].append(idx.allocation_state()["used_nodes"])
            n_ins += ins.numel()
            n_del += dels.numel()
            n_suc += probes.numel()
        alloc = idx.allocation_state()
        t_ins, t_del = sum(per["insert_ms"]), sum(per["delete_ms"])
        t_ord, t_suc = sum(per["ordered_successor_ms"]), sum(per["unsorted_successor_ms"])
        ni, nd, ns = rounds[0][0].numel(), rounds[0][2].numel(), rounds[0][4].numel()
        res[name] = {"build_ms": round(build_ms, 2), "build_mkeys_s": round(n_build / build_ms / 1e3, 1),
                     "insert_mkeys_s": round(n_ins / t_ins / 1e3, 1), "delete_mkeys_s": round(n_del / t_del / 1e3, 1),
                     "ordered_successor_mops_s": round(n_suc / t_ord / 1e3, 1),
                     "unsorted_successor_mops_s": round(n_suc / t_suc / 1e3, 1), "status": idx.status(),
                     "keys_after": idx.size(), "resident_gb": round(idx.gpu_resident_bytes() / 1e9, 2),
                     "allocation_region": alloc,
                     # per timed round, in order: G keys/s (or G probes/s) and region nodes used
                     "per_round": {
                         "insert_gkeys_s": [round(ni / t / 1e6, 2) for t in per["insert_ms"]],
                         "delete_gkeys_s": [round(nd / t / 1e6, 2) for t in per["delete_ms"]],
                         "ordered_successor_gops_s": [round(ns / t / 1e6, 1) for t in per["ordered_successor_ms"]],
                         "region_used_nodes": per["region_used_nodes"]}}
        idx.close()
        torch.cuda.synchronize()
    res["learned_successor_speedup"] = round(res["learned"]["ordered_successor_mops_s"] /
                                             res["plain"]["ordered_successor_mops_s"], 3)
    res["learned_insert_speedup"] = round(res["learned"]["insert_mkeys_s"] / res["plain"]["insert_mkeys_s"], 3)
    return res


def tenant_round(rng, sizes, lo=6, hi=16):
    """One round of the multi-tenant configuration: per tenant a batch of
    log-uniform size in [2^lo, 2^hi], keys uniform in the tenant's key span
    [0, size) (upserts, so a tenant never outgrows its size)."""
    n = np.exp(rng.uniform(lo * np.log(2), hi * np.log(2), sizes.size)).astype(np.int64)
    off = np.zeros(sizes.size + 1, np.int64)
    off[1:] = np.cumsum(n)
    span = np.repeat(sizes.astype(np.float64), n)
    keys = (rng.random(int(off[-1])) * span).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, int(off[-1]), dtype=np.uint64).astype(np.uint32)
    return keys, vals, off


def tenants_leg(args, gl, dev):
    """Multi-tenant batched mode: 4096 dictionaries of log-uniform size in
    [2^10, 2^20], per-tenant batches log-uniform in [2^6, 2^16], one persistent
    merge launch per round replayed from a CUDA graph, tile / fan-in / fanout
    picked by the autotuner on a 512-tenant sample; against the plain form
    (one dictionary per tenant, a call per tenant) timed on a 256-tenant sample."""
    import torch

    tune = importlib.import_module("gpu-lsm-tree_b200.autotune")
    rng = np.random.default_rng(17)
    T = 4096
    sizes = np.exp(rng.uniform(10 * np.log(2), 20 * np.log(2), T)).astype(np.uint64)

    def dev_round(r):
        k, v, off = r
        return (torch.from_numpy(k.view(np.int32)).to(dev), torch.from_numpy(v.view(np.int32)).to(dev),
                torch.from_numpy(off).to(dev))

    # autotune on a sample of the workload (cached by signature)
    ts = 512
    s_sizes = sizes[:ts]
    s_rounds = [dev_round(tenant_round(rng, s_sizes, 6, 12)) for _ in range(2)]
    s_lookup = (torch.from_numpy(rng.integers(0, ts, 1 << 16).astype(np.int32)).to(dev),
                torch.from_numpy(rng.integers(0, 1 << 20, 1 << 16).astype(np.int32)).to(dev))
    best = tune.autotune(s_sizes * 2 + 8, s_rounds, s_lookup, max(int(r[2][-1].item()) for r in s_rounds),
                         cache_path=None)
    rounds = [tenant_round(rng, sizes) for _ in range(args.tenant_rounds + 1)]
    max_round = max(int(r[2][-1]) for r in rounds)
    pool = gl.TenantPool(sizes * 2 + 8, max_round, best["tile"], best["fan_in"], best["fanout"])
    kbuf = torch.empty(max_round, dtype=torch.int32, device=dev)
    vbuf = torch.empty(max_round, dtype=torch.int32, device=dev)
    obuf = torch.empty(T + 1, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(dev)
    keys_total, ms_total = 0, 0.0
    for i, r in enumerate(rounds):
        k, v, off = dev_round(r)
        n = int(r[2][-1])
        with torch.cuda.stream(stream):
            kbuf[:n].copy_(k)
            vbuf[:n].copy_(v)
            obuf.copy_(off)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pool.insert_round(kbuf, vbuf, obuf, stream=stream, graph=True)
            e1.record(stream)
        stream.synchronize()
        if i > 0:  # round 0 warms up (and captures the graph)
            keys_total += n
            ms_total += e0.elapsed_time(e1)
    nq = 1 << 24
    tid = torch.from_numpy(rng.integers(0, T, nq).astype(np.int32)).to(dev)
    qk = torch.from_numpy((rng.random(nq) * sizes[tid.cpu().numpy()].astype(np.float64)).astype(np.uint32).view(np.int32)).to(dev)
    out = torch.empty(nq, dtype=torch.int32, device=dev)
    pool.lookup(tid, qk, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pool.lookup(tid, qk, out)
    e1.record()
    torch.cuda.synchronize()
    look_ms = e0.elapsed_time(e1)
    status = pool.status()
    resident = pool.gpu_resident_bytes()
    pool.close()
    del kbuf, vbuf
    # plain form: one dictionary per tenant, a call per tenant, on a sample
    ps = 256
    plain = [gl.GPULSMOpt(gl.DictionaryConfig(max_elements=int(c) + 8, batch_capacity=1 << 16)) for c in sizes[:ps]]
    r = rounds[1]
    k, v, off = dev_round(r)
    pk = 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for t in range(ps):
        a, b = int(off[t]), int(off[t + 1])
        plain[t].insert(k[a:b], v[a:b])
        pk += b - a
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    for d in plain:
        d.close()
    return {
        "tenants": T, "total_size_keys": int(sizes.sum()), "rounds_timed": args.tenant_rounds,
        "keys_per_round": int(keys_total / max(args.tenant_rounds, 1)),
        "tuning": {"tile": best["tile"], "fan_in": best["fan_in"], "fanout": best["fanout"]},
        "insert_mkeys_s": round(keys_total / (ms_total * 1e-3) / 1e6, 1),
        "round_ms": round(ms_total / max(args.tenant_rounds, 1), 3),
        "lookup_mops_s": round(nq / (look_ms * 1e-3) / 1e6, 1),
        "plain_form_insert_mkeys_s": round(pk / (plain_ms * 1e-3) / 1e6, 1),
        "plain_form_sample_tenants": ps,
        "speedup_vs_plain_form": round((keys_total / ms_total) / (pk / plain_ms), 2),
        "resident_gb": round(resident / 1e9, 2), "status": status,
    }


def serving_leg(args, gl, w, dev):
    """The serving mode over the same dictionary: every inserted key loaded,
    a 16 GB device budget, requests of log-uniform size in [1, 2^16] keys
    (60% lookup, 20% insert, 10% erase, 10% range sum; Zipf s=1.1 keys).
    Peak = the best closed loop of 64, 128 and 256 requests in flight (the
    curve is reported: more requests in flight make larger rounds, until the
    device saturates); latency = open-loop Poisson arrivals at half the peak
    request rate (host submit to results in host buffers).  Run once with each
    level search: the radix directory (plain) and the learned position model
    (learned), and with staged updates."""
    import torch

    keys = np.concatenate([o[1] for o in w.ops if o[0] == "insert"])
    secs = args.serving_seconds
    out = {"dictionary_keys": int(keys.size), "budget_gb": 16}
    # plain / learned: search modes of the levels, update runs direct (admitted
    # and merged at once, the round waiting for its merges); plain_staged:
    # update runs admitted into staging runs by captured CUDA graphs and merged
    # into the levels when the staging slots fill
    for name, mode, staged in (("plain", 0, False), ("learned", 1, False), ("plain_staged", 0, True)):
        # serving requests are small: a small level 0 (2^17 rows, fan-in 4) keeps
        # a run's merge proportional to the run instead of to a 4M-row level
        srv = gl.Server(gl.DictionaryConfig(max_elements=keys.size + w.erased_keys + (1 << 24), search_mode=mode,
                                            level_zero_capacity=1 << 17),
                        budget_bytes=16 << 30, max_round_keys=1 << 20, depth=3)
        srv.set_staged_updates(staged)
        kd = torch.from_numpy(keys.view(np.int32)).to(dev)
        vd = torch.arange(keys.size, dtype=torch.int32, device=dev)
        srv.bulk_build(kd, vd)
        del kd, vd
        srv.run_load(keys, rate_per_s=0, seconds=0.3, max_outstanding=64, seed=3)  # warm-up
        curve, peak, peak_out = {}, None, 0
        for outstanding in (64, 128, 256):
            r = srv.run_load(keys, rate_per_s=0, seconds=0.75 * secs, max_outstanding=outstanding, seed=4)
            curve[str(outstanding)] = {"mkeys_s": round(r["keys"] / max(r["wall_s"], 1e-9) / 1e6, 1),
                                       "p99_ms": round(r["p99_us"] / 1e3, 4)}
            if peak is None or r["keys"] / r["wall_s"] > peak["keys"] / peak["wall_s"]:
                peak, peak_out = r, outstanding
        peak_rate = peak["completed"] / max(peak["wall_s"], 1e-9)
        half = srv.run_load(keys, rate_per_s=0.5 * peak_rate, seconds=secs, seed=5)
        srv.close()
        out[name] = {
            "peak_mkeys_s": round(peak["keys"] / max(peak["wall_s"], 1e-9) / 1e6, 1),
            "peak_requests_s": round(peak_rate, 1), "peak_outstanding": peak_out,
            "closed_loop_curve": curve,
            "load_requests_s": round(0.5 * peak_rate, 1),
            "mkeys_s": round(half["keys"] / max(half["wall_s"], 1e-9) / 1e6, 1),
            "p50_ms": round(half["p50_us"] / 1e3, 4), "p99_ms": round(half["p99_us"] / 1e3, 4),
            "max_ms": round(half["max_us"] / 1e3, 4),
            # the worst round at half load: its device time and the worker's launch time
            "max_round_gpu_ms": round(half["max_round_gpu_us"] / 1e3, 4),
            "max_launch_ms": round(half["max_launch_us"] / 1e3, 4),
            "peak_p50_ms": round(peak["p50_us"] / 1e3, 4), "peak_p99_ms": round(peak["p99_us"] / 1e3, 4),
            "mean_round_keys": round(half["mean_round_keys"], 1),
            "peak_mean_round_keys": round(peak["mean_round_keys"], 1),
            "peak_gpu_busy_frac": round(peak["gpu_busy_s"] / max(peak["wall_s"], 1e-9), 3),
            "peak_host_launch_frac": round(peak["host_launch_s"] / max(peak["wall_s"], 1e-9), 3),
            # where a peak round's time goes: device time per request kind (the
            # merges still running when a round ends are charged to insert;
            # sampled on every eighth round), the submitting thread's copy into
            # the server's pinned ring, the completion thread's result scatter
            "peak_kind_gpu_frac": {k: round(v / max(peak["wall_s"], 1e-9), 3)
                                   for k, v in zip(("lookup", "insert", "erase", "range"), peak["kind_gpu_s"])},
            "peak_host_copy_frac": round(peak["host_copy_s"] / max(peak["wall_s"], 1e-9), 3),
            "peak_host_scatter_frac": round(peak["host_scatter_s"] / max(peak["wall_s"], 1e-9), 3),
            "requests": int(half["completed"]), "rejected": int(half["rejected"] + peak["rejected"]),
            "peak_graph_update_runs": int(peak["graph_updates"]), "peak_stage_flushes": int(peak["stage_flushes"]),
            "peak_graph_lookup_rounds": int(peak["graph_rounds"]), "peak_rounds": int(peak["rounds"]),
        }
    return out


def e2e_ours(args, gl, w, dev, total_pairs, max_el):
    """Same step through the public API with HOST buffers: every step copies
    its inputs from pinned host memory and reads every result back."""
    import torch

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).pin_memory()  # noqa: E731
    host_ops = [(o[0], pin(o[1]), pin(o[2]) if o[0] == "insert" else None) for o in w.ops]
    hq, hlo, hhi = pin(w.lookups), pin(w.range_lo), pin(w.range_hi)
    nq, nr = w.lookups.size, w.range_lo.size
    h_out_v = torch.empty(nq, dtype=torch.int32).pin_memory()
    h_out_f = torch.empty(nq, dtype=torch.uint8).pin_memory()
    h_off = torch.empty(nr + 1, dtype=torch.int64).pin_memory()
    h_pk = torch.empty(max(total_pairs, 1), dtype=torch.int32).pin_memory()
    h_pv = torch.empty(max(total_pairs, 1), dtype=torch.int32).pin_memory()
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=max_el))
    dk = [(o[0], torch.empty_like(o[1], device=dev), torch.empty_like(o[2], device=dev) if o[2] is not None else None)
          for o in host_ops]
    q = torch.empty(nq, dtype=torch.int32, device=dev)
    lo = torch.empty(nr, dtype=torch.int32, device=dev)
    hi = torch.empty(nr, dtype=torch.int32, device=dev)
    ov = torch.empty(nq, dtype=torch.int32, device=dev)
    of = torch.empty(nq, dtype=torch.uint8, device=dev)
    off = torch.empty(nr + 1, dtype=torch.int64, device=dev)
    pk = torch.empty(max(total_pairs, 1), dtype=torch.int32, device=dev)
    pv = torch.empty(max(total_pairs, 1), dtype=torch.int32, device=dev)
    h2d = sum(o[1].numel() * 4 + (o[2].numel() * 4 if o[2] is not None else 0) for o in host_ops) + (nq + 2 * nr) * 4
    d2h = nq * 5 + (nr + 1) * 8 + total_pairs * 8

    def step():
        d.clear()
        for (kind, hk, hv), (_, gk, gv) in zip(host_ops, dk):
            gk.copy_(hk, non_blocking=True)
            if kind == "insert":
                gv.copy_(hv, non_blocking=True)
                d.insert(gk, gv)
            else:
                d.erase(gk)
        q.copy_(hq, non_blocking=True)
        d.lookup(q, ov, of)
        h_out_v.copy_(ov, non_blocking=True)
        h_out_f.copy_(of, non_blocking=True)
        lo.copy_(hlo, non_blocking=True)
        hi.copy_(hhi, non_blocking=True)
        d.range_offsets(lo, hi, off)
        d.range_pairs(lo, hi, off, pk, pv)
        h_off.copy_(off, non_blocking=True)
        h_pk[:total_pairs].copy_(pk[:total_pairs], non_blocking=True)
        h_pv[:total_pairs].copy_(pv[:total_pairs], non_blocking=True)

    steps = max(1, min(args.steps, 3))
    step()
    torch.cuda.synchronize(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        step()
    e.record()
    torch.cuda.synchronize(dev)
    ms = s.elapsed_time(e) / steps
    ops = w.inserted_keys + w.erased_keys + nq + nr
    d.close()
    return {"value": round(ops / (ms * 1e-3) / 1e6, 2), "unit": "M ops/s", "ms_per_step": round(ms, 3),
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": steps}


def cpu_step(w, engine):
    """One pass of the workload through a CPU engine with the path's semantics
    (updates, lookups with found flags, range pairs)."""
    for op in w.ops:
        engine.insert(op[1], op[2]) if op[0] == "insert" else engine.erase(op[1])
    engine.lookup(w.lookups, with_found=True)
    engine.range_pairs(w.range_lo, w.range_hi)


def cpu_baseline(args, W, w):
    """The CPU baselines over the same workload: the multi-threaded leveled LSM
    on every host thread at full size (one pass, seconds), and a single-thread
    std::map over a 1/16-size sample of the same shape."""
    from oracle import CpuLsm, CpuMap

    threads = os.cpu_count() or 1
    t = time.perf_counter()
    cpu_step(w, CpuLsm())
    dt = time.perf_counter() - t
    ops = w.inserted_keys + w.erased_keys + w.lookups.size + w.range_lo.size
    ws = W.lsm_scale(args.scale + 4) if args.workload == "lsm_scale" else W.lsm_small(args.scale + 4)
    t = time.perf_counter()
    cpu_step(ws, CpuMap())
    dts = time.perf_counter() - t
    ops_s = ws.inserted_keys + ws.erased_keys + ws.lookups.size + ws.range_lo.size
    return {"value": round(ops / dt / 1e6, 3), "unit": "M ops/s", "cores": threads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"the same workload at full size, one pass, {dt:.1f} s (multi-threaded leveled CPU LSM)",
            "std_map_single_thread": {"value": round(ops_s / dts / 1e6, 3), "unit": "M ops/s", "cores": 1,
                                      "sample": f"same shape at 1/16 of every size, one pass, {dts:.1f} s"}}


def run_reference(args):
    """CPU implementation of the path (the oracle restatement on every host core)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import CpuLsm

    W = importlib.import_module("gpu-lsm-tree_b200.workloads")
    used = os.cpu_count() or 1
    w = make_workload(W, args.workload, args.scale, 0)
    for _ in range(args.warmup):
        cpu_step(w, CpuLsm())
    t = time.perf_counter()
    for _ in range(args.steps):
        cpu_step(w, CpuLsm())
    dt = (time.perf_counter() - t) / args.steps
    ops = w.inserted_keys + w.erased_keys + w.lookups.size + w.range_lo.size
    value = ops / dt / 1e6
    sample = ("the whole workload every step at full size, on a fresh multi-threaded leveled CPU LSM "
              "(parallel-mode std::sort of each batch, OpenMP run merges and query batches)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "M ops/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": step_config(args, w, 1),
        "cpu_baseline": {"value": round(value, 3), "unit": "M ops/s", "cores": used, "kind": "port",
                         "cpu_model": cpu_model(), "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "M ops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def profile_case(args):
    """Small, self-contained cases for ncu captures (a few GB on the device):
    merge       a 2^24-key level plus one 2^20-key batch, then full-width
                range counts that compact both into one: a single 17M-row merge
                whose inputs and output exceed L2;
    admit       8 + 64 x (clear + insert of a 2^20-key batch): the admission
                kernels alone, no merges;
    serving-mix the serving loop over 2^26 keys, closed loop for 0.3 s with
                the default request mix;
    flix        FliX at 1/4 of its sizes: 2^26 sorted u64 keys built, then 2
                rounds of 2^20 sorted inserts, 2^19 sorted deletes and 2^22
                sorted successor probes (plain bucket routing);
    lookup      the at-scale step's 2^24 lookups (70% Zipf hits) against one
                level bulk-built from its 2^26 inserted pairs, twice."""
    import torch

    gl = importlib.import_module("gpu-lsm-tree_b200")
    rng = np.random.default_rng(1)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    def keys(n):
        return rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)

    if args.case == "merge":
        d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 25, batch_capacity=1 << 20))
        base = keys(1 << 24)
        d.bulk_build(dev(base), dev(np.arange(base.size, dtype=np.uint32)))
        k = keys(1 << 20)
        d.insert(dev(k), dev(np.arange(k.size, dtype=np.uint32)))
        # 1024 full-width ranges: the covered rows outweigh a compaction
        out = torch.empty(1024, dtype=torch.int32, device="cuda")
        d.range_count(dev(np.zeros(1024, np.uint32)), dev(np.full(1024, 0xFFFFFFFF, np.uint32)), out)
        torch.cuda.synchronize()
        print(json.dumps({"case": "merge", "rows": d.size()[0], "status": d.canonical_carry_status()}))
    elif args.case == "admit":
        d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 22, batch_capacity=1 << 20))
        batches = [dev(keys(1 << 20)) for _ in range(8)]
        vals = dev(np.arange(1 << 20, dtype=np.uint32))
        for i in range(8):  # buffers allocated, kernels loaded
            d.clear()
            d.insert(batches[i], vals)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(64):
            d.clear()
            d.insert(batches[i % 8], vals)
        d.join()
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"case": "admit", "ms_per_batch": round(e0.elapsed_time(e1) / 64, 4),
                          "status": d.canonical_carry_status()}))
    elif args.case == "lookup":
        # the at-scale step's 2^24 lookups against one level bulk-built from its
        # 2^26 inserted pairs (the erases are not applied)
        W = importlib.import_module("gpu-lsm-tree_b200.workloads")
        w = W.lsm_scale(0)
        ks = np.concatenate([o[1] for o in w.ops if o[0] == "insert"])
        vs = np.concatenate([o[2] for o in w.ops if o[0] == "insert"])
        d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=ks.size))
        d.bulk_build(dev(ks), dev(vs))
        q = dev(w.lookups)
        out_v = torch.empty(q.numel(), dtype=torch.int32, device="cuda")
        out_f = torch.empty(q.numel(), dtype=torch.uint8, device="cuda")
        for _ in range(2):
            d.lookup(q, out_v, out_f)
        torch.cuda.synchronize()
        print(json.dumps({"case": "lookup", "queries": q.numel(), "hits": int(out_f.sum().item()),
                          "status": d.canonical_carry_status()}))
    elif args.case == "flix":
        W = importlib.import_module("gpu-lsm-tree_b200.workloads")
        w = W.flix_fast(2, rounds=2)
        u64 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()  # noqa: E731
        cap = w.build_keys.size + 2 * (1 << 20)
        idx = gl.FlixIndex(key_bits=64, max_elements=cap)
        idx.build(u64(w.build_keys), max_size=cap)
        out = torch.empty(1 << 22, dtype=torch.int64, device="cuda")
        for ins, vals, dels, probes in w.rounds:
            o = np.argsort(ins, kind="stable")
            idx.insert(u64(ins[o]), torch.from_numpy(vals[o].view(np.int32)).cuda())
            idx.remove(u64(np.sort(dels)))
            idx.lookups_successor(u64(np.sort(probes)), out)
        torch.cuda.synchronize()
        print(json.dumps({"case": "flix", "status": idx.status()}))
        idx.close()
    else:
        base = keys(1 << 26)
        srv = gl.Server(gl.DictionaryConfig(max_elements=(1 << 26) + (1 << 25), level_zero_capacity=1 << 17),
                        budget_bytes=16 << 30)
        srv.bulk_build(dev(base), torch.arange(base.size, dtype=torch.int32, device="cuda"))
        srv.run_load(base, rate_per_s=0, seconds=0.2, seed=2)
        st = srv.run_load(base, rate_per_s=0, seconds=0.3, seed=3)
        srv.close()
        print(json.dumps({"case": "serving-mix", "completed": st["completed"], "p99_us": round(st["p99_us"], 1)}))


if __name__ == "__main__":
    a = parse()
    if a.case:
        profile_case(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
