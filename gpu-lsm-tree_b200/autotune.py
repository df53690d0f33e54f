"""Autotuner of the multi-tenant batched dictionary.

Searches merge tile size {256 .. 4096}, merge fan-in {2, 4, 8} (rounds of
updates a tenant's delta run gathers before it is merged into the main run)
and search fanout {8, 16, 32} (the B-ary fence tree of every run) on a sample
of the real workload: for every candidate a fresh pool replays the sample
rounds and a lookup batch, timed with CUDA events on the launching stream.
The best candidate (lowest time per (updated key + lookup)) is cached in a
JSON file keyed by the workload's signature, so later pools reuse it.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os

import numpy as np

from .tenants import TenantPool

TILES = (256, 512, 1024, 2048, 4096)
FAN_INS = (2, 4, 8)
FANOUTS = (8, 16, 32)
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "gpulsm_b200", "tenant_tuning.json")


def signature(capacities, rounds, lookup_count: int) -> str:
    caps = np.asarray(capacities, dtype=np.uint64)
    sizes = [int(r[2][-1].item()) if hasattr(r[2], "item") else int(r[2][-1]) for r in rounds]
    desc = f"{caps.size}:{int(caps.sum())}:{int(caps.max())}:{sum(sizes) // max(len(sizes), 1)}:{lookup_count}"
    return hashlib.sha1(desc.encode()).hexdigest()[:16]


def _time_candidate(capacities, max_round, rounds, lookup, tile, fan_in, fanout, repeats):
    import torch

    pool = TenantPool(capacities, max_round, tile, fan_in, fanout)
    tid, keys = lookup
    out = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(repeats):
        for k, v, off in rounds:
            pool.insert_round(k, v, off)
    pool.lookup(tid, keys, out)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e)
    if pool.status() != 0:
        ms = float("inf")
    pool.close()
    return ms


def autotune(capacities, rounds, lookup, max_round: int, cache_path: str | None = DEFAULT_CACHE,
             tiles=TILES, fan_ins=FAN_INS, fanouts=FANOUTS, repeats: int = 1) -> dict:
    """rounds: list of (keys, values, offsets) CUDA tensors; lookup: (tenant_ids, keys).
    Returns {"tile", "fan_in", "fanout", "ms", "table"} and caches the winner."""
    sig = signature(capacities, rounds, lookup[1].numel())
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if sig in cache:
        return cache[sig] | {"cached": True}
    table = []
    for tile, fan_in, fanout in itertools.product(tiles, fan_ins, fanouts):
        ms = _time_candidate(capacities, max_round, rounds, lookup, tile, fan_in, fanout, repeats)
        table.append({"tile": tile, "fan_in": fan_in, "fanout": fanout, "ms": ms})
    best = min(table, key=lambda r: r["ms"])
    result = {"tile": best["tile"], "fan_in": best["fan_in"], "fanout": best["fanout"], "ms": best["ms"],
              "table": table}
    if cache_path:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        cache[sig] = result
        with open(cache_path, "w") as f:
            json.dump(cache, f)
    return result | {"cached": False}
