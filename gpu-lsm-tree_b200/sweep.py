"""Paper-sweep runner: the reference's LSM insertion / lookup / range sweep
(FliX/paper_lsmu_sweep.cu:915-1140) over this library's GPU dictionary,
writing the same CSV files with the same columns so the reference's plotting
scripts read both side by side:

    insertion_b<B>.csv  system,batch_log,r,resident_elements,time_ms,rate_mops,
                        cumulative_ms,effective_rate_mops
    lookup_b<B>.csv     system,batch_log,r,resident_elements,scenario,time_ms,rate_mops
    range_b<B>.csv      system,batch_log,r,resident_elements,operation,expected_hits,
    (count_range_b<B>)  time_ms,rate_mops,chunk_size,checksum_sum,checksum_xor

Protocol (the reference's, restated): for batch size 2^B, insert batch r
(keys key_for_index(begin .. begin + 2^B), values 1) and time it (GPU events
around the call and a device synchronise); while the resident count is at
most 2^query_limit_log, time `resident` hit lookups and `resident` miss
lookups (each validated), and for B in [16, 20] `resident` range queries of
8 and 1024 expected hits in chunks of 2^range_chunk_log, with the
(sum, xor) digest of the results.  Inputs are generated on the host outside
the timed calls.

Usage: python gpu-lsm-tree_b200/sweep.py --out DIR --batch-logs 16 20 [--stop-after-r R]
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys

import numpy as np

KEY_DOMAIN = 1 << 30       # key_mask + 1 of the sweep (FliX/paper_lsmu_sweep.cu:64-67)
PAPER_INSERT_LIMIT = 1 << 27
NOT_FOUND = 0xFFFFFFFF
SYSTEM = "gpulsm_b200"


def key_for_index(i):
    """(index * 747796405 + 289133645) & (2^30 - 1), paper_lsmu_sweep.cu:64-67."""
    i = np.asarray(i, dtype=np.uint64)
    return ((i * np.uint64(747796405) + np.uint64(289133645)) & np.uint64(KEY_DOMAIN - 1)).astype(np.uint32)


def mix32(v):
    """The sweep's 32-bit mixer, paper_lsmu_sweep.cu:68-76."""
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(16)
    v = (v * np.uint64(0x7FEB352D)) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(15)
    v = (v * np.uint64(0x846CA68B)) & np.uint64(0xFFFFFFFF)
    v ^= v >> np.uint64(16)
    return v


def lookup_queries(count: int, resident: int, hits: bool, seed: int):
    """fill_lookup_queries, paper_lsmu_sweep.cu:95-116."""
    r = mix32(np.arange(count, dtype=np.uint64) + np.uint64(seed))
    if hits:
        return key_for_index(r % np.uint64(resident))
    miss_begin = max(resident, PAPER_INSERT_LIMIT)
    return key_for_index(np.uint64(miss_begin) + r % np.uint64(KEY_DOMAIN - miss_begin))


def range_queries(count: int, resident: int, expected_hits: int, seed: int):
    """fill_range_queries, paper_lsmu_sweep.cu:117-136."""
    width = (expected_hits * KEY_DOMAIN + resident - 1) // resident
    width = min(max(width, 1), KEY_DOMAIN)
    starts = KEY_DOMAIN - width + 1
    first = mix32(np.arange(count, dtype=np.uint64) + np.uint64(seed)) % np.uint64(starts)
    return first.astype(np.uint32), (first + np.uint64(width - 1)).astype(np.uint32)


def range_digest(results, query_offset: int):
    """(sum, xor of digest_mix(query << 32 | result)) as digest_range_results
    accumulates it (paper_lsmu_sweep.cu:196-230)."""
    r = np.asarray(results, dtype=np.uint64)
    q = np.arange(r.size, dtype=np.uint64) + np.uint64(query_offset)
    v = (q << np.uint64(32)) | r
    with np.errstate(over="ignore"):
        v = v + np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    return int(r.sum(dtype=np.uint64)), int(np.bitwise_xor.reduce(v)) if v.size else 0


def run_batch_log(gl, torch, b: int, args) -> dict:
    """One batch size of the main sweep; returns a summary of what was checked."""
    dev = torch.device("cuda")
    batch = 1 << b
    maximum = 1 << args.insert_limit_log
    count = maximum // batch
    if args.stop_after_r:
        count = min(count, args.stop_after_r)
    run_lookups = 16 <= b <= 24 and args.query_limit_log >= b
    run_ranges = 16 <= b <= 20 and args.query_limit_log >= b
    query_max = (1 << args.query_limit_log) if run_lookups else 0
    chunk = 1 << args.range_chunk_log

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)

    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=maximum, batch_capacity=min(batch, 1 << 20)))
    ones = up(np.ones(batch, np.uint32))
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    suffix = f"_b{b}.csv"
    os.makedirs(args.out, exist_ok=True)
    ins_f = open(os.path.join(args.out, "insertion" + suffix), "w")
    look_f = open(os.path.join(args.out, "lookup" + suffix), "w")
    rng_f = open(os.path.join(args.out, ("count_range" if args.include_count else "range") + suffix), "w")
    ins_f.write("system,batch_log,r,resident_elements,time_ms,rate_mops,cumulative_ms,effective_rate_mops\n")
    look_f.write("system,batch_log,r,resident_elements,scenario,time_ms,rate_mops\n")
    rng_f.write("system,batch_log,r,resident_elements,operation,expected_hits,time_ms,rate_mops,chunk_size,"
                "checksum_sum,checksum_xor\n")
    errors = 0
    cumulative = 0.0

    def timed(fn):
        e0, e1 = ev(), ev()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for r in range(1, count + 1):
        begin = (r - 1) * batch
        keys = up(key_for_index(np.arange(begin, begin + batch, dtype=np.uint64)))
        torch.cuda.synchronize()
        ms = timed(lambda: (d.insert(keys, ones), d.join()))  # admitted and merged
        cumulative += ms
        resident = r * batch
        ins_f.write(f"{SYSTEM},{b},{r},{resident},{ms:.12g},{batch / ms / 1e3:.12g},{cumulative:.12g},"
                    f"{resident / cumulative / 1e3:.12g}\n")
        if run_lookups and resident <= query_max:
            out = torch.empty(resident, dtype=torch.int32, device=dev)
            for scenario, hits, seed in (("all_existing", True, 0x10000 + r), ("none_existing", False, 0x20000 + r)):
                q = up(lookup_queries(resident, resident, hits, seed))
                torch.cuda.synchronize()
                ms_l = timed(lambda: d.lookup(q, out))
                got = out.cpu().numpy().view(np.uint32)
                errors += int(np.count_nonzero(got != (1 if hits else NOT_FOUND)))
                look_f.write(f"{SYSTEM},{b},{r},{resident},{scenario},{ms_l:.12g},{resident / ms_l / 1e3:.12g}\n")
        if run_ranges and resident <= query_max:
            for expected in (8, 1024):
                t_count = t_range = 0.0
                digest_sum, digest_xor = 0, 0
                seed = 0x30000 + r + expected
                for off in range(0, resident, chunk):
                    cur = min(chunk, resident - off)
                    lo, hi = range_queries(cur, resident, expected, seed + off)
                    lo_d, hi_d = up(lo), up(hi)
                    res = torch.empty(cur, dtype=torch.int32, device=dev)
                    torch.cuda.synchronize()
                    if args.include_count:
                        cnt = torch.empty(cur, dtype=torch.int32, device=dev)
                        t_count += timed(lambda: d.range_count(lo_d, hi_d, cnt))
                    t_range += timed(lambda: d.range(lo_d, hi_d, res))
                    vals = res.cpu().numpy().view(np.uint32)
                    if args.include_count:  # values are all 1: the sum equals the count
                        errors += int(np.count_nonzero(cnt.cpu().numpy().view(np.uint32) != vals))
                    s_, x_ = range_digest(vals, off)
                    digest_sum = (digest_sum + s_) & 0xFFFFFFFFFFFFFFFF
                    digest_xor ^= x_
                if args.include_count:
                    rng_f.write(f"{SYSTEM},{b},{r},{resident},count,{expected},{t_count:.12g},"
                                f"{resident / t_count / 1e3:.12g},{chunk},0,0\n")
                rng_f.write(f"{SYSTEM},{b},{r},{resident},range,{expected},{t_range:.12g},"
                            f"{resident / t_range / 1e3:.12g},{chunk},{digest_sum},{digest_xor}\n")
    for f in (ins_f, look_f, rng_f):
        f.close()
    status = d.canonical_carry_status()
    d.close()
    return {"batch_log": b, "inserts": count, "errors": errors, "status": status}


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--out", default="paper_sweep_results")
    p.add_argument("--batch-logs", type=int, nargs="+", default=[16, 18, 20])
    p.add_argument("--insert-limit-log", type=int, default=27)
    p.add_argument("--query-limit-log", type=int, default=24)
    p.add_argument("--range-chunk-log", type=int, default=18)
    p.add_argument("--stop-after-r", type=int, default=0)
    p.add_argument("--include-count", action="store_true", help="also time range counts (LSMu's count)")
    args = p.parse_args(argv)
    import torch

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    gl = importlib.import_module(os.path.basename(here))
    bad = 0
    for b in args.batch_logs:
        if b > args.insert_limit_log:
            continue
        summary = run_batch_log(gl, torch, b, args)
        print(summary, flush=True)
        bad += summary["errors"] + (1 if summary["status"] else 0)
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main())
