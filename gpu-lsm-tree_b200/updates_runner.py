"""Updates-benchmark runner: the FliX update experiment
(FliX/benchmarks_updates.cuh:1259-2540) over this library's FliX index or its
GPULSMOpt adapter, writing the reference's result file - one
result_collector table (FliX/result_collector.h:106-296) in long form with a
first-line header, packed columns, ", " separators and empty strings for
missing entries (FliX/main.cu:251-252) - with the parameter and measurement
names of the reference's records (benchmarks_updates.cuh:2498-2532), so the
reference's plotting scripts read both files side by side.

Protocol (the reference's update loop with insert-before-delete and no
alternation, restated): build 2^build_size_log keys with values 0..n-1; then
2 * batch_count + 1 steps - step 0 only probes, steps 1..batch_count each
insert the next insert_batch_size generated keys (values = their generation
index), the remaining steps each delete delete_batch_size live keys drawn
uniformly without replacement (sorted).  Every step times its update (CUDA
events, then a device synchronise; a GPULSMOpt update is joined, so its
merges are inside the time), an optional rebuild, the probe sort, the probe
of 2^probe_size_log live keys (checked against their values), the probe of as
many keys the run never inserts (checked as misses) and, for the FliX index, successor
probes of live keys (checked equal to themselves) and of absent keys
(checked against the ceiling in the live set).  Key draws are this runner's
own, seeded: unique keys in [2, 2^key_bits - 2] (FliX reserves 0 and 1, and a
64-bit successor miss reads 2^32 - 1 widened).  The file is rewritten after
every step, so a run cut short keeps the steps it finished.  This index has no separate
index layer: index_layer_time_ms is 0 and bucket_layer_time_ms is the probe.

Usage: python gpu-lsm-tree_b200/updates_runner.py --out updates.csv [--index flix|gpulsmopt]
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys

import numpy as np

NOT_FOUND = 0xFFFFFFFF
DELETE_SEED = 0x5EED


# ---------------------------------------------------------------------------
# result_collector, long form
def stringify(v) -> str:
    """A value as result_collector's stringify writes it (stream precision 16)."""
    if isinstance(v, (bool, np.bool_)):
        return "1" if v else "0"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return f"{float(v):.16g}"
    return str(v)


class ResultCollector:
    """Rows of (name, value, is_measurement) entries; columns in first-seen order."""

    def __init__(self, description_column_name: str = "DESCRIPTION", value_column_name: str = "VALUE"):
        self.parameter_names: list[str] = []
        self.measurement_names: list[str] = []
        self.kind: dict[str, bool] = {}
        self.rows: list[list[tuple[str, str, bool]]] = []
        self.description = description_column_name
        self.value = value_column_name

    def commit(self, parameters: list[tuple[str, object]], measurements: list[tuple[str, object]]):
        entries = [(n, stringify(v), False) for n, v in parameters] + [(n, stringify(v), True) for n, v in measurements]
        seen = set()
        for name, _, is_m in entries:
            if name in seen:
                raise ValueError(f"duplicate entry {name!r} in one record")
            seen.add(name)
            if name not in self.kind:
                self.kind[name] = is_m
                (self.measurement_names if is_m else self.parameter_names).append(name)
            elif self.kind[name] != is_m:
                raise ValueError(f"column {name!r} is both a parameter and a measurement")
        self.rows.append(entries)

    def long_form_packed(self, sep: str = ", ", empty: str = "", line_break: str = "\n") -> str:
        """write_csv(first_line_header, long_form, pack_columns): the parameter
        columns, then DESCRIPTION and VALUE; one line per measurement of a row,
        repeating the row's parameters."""
        out = [sep.join(self.parameter_names + [self.description, self.value]) + line_break]
        for entries in self.rows:
            values = {n: v for n, v, is_m in entries if not is_m}
            params = sep.join(values.get(n, empty) for n in self.parameter_names)
            for name, value, is_m in entries:
                if not is_m:
                    continue
                out.append((params + sep if params else "") + name + sep + value + line_break)
        return "".join(out)


# ---------------------------------------------------------------------------
def ceiling(live_sorted: np.ndarray, q: np.ndarray, miss: int) -> np.ndarray:
    i = np.searchsorted(live_sorted, q, side="left")
    out = np.full(q.size, miss, dtype=live_sorted.dtype)
    ok = i < live_sorted.size
    out[ok] = live_sorted[i[ok]]
    return out


def run(gl, torch, args, rc: ResultCollector, run_id: int, save=None) -> int:
    dev = torch.device("cuda")
    kb = args.key_bits
    kdt = np.uint32 if kb == 32 else np.uint64
    tdt = torch.int32 if kb == 32 else torch.int64

    def up(a, dtype=None):
        a = np.ascontiguousarray(a, dtype=dtype or kdt)
        return torch.from_numpy(a.view(np.int32 if a.dtype.itemsize == 4 else np.int64)).to(dev)

    build_size = 1 << args.build_size_log
    probe_size = 1 << args.probe_size_log
    ins_bs = build_size * args.insert_percent // (100 * args.batch_count)
    del_bs = build_size * args.delete_percent // (100 * args.batch_count)
    gen_size = build_size + ins_bs * args.batch_count
    rng = np.random.default_rng(0x1D5 + run_id)
    hi = (1 << kb) - 2 if kb == 32 else (1 << 40)
    # unique keys: draw with slack, deduplicate, keep the generation order
    # gen_size keys to insert, then probe_size keys that are never inserted
    # (the miss probes): unique, in a shuffled order
    total = gen_size + probe_size
    draw = rng.integers(2, hi, int(total * 1.1) + 1024, dtype=np.uint64)
    draw = draw[draw != NOT_FOUND]  # a 64-bit successor miss reads 2^32 - 1
    uniq = np.unique(draw)
    if uniq.size < total:
        raise RuntimeError("key space too small for the generated key set")
    generated = rng.permutation(uniq)[:total].astype(kdt)
    absent = np.sort(generated[gen_size:])
    generated = generated[:gen_size]
    live_k = generated[:build_size].copy()  # live keys and their values, unordered
    live_v = np.arange(build_size, dtype=np.uint32)
    inserted_end = build_size

    if args.index == "flix":
        index = gl.FlixIndex(key_bits=kb, max_elements=gen_size)
        index.build_bucket_layer_only(up(generated[:build_size]), build_size, gen_size)
        index_type, params = "flix_b200", [("node_size", "32"), ("initial fill", "50"), ("search", "directory")]
    else:
        if kb != 32:
            raise ValueError("the GPULSMOpt adapter takes 32-bit keys")
        index = gl.GpuLsmOptIndex(batch_capacity=1 << 20)
        index.build(up(generated[:build_size]), build_size, gen_size + del_bs * args.batch_count)
        index_type, params = "gpulsmopt_b200", [("batch capacity", str(1 << 20))]
    index_parameters = "&".join(f"{k}={v}" for k, v in params)
    index_id = index_type + "__" + "_".join(v for _, v in params)
    delete_gen = np.random.default_rng(DELETE_SEED + run_id)
    errors = 0

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def settle():
        join = getattr(getattr(index, "dictionary", None), "join", None)
        if join:
            join()

    for step in range(2 * args.batch_count + 1):
        do_insert = step < args.batch_count + 1  # insert before delete, no alternation
        do_delete = not do_insert
        m = dict.fromkeys(("insert_or_delete_time_ms", "probe_time_ms", "sort_time_ms", "probe_miss_time_ms",
                           "successor_hits_probe_time_ms", "successor_misses_probe_time_ms",
                           "index_layer_time_ms", "bucket_layer_time_ms", "rebuild_time_ms"), 0.0)
        before_size = live_k.size
        before_bytes = after_bytes = 0
        if step > 0:
            before_bytes = index.gpu_resident_bytes()
            if do_insert:
                k = generated[inserted_end:inserted_end + ins_bs]
                v = np.arange(inserted_end, inserted_end + ins_bs, dtype=np.uint32)
                order = np.argsort(k, kind="stable")  # FliX takes sorted batches
                kd, vd = up(k[order]), up(v[order], np.uint32)
                m["insert_or_delete_time_ms"] = timed(lambda: (index.insert(kd, vd, ins_bs), settle()))
                live_k = np.concatenate([live_k, k])
                live_v = np.concatenate([live_v, v])
                inserted_end += ins_bs
            else:
                idx = delete_gen.choice(live_k.size, size=min(del_bs, live_k.size), replace=False)
                dk = np.sort(live_k[idx])
                dd = up(dk)
                m["insert_or_delete_time_ms"] = timed(lambda: (index.remove(dd, dk.size), settle()))
                keep = np.ones(live_k.size, dtype=bool)
                keep[idx] = False
                live_k, live_v = live_k[keep], live_v[keep]
            if args.rebuild and args.index == "flix":
                m["rebuild_time_ms"] = timed(index.rebuild_bucket_layer_only)
        # probes: live keys (hits), then absent keys (misses)
        live_sorted = np.sort(live_k)
        pick = rng.integers(0, live_k.size, probe_size)
        hits, hit_vals = live_k[pick], live_v[pick]
        hd = up(hits)
        sorted_hd = torch.empty_like(hd)
        idx = torch.arange(probe_size, dtype=torch.int32, device=dev)
        perm = torch.empty(probe_size, dtype=torch.int32, device=dev)

        def sort_probes():  # this library's onesweep radix sort of (probe, input index)
            gl.sort_pairs(hd, idx, sorted_hd, perm)

        m["sort_time_ms"] = timed(sort_probes)
        res = torch.empty(probe_size, dtype=torch.int32, device=dev)
        if args.index == "flix":
            m["probe_time_ms"] = timed(lambda: index.lookups_ordered(sorted_hd, res, probe_size))
            got = np.empty(probe_size, np.uint32)
            got[perm.cpu().numpy()] = res.cpu().numpy().view(np.uint32)
        else:
            m["probe_time_ms"] = timed(lambda: index.lookup(hd, res, probe_size))
            got = res.cpu().numpy().view(np.uint32)
        errors += int(np.count_nonzero(got != hit_vals))
        m["bucket_layer_time_ms"] = m["probe_time_ms"]
        ad = up(absent)
        mres = torch.empty(absent.size, dtype=torch.int32, device=dev)
        if args.index == "flix":
            m["probe_miss_time_ms"] = timed(lambda: index.lookups_ordered(ad, mres, absent.size))
        else:
            m["probe_miss_time_ms"] = timed(lambda: index.lookup(ad, mres, absent.size))
        errors += int(np.count_nonzero(mres.cpu().numpy().view(np.uint32) != NOT_FOUND))
        if args.index == "flix":
            sres = torch.empty(probe_size, dtype=tdt, device=dev)
            m["successor_hits_probe_time_ms"] = timed(lambda: index.lookups_successor(sorted_hd, sres, probe_size))
            errors += int(np.count_nonzero(sres.cpu().numpy().view(kdt) != np.sort(hits)))
            smres = torch.empty(absent.size, dtype=tdt, device=dev)
            m["successor_misses_probe_time_ms"] = timed(lambda: index.lookups_successor(ad, smres, absent.size))
            errors += int(np.count_nonzero(smres.cpu().numpy().view(kdt) != ceiling(live_sorted, absent, NOT_FOUND)))
        after_bytes = index.gpu_resident_bytes()
        parameters = [
            ("EXPERIMENT", "batches"), ("index_type", index_type), ("index_parameters", index_parameters),
            ("index_id", index_id), ("run", run_id), ("key_bits", kb), ("build_size_log", args.build_size_log),
            ("probe_size_log", args.probe_size_log), ("batch_count", args.batch_count),
            ("total_inserts_percentage_of_build_size", args.insert_percent),
            ("total_deletes_percentage_of_build_size", args.delete_percent),
            ("delete_selection", "uniform_live"), ("delete_seed", DELETE_SEED + run_id),
            ("alternating_insert_delete", False), ("insert_before_delete", True), ("step", step),
            ("do_insert", do_insert), ("do_delete", do_delete),
            ("current_batch_size", ins_bs if do_insert else del_bs if do_delete else 0),
            ("before_update_size", before_size), ("after_update_size", live_k.size),
        ]
        measurements = [(k, v) for k, v in m.items()] + [("before_update_bytes", before_bytes),
                                                         ("after_update_bytes", after_bytes)]
        rc.commit(parameters, measurements)
        if save:
            save()  # the file is complete after every step
    close = getattr(index, "close", None)
    if close:
        close()
    return errors


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--out", default="updates.csv")
    p.add_argument("--index", choices=["flix", "gpulsmopt"], default="flix")
    p.add_argument("--key-bits", type=int, choices=[32, 64], default=64)
    p.add_argument("--build-size-log", type=int, default=22)
    p.add_argument("--probe-size-log", type=int, default=22)
    p.add_argument("--batch-count", type=int, default=4)
    p.add_argument("--insert-percent", type=int, default=100)
    p.add_argument("--delete-percent", type=int, default=100)
    p.add_argument("--runs", type=int, default=1)
    p.add_argument("--rebuild", action="store_true", help="rebuild the bucket layer after every update")
    args = p.parse_args(argv)
    if args.index == "gpulsmopt":
        args.key_bits = 32
    import torch

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    gl = importlib.import_module(os.path.basename(here))
    rc = ResultCollector()

    def save():
        with open(args.out, "w") as f:
            f.write(rc.long_form_packed())

    errors = sum(run(gl, torch, args, rc, r, save) for r in range(args.runs))
    save()
    print({"out": args.out, "rows": len(rc.rows), "errors": errors}, flush=True)
    return 1 if errors else 0


if __name__ == "__main__":
    sys.exit(main())
