"""Multi-tenant batched dictionary: per-tenant answers equal one GPULSMOpt-
semantics oracle per tenant, for every tuning and for graph-replayed rounds;
the batched mode beats the plain form (one dictionary per tenant)."""
import time

import numpy as np
import pytest

from conftest import to_dev
from oracle import OracleLSM

pytestmark = pytest.mark.gpu


def make_rounds(rng, caps, rounds, max_batch):
    T = caps.size
    out = []
    for r in range(rounds):
        per = [rng.integers(0, max(1, min(int(caps[t]) // 4, max_batch)) + 1) for t in range(T)]
        keys, vals = [], []
        for t in range(T):
            n = int(per[t])
            span = max(4, int(caps[t]) * 2)
            k = rng.integers(0, span, n, dtype=np.uint64).astype(np.uint32) * np.uint32(2654435761 % (1 << 32) | 1)
            keys.append(k)
            vals.append(rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32))
        off = np.zeros(T + 1, np.uint64)
        off[1:] = np.cumsum([k.size for k in keys])
        out.append((keys, vals, off))
    return out


def apply(oracles, rnd):
    keys, vals, _ = rnd
    for t, (k, v) in enumerate(zip(keys, vals)):
        if k.size:
            oracles[t].insert(k, v)


def check(pool, oracles, rng, caps, gl):
    import torch

    T = caps.size
    tid = rng.integers(0, T, 20000).astype(np.uint32)
    q = np.empty(tid.size, np.uint32)
    for i, t in enumerate(tid):
        kt, _ = oracles[t].dump()
        if kt.size and rng.random() < 0.7:
            q[i] = kt[rng.integers(0, kt.size)]
        else:
            q[i] = rng.integers(0, 1 << 32, dtype=np.uint64)
    out = torch.empty(tid.size, dtype=torch.int32, device="cuda")
    found = torch.empty(tid.size, dtype=torch.uint8, device="cuda")
    pool.lookup(to_dev(tid), to_dev(q), out, found)
    got = out.cpu().numpy().view(np.uint32)
    want = np.empty_like(got)
    for t in np.unique(tid):
        m = tid == t
        want[m] = oracles[t].lookup(q[m])
    got_f = found.cpu().numpy()
    assert np.array_equal(np.where(got_f == 1, got, np.uint32(0xFFFFFFFF)), want)
    # main + delta rows bound the live keys (a key may sit in both runs)
    assert np.all(pool.sizes() >= np.array([len(o) for o in oracles], np.uint64))
    assert pool.status() == 0


def upload(rnd):
    import torch

    keys, vals, off = rnd
    k = np.concatenate(keys) if off[-1] else np.zeros(1, np.uint32)
    v = np.concatenate(vals) if off[-1] else np.zeros(1, np.uint32)
    return to_dev(k), to_dev(v), torch.from_numpy(off.view(np.int64)).cuda()


@pytest.mark.parametrize("tile,fan_in,fanout", [(2048, 2, 16), (256, 4, 8), (4096, 1, 32), (512, 8, 16)])
def test_rounds_match_per_tenant_oracles(gl, cuda, tile, fan_in, fanout):
    rng = np.random.default_rng(tile + fan_in + fanout)
    T = 48
    caps = np.exp(rng.uniform(np.log(64), np.log(4096), T)).astype(np.uint64)
    caps[0] = 1  # a tiny tenant
    rounds = make_rounds(rng, caps, 7, 300)
    pool = gl.TenantPool(caps * 2 + 8, max_round_keys=sum(int(r[2][-1]) for r in rounds), tile=tile,
                         fan_in=fan_in, fanout=fanout)
    oracles = [OracleLSM() for _ in range(T)]
    for r in rounds:
        pool.insert_round(*upload(r))
        apply(oracles, r)
        check(pool, oracles, rng, caps, gl)


def test_graph_replayed_rounds(gl, cuda):
    import torch

    rng = np.random.default_rng(7)
    T = 32
    caps = np.exp(rng.uniform(np.log(64), np.log(2048), T)).astype(np.uint64)
    rounds = make_rounds(rng, caps, 6, 200)
    cap_round = max(int(r[2][-1]) for r in rounds)
    pool = gl.TenantPool(caps * 2 + 8, max_round_keys=cap_round, fan_in=2)
    kbuf = torch.empty(cap_round, dtype=torch.int32, device="cuda")
    vbuf = torch.empty(cap_round, dtype=torch.int32, device="cuda")
    obuf = torch.empty(T + 1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    oracles = [OracleLSM() for _ in range(T)]
    for r in rounds:
        k, v, off = upload(r)
        n = int(r[2][-1])
        with torch.cuda.stream(stream):
            kbuf[:n].copy_(k[:n])
            vbuf[:n].copy_(v[:n])
            obuf.copy_(off)
            pool.insert_round(kbuf, vbuf, obuf, stream=stream, graph=True)  # same buffers: one capture per shape
        stream.synchronize()
        apply(oracles, r)
        check(pool, oracles, rng, caps, gl)


def test_batched_mode_beats_plain_form(gl, cuda):
    """512 tenants, 4 rounds: one pool (a few launches per round for all
    tenants) against one dictionary per tenant (a call per tenant per round)."""
    import torch

    rng = np.random.default_rng(11)
    T = 512
    caps = np.exp(rng.uniform(np.log(1024), np.log(16384), T)).astype(np.uint64)
    rounds = make_rounds(rng, caps, 4, 2048)
    dev_rounds = [upload(r) for r in rounds]
    pool = gl.TenantPool(caps * 2 + 8, max_round_keys=max(int(r[2][-1]) for r in rounds))
    plain = [gl.GPULSMOpt(gl.DictionaryConfig(max_elements=int(c) * 2, batch_capacity=4096)) for c in caps]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k, v, off in dev_rounds:
        pool.insert_round(k, v, off)
    torch.cuda.synchronize()
    batched = time.perf_counter() - t0
    t0 = time.perf_counter()
    for (keys, vals, off), (k, v, _) in zip(rounds, dev_rounds):
        for t in range(T):
            a, b = int(off[t]), int(off[t + 1])
            if b > a:
                plain[t].insert(k[a:b], v[a:b])
    torch.cuda.synchronize()
    per_tenant = time.perf_counter() - t0
    print(f"\n512 tenants x 4 rounds: batched {batched * 1e3:.2f} ms, one dictionary per tenant {per_tenant * 1e3:.2f} ms")
    assert batched < per_tenant


def test_autotuner_picks_and_caches(gl, cuda, tmp_path):
    import importlib

    tune = importlib.import_module("gpu-lsm-tree_b200.autotune")
    rng = np.random.default_rng(3)
    T = 16
    caps = np.full(T, 2048, np.uint64)
    rounds = make_rounds(rng, caps, 3, 256)
    dev_rounds = [upload(r) for r in rounds]
    tid = to_dev(rng.integers(0, T, 4096).astype(np.uint32))
    q = to_dev(rng.integers(0, 1 << 32, 4096, dtype=np.uint64).astype(np.uint32))
    cache = str(tmp_path / "tune.json")
    r1 = tune.autotune(caps * 2, dev_rounds, (tid, q), max(int(r[2][-1]) for r in rounds), cache_path=cache,
                       tiles=(256, 2048), fan_ins=(2, 4), fanouts=(8, 32))
    assert not r1["cached"] and len(r1["table"]) == 8
    assert r1["tile"] in (256, 2048) and r1["fan_in"] in (2, 4) and r1["fanout"] in (8, 32)
    r2 = tune.autotune(caps * 2, dev_rounds, (tid, q), max(int(r[2][-1]) for r in rounds), cache_path=cache)
    assert r2["cached"] and r2["tile"] == r1["tile"]
