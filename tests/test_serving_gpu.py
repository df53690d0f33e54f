"""GPU tests of the serving loop (gpulsm_server_*): continuous batching must
give every request the result it gets alone, equal to the oracle applied in
the server's order (rounds in order; inside a round its updates in submission
order, then its reads); the device-memory budget must refuse updates it
cannot hold; the native load generator must report consistent statistics."""
import threading

import numpy as np
import pytest

from conftest import to_dev
from oracle import OracleLSM

pytestmark = pytest.mark.gpu

KINDS = ("lookup", "insert", "erase", "range")


def make_requests(rng, universe, count, max_keys=4096):
    reqs = []
    for _ in range(count):
        kind = KINDS[rng.choice(4, p=[0.5, 0.2, 0.15, 0.15])]
        n = int(np.exp(rng.uniform(0, np.log(max_keys + 1))))
        n = max(1, min(max_keys, n))
        # skewed choice of keys: half from a hot prefix of the universe
        hot = rng.integers(0, 64, n)
        cold = rng.integers(0, universe.size, n)
        keys = universe[np.where(rng.random(n) < 0.5, hot, cold)]
        if kind == "insert":
            reqs.append((kind, keys, rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)))
        elif kind == "range":
            width = np.exp(rng.uniform(0, np.log(1 << 20), n)).astype(np.uint64)
            hi = np.minimum(keys.astype(np.uint64) + width, 0xFFFFFFFF).astype(np.uint32)
            reqs.append((kind, keys, hi))
        else:
            reqs.append((kind, keys, None))
    return reqs


def submit(srv, req):
    kind, keys, aux = req
    if kind == "lookup":
        return srv.submit_lookup(keys, with_found=True)
    if kind == "insert":
        return srv.submit_insert(keys, aux)
    if kind == "erase":
        return srv.submit_erase(keys)
    return srv.submit_range_sum(keys, aux)


def fresh_server(gl, base_k, base_v, staged=False):
    srv = gl.Server(gl.DictionaryConfig(max_elements=1 << 20, batch_capacity=1 << 16), budget_bytes=4 << 30,
                    max_round_keys=1 << 16, depth=3)
    srv.set_staged_updates(staged)
    srv.bulk_build(to_dev(base_k), to_dev(base_v))
    return srv


def oracle_answers(base_k, base_v, ordered):
    o = OracleLSM()
    o.bulk_build(base_k, base_v)
    out = []
    for kind, keys, aux in ordered:
        if kind == "lookup":
            out.append(o.lookup(keys, with_found=True))
        elif kind == "insert":
            o.insert(keys, aux)
            out.append(None)
        elif kind == "erase":
            o.erase(keys)
            out.append(None)
        else:
            out.append(o.range_sum(keys, aux))
    return out


def same(a, b):
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, tuple):
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return np.array_equal(a, b)


@pytest.mark.parametrize("staged", [False, True], ids=["direct", "staged"])
def test_results_same_alone_and_in_mix(gl, cuda, staged):
    rng = np.random.default_rng(11)
    base_k = rng.integers(0, 1 << 32, 1 << 16, dtype=np.uint64).astype(np.uint32)
    base_v = np.arange(base_k.size, dtype=np.uint32)
    universe = np.concatenate([base_k, rng.integers(0, 1 << 32, 1 << 14, dtype=np.uint64).astype(np.uint32)])
    per_thread = [make_requests(np.random.default_rng(100 + t), universe, 60) for t in range(4)]

    # in the mix: four threads submit at once, nothing waits until all are in
    srv = fresh_server(gl, base_k, base_v, staged)
    submitted = [[] for _ in range(4)]

    def client(t):
        for req in per_thread[t]:
            submitted[t].append((submit(srv, req), req))

    threads = [threading.Thread(target=client, args=(t,)) for t in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    flat = sorted((tk.id, tk, req) for lst in submitted for tk, req in lst)
    got = {tk.id: srv.wait(tk) for _, tk, _ in flat}
    st = srv.stats()
    assert st["completed"] == len(flat) and st["rejected"] == 0
    assert st["rounds"] < len(flat), "requests that arrived together were not coalesced"
    srv.close()
    # the server's order: rounds in order, inside a round its updates in
    # submission order, then its reads
    assert all(tk.round >= 1 for _, tk, _ in flat)
    flat.sort(key=lambda x: (x[1].round, x[2][0] not in ("insert", "erase"), x[0]))
    mix = [got[tk.id] for _, tk, _ in flat]
    kinds_of_round = {}
    for _, tk, req in flat:
        kinds_of_round.setdefault(tk.round, set()).add(req[0])
    assert any({"insert", "erase"} <= k for k in kinds_of_round.values()), "no round mixed inserts and erases"
    assert any(len(k) >= 3 for k in kinds_of_round.values()), "no round held three request kinds"

    # alone: one request at a time, in the server's order
    ordered = [req for _, _, req in flat]
    srv = fresh_server(gl, base_k, base_v, staged)
    alone = [srv.wait(submit(srv, req)) for req in ordered]
    # a lookup submitted alone is a lookup-only round: replayed from a CUDA graph;
    # an update submitted alone is one staged admission replayed from a graph,
    # and the staged runs merged into the levels whenever the staging slots filled
    st = srv.stats()
    assert st["graph_rounds"] == sum(1 for r in ordered if r[0] == "lookup")
    n_updates = sum(1 for r in ordered if r[0] in ("insert", "erase"))
    if staged:
        assert st["graph_updates"] == n_updates
        assert st["stage_flushes"] >= 1 and st["stage_flushes"] >= n_updates // 4 - 1
    else:
        assert st["graph_updates"] == 0 and st["stage_flushes"] == 0
    srv.close()

    want = oracle_answers(base_k, base_v, ordered)
    for i, (m, a, w) in enumerate(zip(mix, alone, want)):
        assert same(m, a), f"request {i} ({ordered[i][0]}): result differs between the mix and alone"
        assert same(a, w), f"request {i} ({ordered[i][0]}): result differs from the oracle"


def test_budget_refuses_updates_it_cannot_hold(gl, cuda):
    rng = np.random.default_rng(5)
    base_k = rng.integers(0, 1 << 32, 1 << 14, dtype=np.uint64).astype(np.uint32)
    base_v = np.arange(base_k.size, dtype=np.uint32)
    srv = gl.Server(gl.DictionaryConfig(max_elements=1 << 20), budget_bytes=1, max_round_keys=1 << 16, depth=2)
    srv.bulk_build(to_dev(base_k), to_dev(base_v))
    t_ins = srv.submit_insert(base_k[:100], base_v[:100])
    t_look = srv.submit_lookup(base_k[:1000])
    with pytest.raises(gl.CapacityError):
        srv.wait(t_ins)
    assert np.array_equal(srv.wait(t_look), base_v[:1000])  # reads are still served
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_load_generator_reports_consistent_stats(gl, cuda):
    rng = np.random.default_rng(7)
    base_k = rng.integers(0, 1 << 32, 1 << 18, dtype=np.uint64).astype(np.uint32)
    srv = gl.Server(gl.DictionaryConfig(max_elements=1 << 21), budget_bytes=8 << 30, max_round_keys=1 << 18)
    srv.bulk_build(to_dev(base_k), to_dev(np.arange(base_k.size, dtype=np.uint32)))
    closed = srv.run_load(base_k, rate_per_s=0, seconds=0.3, max_keys=1 << 12, max_outstanding=32)
    assert closed["completed"] > 10 and closed["rejected"] == 0
    assert 0 < closed["p50_us"] <= closed["p99_us"] <= closed["max_us"]
    rate = 0.3 * closed["completed"] / max(closed["wall_s"], 1e-6)
    opened = srv.run_load(base_k, rate_per_s=rate, seconds=0.3, max_keys=1 << 12, seed=2)
    assert opened["completed"] > 5 and opened["p50_us"] <= opened["p99_us"]
    srv.close()


def test_staged_updates_merge_into_levels_and_stay_exact(gl, cuda):
    """Update rounds go through the staged path: each admits its (padded)
    batch into a staging run by one captured graph; when the staging slots are
    full they merge into the levels.  Many small update rounds of every size
    class, interleaved with reads of every kind (lookups see the staged runs
    directly; range sums and the rest merge them first), stay equal to the
    oracle, and the padding never changes an answer."""
    rng = np.random.default_rng(23)
    base_k = rng.integers(0, 1 << 32, 1 << 15, dtype=np.uint64).astype(np.uint32)
    base_v = np.arange(base_k.size, dtype=np.uint32)
    universe = np.concatenate([base_k, rng.integers(0, 1 << 32, 1 << 13, dtype=np.uint64).astype(np.uint32)])
    srv = fresh_server(gl, base_k, base_v, staged=True)
    o = OracleLSM()
    o.bulk_build(base_k, base_v)
    for step in range(40):
        n = int(rng.choice([1, 7, 1000, 1025, 3000, 5000]))
        keys = universe[rng.integers(0, universe.size, n)]
        if step % 5 == 4:
            srv.wait(srv.submit_erase(keys))
            o.erase(keys)
        else:
            vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            srv.wait(srv.submit_insert(keys, vals))
            o.insert(keys, vals)
        if step % 3 == 0:
            q = universe[rng.integers(0, universe.size, 4000)]
            got = srv.wait(srv.submit_lookup(q, with_found=True))
            want = o.lookup(q, with_found=True)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), f"step {step}"
        if step % 7 == 6:
            lo = universe[rng.integers(0, universe.size, 500)]
            hi = np.minimum(lo.astype(np.uint64) + (1 << 24), 0xFFFFFFFF).astype(np.uint32)
            assert np.array_equal(srv.wait(srv.submit_range_sum(lo, hi)), o.range_sum(lo, hi)), f"step {step}"
    st = srv.stats()
    assert st["graph_updates"] == 40 and st["stage_flushes"] >= 5
    srv.close()


def test_request_ring_wraps_and_stays_exact(gl, cuda):
    """Requests are copied into the server's pinned ring at submit.  A small
    round limit (2^12 keys, a ring of 200 KB) and ~12 MB of requests wrap the
    ring many times, with requests of the largest size (which start over at
    the ring's beginning when they do not fit before its end) and empty
    requests in between; every result still equals the oracle replayed in the
    server's round order."""
    rng = np.random.default_rng(31)
    base_k = rng.integers(0, 1 << 32, 1 << 14, dtype=np.uint64).astype(np.uint32)
    base_v = np.arange(base_k.size, dtype=np.uint32)
    universe = np.concatenate([base_k, rng.integers(0, 1 << 32, 1 << 12, dtype=np.uint64).astype(np.uint32)])
    srv = gl.Server(gl.DictionaryConfig(max_elements=1 << 20, batch_capacity=1 << 12), budget_bytes=4 << 30,
                    max_round_keys=1 << 12, depth=2)
    srv.bulk_build(to_dev(base_k), to_dev(base_v))
    reqs = []
    for i in range(3000):
        kind = KINDS[rng.choice(4, p=[0.5, 0.2, 0.15, 0.15])]
        n = int(rng.choice([0, 1, 17, 300, 4096])) if i % 7 else 4096
        keys = universe[rng.integers(0, universe.size, n)]
        if kind == "insert":
            reqs.append((kind, keys, rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)))
        elif kind == "range":
            hi = np.minimum(keys.astype(np.uint64) + (1 << 22), 0xFFFFFFFF).astype(np.uint32)
            reqs.append((kind, keys, hi))
        else:
            reqs.append((kind, keys, None))
    done = []
    window = []
    for req in reqs:  # keep up to 48 requests in flight
        window.append((submit(srv, req), req))
        if len(window) >= 48:
            tk, rq = window.pop(0)
            done.append((tk, rq, srv.wait(tk)))
    for tk, rq in window:
        done.append((tk, rq, srv.wait(tk)))
    assert srv.stats()["rejected"] == 0
    srv.close()
    # empty requests complete without a round (round 0): they change nothing
    order = sorted(done, key=lambda x: (x[0].round, x[1][0] not in ("insert", "erase"), x[0].id))
    want = oracle_answers(base_k, base_v, [rq for _, rq, _ in order])
    for i, ((tk, rq, got), w) in enumerate(zip(order, want)):
        if rq[1].size == 0:
            continue
        assert same(got, w), f"request {tk.id} ({rq[0]}, {rq[1].size} keys, round {tk.round}) differs from the oracle"
