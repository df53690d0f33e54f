"""Our GPU engine against the reference's own answers (golden fixtures)."""
import numpy as np
import pytest

import golden_cases as G
from conftest import empty_u32, to_dev, to_host
from oracle import OracleFlix

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not G.available(), reason="golden fixtures not generated")]


def answer(d, probe, name):
    import torch

    q = probe.queries
    n = q.size
    if name in ("lookup", "lookup_found_values", "lookup_found"):
        out = empty_u32(n)
        found = torch.empty(max(n, 1), dtype=torch.uint8, device="cuda") if name != "lookup" else None
        d.lookup(to_dev(q), out, found, count=n)
        if name == "lookup_found":
            return to_host(found, np.uint8)[:n]
        return to_host(out)[:n]
    if name == "successor":
        out = empty_u32(n)
        d.successor(to_dev(q), out, count=n)
        return to_host(out)[:n]
    if name == "range_sum":
        m = probe.lo.size
        out = empty_u32(m)
        d.range(to_dev(probe.lo), to_dev(probe.hi), out, count=m)
        return to_host(out)[:m]
    raise KeyError(name)


@pytest.mark.parametrize("case", G.cases() if G.available() else [], ids=lambda c: c.name)
def test_engine_matches_reference_fixture(gl, cuda, case):
    d = gl.GPULSMOpt(gl.DictionaryConfig(**case.config))
    for ops, probe in case.stages:
        for op in ops:
            if op[0] == "insert":
                d.insert(to_dev(op[1]), to_dev(op[2]))
            else:
                d.erase(to_dev(op[1]))
        for name, want in probe.expect.items():
            assert np.array_equal(answer(d, probe, name), want), f"{case.name}: {name}"


@pytest.mark.skipif(not G.bulk_available(), reason="bulk-build fixture not generated")
def test_engine_matches_reference_bulk_build(gl, cuda):
    d = gl.GPULSMOpt(gl.DictionaryConfig(max_elements=1 << 17, batch_capacity=1 << 12))
    for i, (op, probe) in enumerate(G.bulk_case()):
        if op[0] == "bulk":
            d.bulk_build(to_dev(op[1]), to_dev(op[2]), count=op[1].size)
        elif op[0] == "insert":
            d.insert(to_dev(op[1]), to_dev(op[2]))
        else:
            d.erase(to_dev(op[1]))
        for name, want in probe.expect.items():
            assert np.array_equal(answer(d, probe, name), want), f"stage {i}: {name}"


@pytest.mark.skipif(not G.flix_available(), reason="FliX fixtures not generated")
@pytest.mark.parametrize("case", G.flix_cases() if G.flix_available() else [], ids=lambda c: c[0].name)
def test_flix_engine_matches_reference_fixture(gl, cuda, case):
    """Our FliX bucket layer against the reference's own FliX kernels on the
    same inputs: sorted-probe lookups and successors bit-exact, and the key
    count equal to compute_total_size (FliX/impl_cg_rtx_index_updates.cuh:1657)."""
    import torch

    from test_golden import flix_replay

    sc, z = case
    kdt = np.uint32 if sc.key_bits == 32 else np.uint64
    tdt = torch.int32 if sc.key_bits == 32 else torch.int64
    f = gl.FlixIndex(key_bits=sc.key_bits, max_elements=sc.max_size)
    f.build_bucket_layer_only(to_dev(sc.build_keys), max_size=sc.max_size)
    assert f.size() == int(z["build_total_keys"][0])

    def apply(st):
        if st.kind == "insert":
            f.insert(to_dev(st.keys), to_dev(st.values))
        elif st.kind == "remove":
            f.remove(to_dev(st.keys))
        else:
            f.rebuild_bucket_layer_only()

    def run(probes):
        lv = torch.empty(max(probes.size, 1), dtype=torch.int32, device="cuda")
        f.lookups_ordered(to_dev(probes), lv, size=probes.size)
        sv = torch.empty(max(probes.size, 1), dtype=tdt, device="cuda")
        f.lookups_successor(to_dev(probes), sv, size=probes.size)
        return to_host(lv)[: probes.size], to_host(sv, kdt)[: probes.size]

    def probe(st):
        got = {"successor": run(st.successor_probes)[1], "total_keys": f.size()}
        if st.lookup_probes is not None:
            got["lookup"] = run(st.lookup_probes)[0]
        return got

    # the exact answers: the oracle replayed alongside (std::map semantics)
    o = OracleFlix(sc.key_bits)
    o.build(sc.build_keys)
    o_apply = {"insert": lambda st: o.insert(st.keys, st.values), "remove": lambda st: o.remove(st.keys),
               "rebuild": lambda st: None}

    def apply_both(st):
        apply(st)
        o_apply[st.kind](st)

    def exact(st):
        ex = {"successor": o.successor(st.successor_probes), "total_keys": len(o)}
        if st.lookup_probes is not None:
            ex["lookup"] = o.lookup(st.lookup_probes)
        return ex

    def probe_checked(st):
        got = probe(st)
        ex = exact(st)
        for name in got:  # ours equals std::map everywhere, documented reference deviations included
            assert np.array_equal(np.asarray(got[name]), np.asarray(ex[name])), f"{sc.name}: {name} vs oracle"
        return got

    flix_replay(sc, z, apply_both, probe_checked, exact)
    assert f.status() == 0
