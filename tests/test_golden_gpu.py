"""Our GPU engine against the reference's own answers (golden fixtures)."""
import numpy as np
import pytest

import golden_cases as G
from conftest import empty_u32, to_dev, to_host

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
