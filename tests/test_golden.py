"""Pins the CPU oracle to the reference: replays every golden case (answers
produced by the reference's own GPULSMOpt engine on a B200) through the oracle."""
import numpy as np
import pytest

import golden_cases as G
from oracle import OracleLSM

pytestmark = pytest.mark.skipif(not G.available(), reason="golden fixtures not generated")


def answer(o, probe, name):
    q = probe.queries
    if name == "lookup":
        return o.lookup(q)
    if name == "lookup_found_values":
        return o.lookup(q, with_found=True)[0]
    if name == "lookup_found":
        return o.lookup(q, with_found=True)[1]
    if name == "successor":
        return o.successor(q)
    if name == "range_sum":
        return o.range_sum(probe.lo, probe.hi)
    raise KeyError(name)


@pytest.mark.parametrize("case", G.cases() if G.available() else [], ids=lambda c: c.name)
def test_oracle_matches_reference_fixture(case):
    o = OracleLSM()
    for ops, probe in case.stages:
        for op in ops:
            o.insert(op[1], op[2]) if op[0] == "insert" else o.erase(op[1])
        for name, want in probe.expect.items():
            got = answer(o, probe, name)
            assert np.array_equal(got, want), f"{case.name}: {name}"


def test_oracle_matches_reference_after_capacity_failure():
    c = G.capacity_case()
    # the reference accepted every batch of the loop, then refused the next insert with "capacity"
    assert "capacity" in c["after_error"]
    assert c["status"] & (1 << 3)
    o = OracleLSM()
    for op in c["ops"][: c["accepted"]]:
        o.insert(op[1], op[2])
    got = o.lookup(c["queries"])
    # keys of the failed 16-batch epoch stay readable in the reference ("pending updates were preserved")
    assert np.array_equal(got, c["lookup"])
