"""The reference's own VM known-answer fixtures on the engine's exact VM (CPU).

tests/golden/vm_fixtures.json holds the scenarios of the reference's
cpp/tests/fixtures/runtime/{scalar,control_flow,builtins,typed_values}.json
that fall in the engine's subset (make_vm_fixtures.py converts them and
records what it leaves out and why): wrap-around addition, Python-sign
modulo and ZeroDivisionError, not, branches, a counting loop, a fuel
timeout, abs/min/len, index with a negative index and a range error,
idiv0/imod0 by zero, IntList indexing.  run_program -- the exact VM the
device kernel runs, compiled for the host -- must give each case's value and
tag, or fail where the reference raises."""
import json
import os

import numpy as np
import pytest

import host_harness as H
from gagp_b200 import abi

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vm_fixtures.json")
with open(FIXTURES) as _f:
    DOC = json.load(_f)


def test_fixture_conversion_records_what_it_leaves_out():
    assert len(DOC["scenarios"]) >= 10
    assert sum(len(s["cases"]) for s in DOC["scenarios"]) >= 15
    kinds = {c["error"] for s in DOC["scenarios"] for c in s["cases"]}
    assert {"ZeroDivisionError", "ValueError", "Timeout"} <= kinds
    for s in DOC["skipped"]:
        assert s["why"]


@pytest.mark.parametrize("scenario", DOC["scenarios"], ids=[s["fixture"] + ":" + s["intent"][:40] for s in DOC["scenarios"]])
def test_reference_vm_fixture(scenario):
    n_locals = scenario["n_locals"]
    for case in scenario["cases"]:
        lists = [0]  # offset 0 unused, so that no IntList sits at payload 0 by accident
        inputs = np.zeros((1, max(1, n_locals)), dtype=np.int64)
        tags = [9] * max(1, n_locals)
        for i in case["inputs"]:
            if i["tag"] == 5:
                inputs[0, i["idx"]] = len(lists)
                lists.extend([len(i["value"])] + [int(x) for x in i["value"]])
            else:
                inputs[0, i["idx"]] = int(i["value"])
            tags[i["idx"]] = i["tag"]
        cases = abi.CasesBlob(inputs, tags, np.zeros(1, dtype=np.int64), 0, np.array(lists, dtype=np.int64))
        code = np.array(scenario["code"], dtype=np.int32).reshape(-1, 5)
        consts = np.array(scenario["consts"] + [0], dtype=np.int64)
        ok, value, tag, _ = H.run(cases, tags, scenario["fuel"], code, consts, n_locals, 0)
        if case["error"]:
            assert not ok, (scenario["intent"], case)
        else:
            assert ok, (scenario["intent"], case)
            assert (tag, value) == (case["expected"]["tag"], case["expected"]["value"]), (scenario["intent"], case)
