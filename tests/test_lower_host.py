"""The engine's lowering and exact VM against the reference (CPU).

For every member of a generated population of each grammar in
tests/golden/lower/ (list programs with forward, reverse and nested
traversals, lets, statement programs with grammar locals, loops and
branches, bounded regions with their records and phase code, and the
large scalar grammar), the reference's phase compiler
output and CPU fitness were recorded by ``ref_driver lower``.  The engine's
own ``lower_program`` and ``run_program`` -- the functions its kernels run,
compiled here for the host by tests/host_harness.py -- must emit the same
bytecode (opcodes, operands, fuel charges, constants, locals, stack bound)
and give every program the same fitness and wrong count on every case."""
import gzip
import glob
import json
import os

import pytest

from gagp_b200 import abi, grammar as G

import golden_util as GU
import host_harness as H

LOWER_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lower")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(LOWER_DIR, "*.json.gz")))


def fixture(name):
    with gzip.open(os.path.join(LOWER_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


def case_loss(ok, value, tag, expected, expected_tag, penalty, metric):
    """fitness_case_score as a loss (cpp/include/gagp/core/fitness_policy.hpp:28-58)."""
    if not ok:
        return (1 if metric == "exact" else penalty), 1
    same = tag == expected_tag and value == expected
    if metric == "exact":
        return (0 if same else 1), int(not same)
    if tag != G.TAG_INT or expected_tag != G.TAG_INT:
        return penalty, int(not same)
    return min(abs(value - expected), penalty), int(not same)


def test_lower_fixtures_exist():
    assert len(NAMES) >= 4


@pytest.mark.parametrize("name", NAMES)
def test_lowering_and_vm_match_reference(name):
    fx = fixture(name)
    lt = GU.load_task(fx)
    blob = abi.GrammarBlob(lt.tables)
    cases = lt.cases
    fuel = fx["lower"]["fuel"]
    penalty = int(abs(lt.settings.penalty))
    checked = 0
    for r, row in enumerate(fx["lower"]["rows"]):
        got = H.lower(blob, row["origins"], row["constants"], shape=True)
        if row["status"] != 0:
            assert got is None, (name, r)
            continue
        assert got is not None, (name, r, "rejected")
        code, consts, n_locals, stack_bound, n_main, main_consts = got
        ref = row["code"]
        # a value phase: the reference's main code plus the RETURN that
        # patch_whole_program appends, then its bounded regions' records and
        # phase code (op 255 onwards); a statement program (Program entry)
        # has no terminator
        statements = lt.tables.slot_type == G.TAG_STATEMENT
        ref_main = next((i for i, x in enumerate(ref) if x[0] == 255), len(ref))
        want = ref[:ref_main] + ([] if statements else [[20, 0, 0, 0, 1]]) + ref[ref_main:]
        assert len(code) == len(want) and n_main == ref_main + (0 if statements else 1), (name, r)
        for i, x in enumerate(want):
            mine = [int(code[i][0]), int(code[i][1]) & 3, int(code[i][2]), int(code[i][3]), int(code[i][4])]
            assert mine == x, (name, r, i, mine, x)
        assert len(consts) == len(row["consts"]), (name, r)
        for i, x in enumerate(code[:ref_main]):
            if x[0] == 0:  # PUSH_CONST: the constant's tag and payload
                tag, iv, bv = row["consts"][x[2]]
                assert tag == (G.TAG_BOOL if x[1] & 4 else G.TAG_INT), (name, r, i)
                assert consts[x[2]] == (bv if tag == G.TAG_BOOL else iv), (name, r, i)
        assert n_locals == row["n_locals"] and stack_bound == row["stack_bound"], (name, r)
        loss, wrong = 0, 0
        for c in range(len(cases.expected)):
            if n_main < len(code):
                ok, value, tag, _ = H.run_regions(blob, cases, fuel, code, n_main, consts, main_consts, n_locals, c)
            else:
                ok, value, tag, _ = H.run(cases, lt.tables.local_types, fuel, code, consts, n_locals, c)
            if c < len(row["cases"]):
                err, rtag, rvalue, _ = row["cases"][c]
                assert ok == (err < 0), (name, r, c)
                if ok:
                    assert (tag, value) == (rtag, rvalue), (name, r, c)
            l, w = case_loss(ok, value, tag, int(cases.expected[c]), cases.expected_tag, penalty,
                             lt.settings.metric)
            loss, wrong = loss + l, wrong + w
        assert -loss == row["fitness"] and wrong == row["wrong"], (name, r, -loss, row["fitness"])
        checked += 1
    assert checked > 100
