"""Bounded regions on the host against the reference (CPU).

tests/golden/region/ holds reference runs of the lattice-path workload,
whose grammar holds a memoized coordinate recurrence (a bounded region with
two Int coordinates, two requests, four evolved phases and a captured
input).  The table builder must give the reference's phase tables and
region table (compile_phase_grammar, phase_grammar.hpp:331-385), and the
oracle's generation and variation over them the reference's initial rows
and make_batch children.  Lowering and evaluation of region programs are
compared in test_lower_host.py (golden/lower/lower_grid_paths)."""
import glob
import gzip
import json
import os

import pytest

from gagp_b200 import abi, grammar as G, task as T

REGION_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "region")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(REGION_DIR, "*.json.gz")))
FULL = [n for n in NAMES if n == "region_grid_paths_p256"]


def _fixture(name):
    with gzip.open(os.path.join(REGION_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


def test_region_fixtures_exist_and_ran_resident():
    assert len(NAMES) >= 2
    for name in NAMES:
        run = _fixture(name)["run"]
        assert run["declined"] == "", name
        assert any("bounded_region" in h["text"] for h in run["history"]), name


@pytest.mark.parametrize("name", FULL)
def test_region_tables_match_reference(name):
    fx = _fixture(name)
    ref = fx["tables"]
    t = G.compile_tables(fx["grammar"], ref["inputs"], allow_lists=True)
    p = ref["slots"][0]["profile"]
    assert len(p["expressions"]) == len(t.expressions)
    for i, (re, e) in enumerate(zip(p["expressions"], t.expressions)):
        assert re["kind"] == e.kind, i
        assert re["node"] == [e.node_kind, e.opcode, e.operand, e.arity, e.fuel, e.merge_fuel, e.type], i
        assert re["target"] == e.target and re["children"] == e.children, i
        assert re["scope_count"] == e.scope_count and re["child_scope"] == e.child_scope, i
    assert [(x, float.fromhex(w)) for x, w in p["productions"]] == t.productions
    assert [tuple(n) for n in p["nonterminals"]] == [(a, b, c, int(d), int(e)) for a, b, c, d, e in t.nonterminals]
    assert p["minimum"] == t.minimum
    assert len(p["regions"]) == len(t.regions)
    for rr, r in zip(p["regions"], t.regions):
        plan = r.plan
        assert rr["traversal"] == 0 and rr["phases"] == 4
        assert rr["operands"] == len(plan.state_types) + plan.bound_count
        assert rr["captures"] == [list(c) for c in plan.captures]
        assert rr["operand_types"] == r.operand_types
        assert rr["phase_types"] == plan.phase_types
        assert rr["binding_types"] == [[b[2] for b in pb] for pb in plan.phase_bindings]


def _settings(fx):
    s = T.SearchSettings()
    T.apply_search(s, T.DEFAULT_SEARCH)
    T.apply_search(s, fx["search"])
    return s


@pytest.mark.parametrize("name", FULL)
def test_region_initial_population_matches_reference(name):
    from oracle import oracle
    fx = _fixture(name)
    t = G.compile_tables(fx["grammar"], fx["tables"]["inputs"], allow_lists=True)
    s = _settings(fx)
    rows = oracle.initial_population(abi.GrammarBlob(t), s)
    assert len(fx["initial"]) == s.population
    for i, ref in enumerate(fx["initial"]):
        origins, constants = rows.row(i)
        assert list(origins) == ref["origins"], i
        assert list(constants) == [c[1] for c in ref["constants"]], i


@pytest.mark.parametrize("name", FULL)
def test_region_make_batch_matches_reference(name):
    from oracle import oracle
    fx = _fixture(name)
    t = G.compile_tables(fx["grammar"], fx["tables"]["inputs"], allow_lists=True)
    s = _settings(fx)
    P = s.population
    selection = [float((i * 7919) % P + 1) for i in range(P)]
    ref = fx["batch"]
    rows, reuse = oracle.make_batch(abi.GrammarBlob(t), s, selection, int(ref["round_seed"]))
    for b, child in enumerate(ref["children"]):
        origins, constants = rows.row(b)
        assert list(origins) == child["origins"], b
        assert list(constants) == [c[1] for c in child["constants"]], b
        assert (reuse[b] >= 0) == (ref["reuse"][b] >= 0), b


def test_region_program_text_matches_reference():
    """The champion texts of the reference run, printed from the rows."""
    import golden_util as GU
    fx = _fixture(NAMES[-1])
    lt = GU.load_task(fx)
    for m in fx["run"]["final"][:200]:
        row = m["rows"][0]
        text = T.program_text(lt.tables, row["origins"], [c[1] for c in row["constants"]])
        assert GU.binder_names_in_order(text) == GU.binder_names_in_order(m["text"])
