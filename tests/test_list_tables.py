"""The table builder's list subset against the reference's tables (CPU).

The list programs (a traversal of an IntList with element, index and
accumulator binders, scoped nonterminals, bound names, len) run on the
device.  Their phase tables: ``grammar.compile_tables(..., allow_lists=True)``
must equal the
reference's compile_phase_grammar output (phase_grammar.hpp:94-300, weights
normalised by normalize_static_phase_weights) for the fixtures that
tests/golden/make_golden.py records from the reference engine, including a
nested traversal whose body maps the outer accumulator and the inner binders
by name, and a statement program (Program entry, grammar locals, assign,
for_range, if_stmt and return controls, a variation-disabled entry).
"""
import pytest

from gagp_b200 import grammar as G

import golden_util as GU

# the list fixtures that also hold the reference's tables, initial rows and
# one make_batch (the others hold whole runs only)
NAMES = [n for n in GU.list_names() if "tables" in GU.list_fixture(n)]


def test_list_fixtures_exist():
    assert len(NAMES) >= 3


@pytest.mark.parametrize("name", NAMES)
def test_list_tables_match_reference(name):
    fx = GU.list_fixture(name)
    ref = fx["tables"]
    t = G.compile_tables(fx["grammar"], ref["inputs"], allow_lists=True)
    slot = ref["slots"][0]
    p = slot["profile"]
    assert p["root_expression"] == t.root_expression
    assert (p["depth_count"], p["logical_depth_count"]) == (t.depth_count, t.logical_depth_count)
    assert len(p["expressions"]) == len(t.expressions)
    for i, (re, e) in enumerate(zip(p["expressions"], t.expressions)):
        assert re["kind"] == e.kind, i
        assert re["node"] == [e.node_kind, e.opcode, e.operand, e.arity, e.fuel, e.merge_fuel, e.type], i
        assert re["target"] == e.target and re["children"] == e.children, i
        assert re["scope_count"] == e.scope_count and re["child_scope"] == e.child_scope, i
    assert [(x, float.fromhex(w)) for x, w in p["productions"]] == t.productions
    assert [tuple(n) for n in p["nonterminals"]] == [(a, b, c, int(d), int(e)) for a, b, c, d, e in t.nonterminals]
    assert [tuple(d) for d in p["domains"]] == [
        (d.value_offset, d.value_count, int(d.integer_range), d.minimum, d.maximum) for d in t.domains]
    assert [tuple(v[:2]) for v in p["values"]] == t.values
    assert p["minimum"] == t.minimum
    assert slot["max_depth"] == t.slot_max_depth and slot["type"] == t.slot_type
    assert slot["locals"] == t.local_types
    assert ref["layout"]["fixed_nodes"] == t.fixed_nodes and ref["layout"]["max_nodes"] == t.max_nodes


@pytest.mark.parametrize("name", NAMES)
def test_list_tasks_run_resident_in_the_reference(name):
    """The recorded reference runs took the resident path (no decline)."""
    fx = GU.list_fixture(name)
    run = fx["run"]
    assert run["declined"] == ""
    assert len(run["history"]) == 3
    if fx["grammar"]["entry"].get("category") == "Program":
        # a statement program: the reference's tables hold its controls and
        # the slot is the whole program, without a terminator
        assert fx["tables"]["layout"]["program_terminator"] == 0 and fx["tables"]["layout"]["fixed_nodes"] == 0
    else:
        assert run["history"][0]["text"].startswith("(traverse xs")


def test_every_list_run_took_the_resident_path():
    for name in GU.list_names():
        fx = GU.list_fixture(name)
        run = fx["run"]
        assert run["declined"] == "", name
        if fx["grammar"]["entry"].get("category") == "Program":
            assert any("for_range" in h["text"] or "(block" in h["text"] for h in run["history"]), name
        else:
            assert any(h["text"].startswith("(traverse") for h in run["history"]), name


@pytest.mark.parametrize("name", NAMES)
def test_list_tables_are_declined_without_the_list_subset(name):
    fx = GU.list_fixture(name)
    with pytest.raises(G.Declined):
        G.compile_tables(fx["grammar"], fx["tables"]["inputs"])


@pytest.mark.parametrize("name", NAMES)
def test_list_initial_population_matches_reference(name):
    """The oracle's generator (generate_phase_initial_population restated)
    over the list tables reproduces the reference's initial rows: scoped
    references, bound leaves and traversal bodies need nothing beyond the
    tables."""
    from gagp_b200 import abi, task as T
    from oracle import oracle
    fx = GU.list_fixture(name)
    t = G.compile_tables(fx["grammar"], fx["tables"]["inputs"], allow_lists=True)
    s = T.SearchSettings()
    T.apply_search(s, T.DEFAULT_SEARCH)
    T.apply_search(s, fx["search"])
    rows = oracle.initial_population(abi.GrammarBlob(t), s)
    assert len(fx["initial"]) == s.population
    for i, ref in enumerate(fx["initial"]):
        origins, constants = rows.row(i)
        assert list(origins) == ref["origins"], i
        assert list(constants) == [c[1] for c in ref["constants"]], i


@pytest.mark.parametrize("name", NAMES)
def test_list_make_batch_matches_reference(name):
    """One make_batch over the list tables (tournaments, typed subtree
    crossover and mutation with scoped sites, traversal bodies included) gives
    the reference owner's children row for row, and reuses a result exactly
    for the children the reference does (its parent's when unchanged, else an
    identical member's; which identical member is taken does not change the
    result)."""
    from gagp_b200 import abi, task as T
    from oracle import oracle
    fx = GU.list_fixture(name)
    t = G.compile_tables(fx["grammar"], fx["tables"]["inputs"], allow_lists=True)
    s = T.SearchSettings()
    T.apply_search(s, T.DEFAULT_SEARCH)
    T.apply_search(s, fx["search"])
    P = s.population
    selection = [float((i * 7919) % P + 1) for i in range(P)]
    ref = fx["batch"]
    rows, reuse = oracle.make_batch(abi.GrammarBlob(t), s, selection, int(ref["round_seed"]))
    assert len(ref["children"]) == len(reuse)
    for b, child in enumerate(ref["children"]):
        origins, constants = rows.row(b)
        assert list(origins) == child["origins"], b
        assert list(constants) == [c[1] for c in child["constants"]], b
        assert (reuse[b] >= 0) == (ref["reuse"][b] >= 0), b
