"""The oracle and the table builder against the reference's golden vectors.

Pins (CPU only):
* grammar admission tables == the reference's compile_phase_variation_grammar
  + normalize_static_phase_weights output;
* initial population rows == generate_phase_initial_population + import;
* whole searches (history, final ranked population) == the reference CPU
  engine's, bit for bit.
"""
import pytest

from gagp_b200 import abi
from oracle import oracle

import golden_util as GU

NAMES = GU.names()


@pytest.mark.parametrize("name", NAMES)
def test_tables_match_reference(name):
    fx = GU.fixture(name)
    lt = GU.load_task(fx)
    t = lt.tables
    slot = fx["tables"]["slots"][0]
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
    layout = fx["tables"]["layout"]
    assert layout["fixed_nodes"] == t.fixed_nodes and layout["max_nodes"] == t.max_nodes
    assert fx["tables"]["fuel"] == lt.settings.fuel and fx["tables"]["penalty"] == lt.settings.penalty


@pytest.mark.parametrize("name", NAMES)
def test_oracle_initial_population_matches_reference(name):
    fx = GU.fixture(name)
    lt = GU.load_task(fx)
    gb = abi.GrammarBlob(lt.tables)
    rows = oracle.initial_population(gb, lt.settings)
    for i, ref in enumerate(fx["initial"]):
        origins, constants = rows.row(i)
        assert list(origins) == ref["origins"], i
        assert list(constants) == [c[1] for c in ref["constants"]], i


@pytest.mark.parametrize("name", NAMES)
def test_oracle_search_matches_reference(name):
    fx = GU.fixture(name)
    lt = GU.load_task(fx)
    got = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
    GU.compare_result(lt, got, fx["run"], name)


def test_oracle_imported_population_reproduces_generated_one():
    """Importing the generated rows (annotate) gives the same search."""
    fx = GU.fixture("poly4_sitedepth4_t4")
    lt = GU.load_task(fx)
    gb = abi.GrammarBlob(lt.tables)
    rows = GU.reference_rows(fx["initial"], lt.tables.max_nodes - lt.tables.fixed_nodes)
    got = oracle.search(gb, lt.cases, lt.settings, initial=rows, member_reuse=True)
    GU.compare_result(lt, got, fx["run"], "imported")


def test_mt19937_64_known_answer():
    # std::mt19937_64 with its default seed 5489: the C++ standard requires
    # the 10000th output to be 9981545732273789042 ([rand.predef]).
    out = oracle.mt19937_64(5489, 10000)
    assert int(out[-1]) == 9981545732273789042
