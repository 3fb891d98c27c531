"""Imported initial populations on the device against the reference (GPU).

tests/golden/init/ holds reference runs started from an imported
population (`gagp run --init`, cpp/src/cli/run.cpp:146-174): a first
reference search's final population, as the reference's phase-row import
gives its rows, then a search of the same task from those members.  The
device search admitted with the same rows (gagp_b200_search_create with
`initial`) must reproduce the history, the final ranked population and the
evaluation counters bit for bit -- steady-state and generational, scalar and
list programs.  Rows that do not derive from the grammar are refused before
anything runs."""
import glob
import gzip
import json
import os

import pytest

import golden_util as GU
from gagp_b200 import abi

pytestmark = pytest.mark.gpu
INIT_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "init")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(INIT_DIR, "*.json.gz")))


def _fixture(name):
    with gzip.open(os.path.join(INIT_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with Engine(0) as e:
        yield e


def _rows(lt, members):
    stride = lt.tables.max_nodes - lt.tables.fixed_nodes
    return abi.RowsBuffer.from_rows([(m["origins"], m["constants"]) for m in members], stride)


@pytest.mark.parametrize("name", NAMES)
def test_imported_population_search_matches_reference(engine, name):
    fx = _fixture(name)
    lt = GU.load_task(fx)
    s = engine.admit(lt, initial=_rows(lt, fx["initial"]))
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    GU.compare_result(lt, got, fx["run"], name)


def test_rows_outside_the_grammar_are_refused(engine):
    from gagp_b200.engine import EngineError
    fx = _fixture(NAMES[0])
    lt = GU.load_task(fx)
    members = [dict(m) for m in fx["initial"]]
    with pytest.raises(EngineError) as err:  # too few rows
        engine.admit(lt, initial=_rows(lt, members[:-1]))
    assert err.value.status == 2
    bad = dict(members[0], origins=[lt.tables.root_expression] + members[0]["origins"][1:])
    with pytest.raises(EngineError) as err:  # the root's origin is a reference, not a production
        engine.admit(lt, initial=_rows(lt, [bad] + members[1:]))
    assert err.value.status == 2


def test_statement_rows_reading_an_unassigned_local_are_refused(engine):
    """A statement program whose first assignment reads the local it
    assigns (acc = acc) fails the definite-assignment check and is refused,
    as the reference's verifier refuses it."""
    from gagp_b200 import grammar as G
    from gagp_b200.engine import EngineError
    fx = _fixture("init_statements")
    lt = GU.load_task(fx)
    ex = lt.tables.expressions
    read_acc = next(i for i, e in enumerate(ex) if e.kind == G.EK_OPERATION and e.node_kind == G.TK_VAR
                    and e.label == "acc")
    member = fx["initial"][0]
    origins, constants = list(member["origins"]), list(member["constants"])
    # program, block_cons, assign acc, then the assigned value's subtree
    assert [ex[o].node_kind for o in origins[:3]] == [G.TK_PROGRAM, G.TK_BLOCK, G.TK_ASSIGN]
    end, pending = 3, 1
    while pending:
        pending += ex[origins[end]].arity - 1
        end += 1
    dropped = sum(1 for o in origins[3:end] if ex[o].kind == G.EK_CONSTANT)
    bad = dict(member, origins=origins[:3] + [read_acc] + origins[end:], constants=constants[dropped:])
    with pytest.raises(EngineError) as err:
        engine.admit(lt, initial=_rows(lt, [bad] + fx["initial"][1:]))
    assert err.value.status == 2 and "local" in str(err.value)
