"""Device row evaluation (lowering + VMs + reduction) against the oracle (GPU).

Covers the fast accumulator VM and the exact general VM: the `mod` grammar
below raises ZeroDiv on some cases (Python-sign modulo by zero), which only
the general VM executes; such programs score the error ceiling per case."""
import copy
import os

import numpy as np
import pytest

from gagp_b200 import abi, task as T, workloads as W
from oracle import oracle

import golden_util as GU

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    e = Engine(0)
    yield e
    e.close()


def _task(tmp_path, files):
    return T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))


@pytest.mark.parametrize("name", ["poly4_p512_g12_s1", "polynomial_p1024_g64", "poly4_exact_metric"])
def test_evaluate_golden_populations(engine, name):
    fx = GU.fixture(name)
    lt = GU.load_task(fx)
    stride = lt.tables.max_nodes - lt.tables.fixed_nodes
    rows = GU.reference_rows([m["rows"][0] for m in fx["run"]["final"]], stride)
    f, w = engine.evaluate_rows(lt, rows)
    want_f, want_w, _ = oracle.evaluate(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, rows)
    assert np.array_equal(f, want_f)
    assert np.array_equal(w, want_w)
    # and the reference's own final fitness / wrong counts
    assert list(f) == [m["fitness"] for m in fx["run"]["final"]]
    assert list(w) == [m["wrong"] for m in fx["run"]["final"]]


def test_evaluate_general_vm_with_errors(engine, tmp_path):
    files = W.poly4(population=512, generations=2, seed=5, cases=97)
    g = copy.deepcopy(files.grammar)
    for alt in g["nonterminals"][0]["alternatives"]:
        if alt["id"] == "imod0":
            alt["expression"]["signature"] = "mod(Int,Int)->Int"
    files.grammar = g
    lt = _task(tmp_path, files)
    gb = abi.GrammarBlob(lt.tables)
    rows = oracle.initial_population(gb, lt.settings)
    f, w = engine.evaluate_rows(lt, rows)
    want_f, want_w, _ = oracle.evaluate(gb, lt.cases, lt.settings, rows)
    assert np.array_equal(f, want_f)
    assert np.array_equal(w, want_w)
    assert (f <= -1000).any()  # some programs divide by zero on some case


def test_evaluate_many_cases_and_lanes(engine, tmp_path):
    """Case counts around the VM's lane tiling (1, 2, 4 cases per lane, tails)."""
    for cases in (1, 31, 33, 64, 65, 129, 300):
        files = W.poly4(population=128, generations=2, seed=cases, cases=cases)
        lt = _task(tmp_path / str(cases), files)
        gb = abi.GrammarBlob(lt.tables)
        rows = oracle.initial_population(gb, lt.settings)
        f, w = engine.evaluate_rows(lt, rows)
        want_f, want_w, _ = oracle.evaluate(gb, lt.cases, lt.settings, rows)
        assert np.array_equal(f, want_f), cases
        assert np.array_equal(w, want_w), cases
