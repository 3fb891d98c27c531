"""The C-ABI boundary driven from the reference's own code (GPU).

oracle/_ref/reference_adapter is tests/native/reference_adapter.cpp -- the
reference-side binding a maintainer adds -- compiled
against the reference's sources and linked with its CPU engine and
libgagp_b200.so.  For each task it builds the engine's tables with the
reference's own phase compiler (compile_phase_grammar), runs the search
through gagp_b200_search_create/run/result, maps the ranked population back
to the reference's genomes through export_native_phase_layout, and compares
with the reference CPU engine's evolve_population on the same task: the
history, the final ranked population (fitness, wrong counts, programs) and
the evaluation counters must be equal."""
import json
import os
import subprocess

import pytest

from gagp_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "oracle", "_ref", "reference_adapter")

TASKS = [
    ("poly4", lambda: W.poly4(population=256, generations=6, seed=5, cases=48, max_nodes=40)),
    ("polynomial", lambda: W.polynomial(population=300, generations=8, seed=2)),
    ("list_threshold", lambda: W.list_threshold(population=128, generations=4, seed=6, cases=30)),
    ("list_max_reservoir", lambda: _with_search(W.list_threshold(population=96, generations=3, seed=7, cases=20,
                                                                 target="max"),
                                                {"sites": {"scope": "genome", "draw": "reservoir"}})),
    ("poly4_generational", lambda: _with_search(W.poly4(population=200, generations=5, seed=8, cases=32,
                                                        max_nodes=40),
                                                {"schedule": {"mode": "generational"}, "elitism": 2})),
    ("list_statements", lambda: W.list_statements(population=128, generations=4, seed=9, cases=24)),
    ("grid_paths", lambda: W.grid_paths(population=128, generations=4, seed=10, cases=30)),
    ("poly4_fuel_charges", lambda: _with_fuel(W.poly4(population=192, generations=5, seed=11, cases=32,
                                                      max_nodes=40))),
    ("list_traversal_fuel", lambda: _with_traversal_fuel(W.list_threshold(population=128, generations=4, seed=12,
                                                                          cases=24))),
]


def _with_traversal_fuel(files):
    """A fuel profile on the list grammar's traversal (every event charged
    at least 1)."""
    top = next(r for r in files.grammar["nonterminals"] if r["id"] == "Top")
    top["alternatives"][0]["expression"]["fuel_events"] = {"store_sequence": 2, "test_cursor": 3, "read_element": 2,
                                                           "advance_cursor": 2, "result": 4}
    return files


def _with_fuel(files):
    """Node-level fuel charges on the large scalar grammar: input reads cost
    2, constants 0, mul 3, the value if's test 2 and merge 0."""
    charges = {"x": {"operation": 2}, "c": {"operation": 0}, "mul": {"operation": 3},
               "iflt": {"branch_test": 2, "branch_merge": 0}}
    for nt in files.grammar["nonterminals"]:
        for alt in nt["alternatives"]:
            if alt["id"] in charges:
                alt["expression"]["fuel_events"] = charges[alt["id"]]
    return files


def _with_search(files, extra):
    files.search.update(extra)
    return files


@pytest.mark.parametrize("name,make", TASKS, ids=[t[0] for t in TASKS])
def test_reference_adapter_matches_reference_engine(tmp_path, name, make):
    assert os.path.exists(ADAPTER), "build it with make -C oracle boundary (gagp_b200 build does)"
    task = make().write(str(tmp_path))
    out = subprocess.run([ADAPTER, task, str(tmp_path / "search.json")], check=True, capture_output=True, text=True,
                         timeout=600).stdout
    r = json.loads(out)
    print(json.dumps(r))
    assert r["ran"], r["declined"]
    assert r["reference_declined"] == ""
    assert r["history_equal"], json.dumps(r)
    assert r["final_equal"], json.dumps(r)
    assert r["program_cases"][0] == r["program_cases"][1], r
    assert r["reused_programs"][0] == r["reused_programs"][1], r
    assert r["best"][0] == r["best"][1]
