"""Regenerates the golden fixtures of this directory from the reference's own
CPU engine, compiled from its sources by ``make -C oracle ref``.

Each fixture ``<name>.json.gz`` holds the task file set (grammar, train cases,
search config) and the reference's outputs for it: the admitted phase tables
and initial population rows (``ref_driver tables``) and one complete CPU
search (``ref_driver run``: per-generation history and the final ranked
population with fitness, wrong counts, node counts, program text and rows).

Run here (the container with the reference tree):
    python tests/golden/make_golden.py [--list-only]
"""
from __future__ import annotations

import gzip
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gagp_b200 import workloads as W  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

# name, workload, workload arguments, search-config overrides
CASES = [
    ("polynomial_p1024_g64", "polynomial", dict(population=1024, generations=64, seed=0), {}),
    ("poly4_p512_g12_s1", "poly4", dict(population=512, generations=12, seed=1, cases=100), {}),
    ("poly4_genome_reservoir", "poly4", dict(population=256, generations=10, seed=2, cases=50),
     {"sites": {"scope": "genome", "draw": "reservoir"}}),
    ("poly4_gate1_mutcap5", "poly4", dict(population=256, generations=10, seed=3, cases=50),
     {"crossover": {"probability": 1.0, "attempts": 3}, "mutation": {"probability": 0.5, "max_subtree_nodes": 5}}),
    ("poly4_batch64_repl3", "poly4", dict(population=256, generations=10, seed=4, cases=50),
     {"schedule": {"mode": "steady_state", "batch": 64, "replacement_size": 3}}),
    ("poly4_sitedepth4_t4", "poly4", dict(population=300, generations=10, seed=5, cases=33),
     {"limits": {"site_depth": 4}, "selection": {"method": "tournament", "size": 4}}),
    ("poly4_sitedepth1", "poly4", dict(population=256, generations=8, seed=6, cases=40), {"limits": {"site_depth": 1}}),
    ("polynomial_grammar_sites", "polynomial", dict(population=200, generations=20, seed=9),
     {"ranking": {"tie_break": "grammar_sites"}}),
    ("poly4_exact_metric", "poly4", dict(population=256, generations=6, seed=7, cases=64), {}),
    ("int64_edges", "int64_edges", dict(population=256, generations=8, seed=8), {}),
]


# List programs (traversals over an IntList, lets, statement programs):
# the reference's tables, initial rows, one make_batch and whole runs of the
# list path.  They live in golden/list/.
LIST_CASES = [
    ("list_threshold_sum", dict(population=64, generations=3, seed=11, cases=12, target="threshold_sum"), None),
    ("list_threshold_count", dict(population=64, generations=3, seed=12, cases=12, target="threshold_count"), None),
    ("list_nested_traversal", dict(population=64, generations=3, seed=13, cases=12, target="max"), "nested"),
    ("list_statements_sum", dict(population=64, generations=3, seed=16, cases=12, target="threshold_sum"),
     "statements"),
]


# the round seed of the recorded make_batch (ref_driver batch)
LIST_ROUND_SEED = 0x9E3779B97F4A7C15

# Whole list searches recorded without a make_batch: a reverse traversal,
# and the list-program benchmark's shape (200 cases, lists of 0..50
# elements, P = 1024) over 16 generations.
LIST_RUNS = [
    ("list_reverse_traversal", dict(population=96, generations=4, seed=14, cases=16, target="max"), "reverse"),
    ("list_config3_p1024_g16", dict(population=1024, generations=16, seed=0, cases=200, target="threshold_sum"),
     None),
    ("list_let_p256_g8", dict(population=256, generations=8, seed=15, cases=30, target="threshold_sum"), "let"),
    ("list_statements_p512_g8", dict(population=512, generations=8, seed=17, cases=40, target="threshold_sum"),
     "statements"),
    ("list_statements_p2048_g12", dict(population=2048, generations=12, seed=18, cases=100, target="max"),
     "statements"),
]

# Lowering pins (golden/lower/): the reference's phase compiler output and
# CPU fitness of every member of a generated population (ref_driver lower).
LOWER_CASES = [
    ("lower_list_threshold", "list", dict(population=256, generations=1, seed=21, cases=24), None),
    ("lower_list_nested", "list", dict(population=256, generations=1, seed=22, cases=24, target="max"), "nested"),
    ("lower_list_reverse", "list", dict(population=256, generations=1, seed=23, cases=24, target="max"), "reverse"),
    ("lower_poly4", "poly4", dict(population=256, generations=1, seed=24, cases=32), None),
    ("lower_list_deep", "list", dict(population=384, generations=1, seed=25, cases=40, target="max"), "deep"),
    ("lower_int64_edges", "int64_edges", dict(population=512, generations=1, seed=26), None),
    ("lower_list_let", "list", dict(population=384, generations=1, seed=27, cases=24, target="threshold_sum"), "let"),
    ("lower_scalar_let", "scalar_let", dict(population=384, generations=1, seed=28, cases=32), None),
    ("lower_list_statements", "list_statements", dict(population=512, generations=1, seed=29, cases=24), None),
    ("lower_grid_paths", "grid_paths", dict(population=512, generations=1, seed=63, cases=30), None),
    ("lower_scalar_fuel", "scalar_fuel", dict(population=384, generations=1, seed=30, cases=32), None),
    ("lower_list_fuel", "list", dict(population=256, generations=1, seed=31, cases=24), "fuel"),
]

# Bounded regions (golden/region/): the lattice-path workload, whose
# grammar holds a memoized coordinate recurrence with evolved phases.  The
# first fixture also holds the reference's tables, initial rows and one
# make_batch.
REGION_CASES = [
    ("region_grid_paths_p256", dict(population=256, generations=6, seed=61, cases=30), True),
    ("region_grid_paths_p1024_g16", dict(population=1024, generations=16, seed=62, cases=49), False),
    # an ambiguous grammar: the reference's initial rows are re-derived
    # (first matching production) from the generated programs
    ("region_grid_paths_ambiguous_p1024", dict(population=1024, generations=6, seed=62, cases=49, ambiguous=True),
     False),
]


def region_fixtures() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "region"), exist_ok=True)
    for name, kwargs, full in REGION_CASES:
        task = W.grid_paths(**kwargs)
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            run = driver("run", tp, "--search", sp)
            if full:
                tables = driver("tables", tp, "--search", sp)
                batch = driver("batch", tp, "--search", sp, "--round-seed", str(LIST_ROUND_SEED))
        assert run["declined"] == "", (name, run["declined"])
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "run": run}
        if full:
            fixture.update(tables={k: v for k, v in tables.items() if k != "initial"},
                           initial=[rows[0] for rows in tables["initial"]], batch=batch)
        with gzip.open(os.path.join(here, "region", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(run["history"]), "history entries,", len(run["final"]), "final members")


# int64 edge values: the extremes, the 32-bit boundaries the fast VM's
# division shortcut tests, and a pair whose squares do and do not wrap.  The
# reference reads case integers through a double (cpp/src/cli/codec.cpp:70-78),
# so every value here is one a double holds exactly: INT64_MIN, INT64_MIN +
# 2048 and INT64_MAX - 2047 (2^63 - 2048) are the extremes it accepts.
INT64_EDGE_X = [-2 ** 63, -2 ** 63 + 2048, 2 ** 63 - 2048, -2 ** 62, 2 ** 62, 2 ** 62 + 4096, -2 ** 31 - 1, -2 ** 31,
                2 ** 31 - 1, 2 ** 31, 3037000499, -3037000500, -1, 0, 1, 7, -7, 100, -100]


def int64_edge_target(x: int) -> int:
    """x*x - 3 where it is exact in a double, else x itself."""
    return x * x - 3 if abs(x) < 2 ** 26 else x


def int64_edge_task(population: int, generations: int, seed: int) -> "W.TaskFiles":
    """The large scalar grammar plus Python-sign `mod` (ZeroDiv on 0) and
    `neg`, on cases at int64 edge values, where programs wrap."""
    g = W.poly4_grammar(max_nodes=40)
    alts = g["nonterminals"][0]["alternatives"]
    ref = {"ref": "Expr"}
    alts.append({"id": "mod", "weight": 1, "expression": {"signature": "mod(Int,Int)->Int", "args": [ref, ref]}})
    alts.append({"id": "neg", "weight": 1, "expression": {"signature": "neg(Int)->Int", "args": [ref]}})
    train = [W._int_case(x, int64_edge_target(x)) for x in INT64_EDGE_X]
    return W.TaskFiles(name="int64-edges-s%d" % seed, grammar=g, train=train,
                       search=W.search_config(population, generations, seed))


def nested_traversal_grammar() -> dict:
    """The list grammar with a second traversal inside the step, whose body
    nonterminal maps the outer accumulator and the inner binders by name
    (binder numbers 3..5, scope map [2, 3, 5])."""
    g = W.list_threshold_grammar()
    step = next(r for r in g["nonterminals"] if r["id"] == "Step")
    step["alternatives"].append({"id": "inner", "weight": 1, "expression": {
        "signature": "traverse(IntList,Int,Int,Int)->Int",
        "args": [{"input": "xs"}, {"constant": {"type": "Int", "values": ["0"]}}, {"bound": "acc"}, {"ref": "Inner"}],
        "bind": {"3": ["e2", "i2", "acc2"]}}})
    g["nonterminals"].append({"id": "Inner", "type": "Int", "scope": [
        {"name": "acc", "type": "Int"}, {"name": "e2", "type": "Int"}, {"name": "acc2", "type": "Int"}],
        "alternatives": [
            {"id": "acc", "weight": 1, "expression": {"bound": "acc"}},
            {"id": "e2", "weight": 1, "expression": {"bound": "e2"}},
            {"id": "sum", "weight": 2, "expression": {"signature": "add(Int,Int)->Int",
                                                      "args": [{"bound": "acc2"}, {"bound": "e2"}]}}]})
    return g


def deep_traversal_grammar() -> dict:
    """The nested-traversal grammar with a third traversal inside the inner
    body (binder numbers 6..8): a program with all three open needs 29
    locals (2 inputs + 3 x 9 temporaries)."""
    g = nested_traversal_grammar()
    inner = next(r for r in g["nonterminals"] if r["id"] == "Inner")
    inner["alternatives"].append({"id": "inner2", "weight": 2, "expression": {
        "signature": "traverse(IntList,Int,Int,Int)->Int",
        "args": [{"input": "xs"}, {"constant": {"type": "Int", "values": ["1"]}}, {"bound": "acc2"}, {"ref": "Inner2"}],
        "bind": {"3": ["e3", "i3", "acc3"]}}})
    g["nonterminals"].append({"id": "Inner2", "type": "Int", "scope": [
        {"name": "e2", "type": "Int"}, {"name": "e3", "type": "Int"}, {"name": "i3", "type": "Int"},
        {"name": "acc3", "type": "Int"}],
        "alternatives": [
            {"id": "acc3", "weight": 1, "expression": {"bound": "acc3"}},
            {"id": "max", "weight": 2, "expression": {"signature": "if(Bool,Int,Int)->Int", "args": [
                {"signature": "gt(Int,Int)->Bool", "args": [{"bound": "e3"}, {"bound": "acc3"}]},
                {"bound": "e3"}, {"bound": "acc3"}]}},
            {"id": "idx", "weight": 1, "expression": {"signature": "add(Int,Int)->Int",
                                                      "args": [{"bound": "i3"}, {"bound": "e2"}]}}]})
    return g


def reverse_traversal_grammar() -> dict:
    """The list grammar with the fold as a reverse traversal beside the
    forward one."""
    g = W.list_threshold_grammar()
    top = next(r for r in g["nonterminals"] if r["id"] == "Top")
    fold = top["alternatives"][0]["expression"]
    top["alternatives"].append({"id": "rfold", "weight": 2, "expression": dict(
        fold, signature="traverse_reverse(IntList,Int,Int,Int)->Int")})
    return g


def let_grammar() -> dict:
    """The list grammar with lets: the step may bind a value (an Int or a
    comparison) for a body that reads it, and lets nest inside traversal
    bodies and inside each other."""
    g = W.list_threshold_grammar()
    step = {"ref": "Step"}
    steps = next(r for r in g["nonterminals"] if r["id"] == "Step")
    steps["alternatives"].append({"id": "let_int", "weight": 1, "expression": {
        "signature": "let(Int,Int)->Int", "args": [step, {"ref": "LetBody"}], "bind": {"1": ["v"]}}})
    g["nonterminals"].append({
        "id": "LetBody", "type": "Int",
        "scope": [{"name": "element", "type": "Int"}, {"name": "acc", "type": "Int"}, {"name": "v", "type": "Int"}],
        "alternatives": [
            {"id": "v", "weight": 3, "expression": {"bound": "v"}},
            {"id": "element", "weight": 1, "expression": {"bound": "element"}},
            {"id": "acc", "weight": 1, "expression": {"bound": "acc"}},
            {"id": "add", "weight": 2, "expression": {"signature": "add(Int,Int)->Int",
                                                      "args": [{"ref": "LetBody"}, {"ref": "LetBody"}]}},
            {"id": "sub", "weight": 1, "expression": {"signature": "sub(Int,Int)->Int",
                                                      "args": [{"ref": "LetBody"}, {"ref": "LetBody"}]}},
            {"id": "pick", "weight": 1, "expression": {"signature": "if(Bool,Int,Int)->Int", "args": [
                {"signature": "gt(Int,Int)->Bool", "args": [{"ref": "LetBody"}, {"ref": "LetBody"}]},
                {"ref": "LetBody"}, {"ref": "LetBody"}]}}]})
    return g


def scalar_let_grammar() -> dict:
    """The large scalar grammar with a let whose body sees the bound value."""
    g = W.poly4_grammar(max_nodes=40)
    expr = next(r for r in g["nonterminals"] if r["id"] == "Expr")
    expr["alternatives"].append({"id": "let", "weight": 1, "expression": {
        "signature": "let(Int,Int)->Int", "args": [{"ref": "Expr"}, {"ref": "Body"}], "bind": {"1": ["y"]}}})
    g["nonterminals"].append({
        "id": "Body", "type": "Int", "scope": [{"name": "y", "type": "Int"}],
        "alternatives": [
            {"id": "y", "weight": 3, "expression": {"bound": "y"}},
            {"id": "x", "weight": 1, "expression": {"input": "x"}},
            {"id": "k", "weight": 1, "expression": {"constant": {"type": "Int", "range": ["-2", "3"]}}},
            {"id": "add", "weight": 1, "expression": {"signature": "add(Int,Int)->Int",
                                                      "args": [{"ref": "Body"}, {"ref": "Body"}]}},
            {"id": "mul", "weight": 1, "expression": {"signature": "mul(Int,Int)->Int",
                                                      "args": [{"ref": "Body"}, {"ref": "Body"}]}}]})
    return g


def scalar_fuel_grammar() -> dict:
    """The scalar let grammar with node-level fuel charges: input reads cost
    2, constants 0, a let's bind 0, the body's mul 3, and the value if's test
    2 and merge 0."""
    g = scalar_let_grammar()
    charges = {("Expr", "x"): {"operation": 2}, ("Expr", "c"): {"operation": 0},
               ("Expr", "iflt"): {"branch_test": 2, "branch_merge": 0}, ("Expr", "let"): {"bind": 0},
               ("Body", "mul"): {"operation": 3}}
    for nt in g["nonterminals"]:
        for alt in nt["alternatives"]:
            if (nt["id"], alt["id"]) in charges:
                alt["expression"]["fuel_events"] = charges[(nt["id"], alt["id"])]
    return g


def list_fuel_grammar() -> dict:
    """The list grammar whose traversal carries a fuel profile (every event
    charged at least 1)."""
    g = W.list_threshold_grammar()
    top = next(r for r in g["nonterminals"] if r["id"] == "Top")
    top["alternatives"][0]["expression"]["fuel_events"] = {
        "store_sequence": 4, "test_cursor": 3, "read_element": 2, "compute_index": 2, "update_state": 2,
        "repeat": 1, "result": 2}
    return g


def variant_grammar(variant):
    if variant == "let":
        return let_grammar()
    if variant == "nested":
        return nested_traversal_grammar()
    if variant == "reverse":
        return reverse_traversal_grammar()
    if variant == "deep":
        return deep_traversal_grammar()
    if variant == "statements":
        return W.list_statements_grammar()
    if variant == "fuel":
        return list_fuel_grammar()
    return None


# Generational schedule (golden/generational/): whole reference CPU-engine
# searches under schedule.mode generational with elites
# (run_phase_population, cpp/src/evolution/evolve.cpp:253-322).
GEN_CASES = [
    ("gen_poly4_e1", "poly4", dict(population=256, generations=8, seed=41, cases=48), {"elitism": 1}),
    ("gen_poly4_e4_t3", "poly4", dict(population=300, generations=8, seed=42, cases=40),
     {"elitism": 4, "selection": {"method": "tournament", "size": 3}}),
    ("gen_polynomial_e0", "polynomial", dict(population=200, generations=10, seed=43), {"elitism": 0}),
    ("gen_poly4_exact_e2", "poly4_exact", dict(population=256, generations=6, seed=44, cases=40), {"elitism": 2}),
    ("gen_list_e2", "list", dict(population=128, generations=5, seed=45, cases=20), {"elitism": 2}),
    ("gen_poly4_p4096", "poly4", dict(population=4096, generations=4, seed=46, cases=64), {"elitism": 3}),
    ("gen_statements_e2", "list_statements", dict(population=128, generations=5, seed=47, cases=20), {"elitism": 2}),
]


def gen_fixtures() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "generational"), exist_ok=True)
    for name, workload, kwargs, extra in GEN_CASES:
        if workload == "list":
            task = W.list_threshold(**kwargs)
        elif workload == "poly4_exact":
            task = W.poly4(**kwargs)
            task.fitness = {"metric": "exact"}
        else:
            task = W.make(workload, **kwargs)
        task.search.update(extra)
        task.search["schedule"] = {"mode": "generational"}
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            run = driver("run", tp, "--search", sp)
        assert run["declined"] == "", (name, run["declined"])
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "run": run}
        with gzip.open(os.path.join(here, "generational", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(run["history"]), "history entries,", len(run["final"]), "final members",
              run["program_cases"], "program-cases,", run["reused_programs"], "reused")


# Imported initial populations (golden/init/): a short reference search A,
# then a search B of the same task started from A's final population
# (`ref_driver run --init`, as `gagp run --init`, run.cpp:146-174).
INIT_CASES = [
    ("init_poly4", "poly4", dict(population=128, generations=3, seed=51, cases=40, max_nodes=40), 6, {}),
    ("init_list", "list", dict(population=96, generations=2, seed=52, cases=20), 4, {}),
    ("init_generational", "poly4", dict(population=120, generations=3, seed=53, cases=32, max_nodes=40), 5,
     {"schedule": {"mode": "generational"}, "elitism": 2}),
    ("init_statements", "list_statements", dict(population=96, generations=2, seed=54, cases=20), 4, {}),
]


def init_fixtures() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "init"), exist_ok=True)
    for name, workload, kwargs, generations_b, extra in INIT_CASES:
        task = W.list_threshold(**kwargs) if workload == "list" else W.make(workload, **kwargs)
        task.search.update(extra)
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            first = driver("run", tp, "--search", sp)
            pp = os.path.join(d, "population.json")
            with open(pp, "w") as f:
                json.dump({"format": "gagp-population-v1", "programs": [m["program"] for m in first["final"]]}, f)
            run = driver("run", tp, "--search", sp, "--init", pp, "--generations", str(generations_b))
        assert run["declined"] == "", (name, run["declined"])
        task.search["generations"] = generations_b
        initial = [{"origins": m["rows"][0]["origins"], "constants": [c[1] for c in m["rows"][0]["constants"]]}
                   for m in first["final"]]
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "initial": initial, "run": run}
        with gzip.open(os.path.join(here, "init", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(initial), "imported members,", len(run["history"]), "history entries")


# Judgement pins (golden/judge/): the reference's `gagp eval --split test`
# verdict (cpp/src/cli/run.cpp:176-238) of generated programs on a test split,
# and one `gagp run` whose result carries the best program's test verdict.
JUDGE_CASES = [
    ("judge_int64_edges", "int64_edges", dict(population=160, generations=1, seed=31)),
    ("judge_polynomial", "polynomial", dict(population=96, generations=1, seed=32)),
    ("judge_list", "list", dict(population=96, generations=1, seed=33, cases=24)),
    ("judge_bool_absolute", "bool", dict(population=96, generations=1, seed=34)),
    ("judge_bool_exact", "bool_exact", dict(population=96, generations=1, seed=35)),
    ("judge_poly4_exact", "poly4_exact", dict(population=96, generations=1, seed=36, cases=40)),
    ("judge_statements", "statements", dict(population=96, generations=1, seed=38, cases=24)),
]
JUDGE_RUN = ("judge_run_polynomial", dict(population=512, generations=24, seed=37))
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "gagp")


def bool_task(population: int, generations: int, seed: int, metric: str = "absolute") -> "W.TaskFiles":
    """A Bool-valued program grammar (comparisons of Int terms, not/and, and a
    Python-sign `mod` that fails on 0) with target x mod 3 == 1 read as x > 2
    and x < 9; the absolute metric scores a Bool case at the penalty ceiling
    whatever its value, the judge counts it correct when it equals."""
    e, c = {"ref": "E"}, {"ref": "Cond"}
    g = {"format_version": "grammar-definition-v2", "entry": {"nonterminal": "Cond", "type": "Bool"},
         "inputs": [{"name": "x", "type": "Int"}], "search_limits": {"max_nodes": 24, "max_depth": 6},
         "execution_limits": {"fuel": 1000},
         "nonterminals": [
             {"id": "Cond", "type": "Bool", "scope": [], "alternatives": [
                 {"id": "lt", "weight": 2, "expression": {"signature": "lt(Int,Int)->Bool", "args": [e, e]}},
                 {"id": "gt", "weight": 2, "expression": {"signature": "gt(Int,Int)->Bool", "args": [e, e]}},
                 {"id": "not", "weight": 1, "expression": {"signature": "not(Bool)->Bool", "args": [c]}},
                 {"id": "and", "weight": 1, "expression": {"signature": "and(Bool,Bool)->Bool", "args": [c, c]}}]},
             {"id": "E", "type": "Int", "scope": [], "alternatives": [
                 {"id": "x", "weight": 3, "expression": {"input": "x"}},
                 {"id": "k", "weight": 2, "expression": {"constant": {"type": "Int", "range": ["-3", "9"]}}},
                 {"id": "add", "weight": 1, "expression": {"signature": "add(Int,Int)->Int", "args": [e, e]}},
                 {"id": "mod", "weight": 1, "expression": {"signature": "mod(Int,Int)->Int", "args": [e, e]}}]}]}

    def case(x):
        return {"inputs": {"x": {"type": "int", "value": x}}, "expected": {"type": "bool", "value": 2 < x < 9}}
    fitness = {"metric": metric, "case_cap": 7} if metric == "absolute" else {"metric": "exact"}
    return W.TaskFiles(name="bool-%s-s%d" % (metric, seed), grammar=g, train=[case(x) for x in range(-6, 14)],
                       test=[case(x) for x in range(-10, 20, 3)] + [case(0)], fitness=fitness,
                       search=W.search_config(population, generations, seed))


def judge_task(workload: str, kwargs: dict) -> "W.TaskFiles":
    """A task with a test split for the judgement pins."""
    if workload == "int64_edges":
        task = int64_edge_task(**kwargs)
        task.test = [W._int_case(x, int64_edge_target(x) + (x & 1)) for x in reversed(INT64_EDGE_X)]
    elif workload == "polynomial":
        task = W.polynomial(**kwargs)
    elif workload == "list":
        task = W.list_threshold(**kwargs)
        task.test = W.list_threshold(population=8, generations=1, seed=kwargs["seed"] + 1000, cases=30).train
    elif workload == "statements":
        task = W.list_statements(**kwargs)
        task.test = W.list_threshold(population=8, generations=1, seed=kwargs["seed"] + 1000, cases=30).train
    elif workload == "bool":
        task = bool_task(**kwargs)
    elif workload == "bool_exact":
        task = bool_task(**kwargs, metric="exact")
    else:
        task = W.poly4(**kwargs)
        task.fitness = {"metric": "exact"}
        task.test = W.poly4(population=8, generations=1, seed=kwargs["seed"] + 1000, cases=25).train
    assert task.test, workload
    return task


def judge_fixtures() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "judge"), exist_ok=True)
    for name, workload, kwargs in JUDGE_CASES:
        task = judge_task(workload, kwargs)
        rows = []
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            lowered = driver("lower", tp, "--search", sp)
            for r in lowered["rows"]:
                if r["status"] != 0:
                    continue
                pp = os.path.join(d, "program.json")
                with open(pp, "w") as f:
                    json.dump(r["program"], f)
                out = subprocess.run([REF_CLI, "eval", tp, pp, "--split", "test"], check=True, capture_output=True,
                                     text=True).stdout
                verdict = json.loads(out)
                rows.append({"origins": r["origins"], "constants": r["constants"],
                             "verdict": {k: verdict[k] for k in ("cases", "correct", "wrong", "runtime_errors",
                                                                 "mean_loss", "solved")}})
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "rows": rows}
        with gzip.open(os.path.join(here, "judge", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        errors = sum(1 for r in rows if r["verdict"]["runtime_errors"])
        print(name, len(rows), "programs,", errors, "with runtime errors")
    name, kwargs = JUDGE_RUN
    task = W.polynomial(**kwargs)
    with tempfile.TemporaryDirectory() as d:
        task.write(d)
        tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
        subprocess.run([REF_CLI, "run", tp, "--engine", "cpu", "--search", sp, "--out", os.path.join(d, "out"),
                        "--quiet"], check=True, capture_output=True)
        with open(os.path.join(d, "out", "result.json")) as f:
            result = json.load(f)
        run = driver("run", tp, "--search", sp)
    assert result["best"]["text"] == run["final"][0]["text"], "the CLI and the driver ran different searches"
    fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
               "train": task.train, "test": task.test, "search": task.search,
               "best": {k: result["best"][k] for k in ("fitness", "wrong", "nodes", "text")}, "test_verdict": result["test"],
               "run": {"history": run["history"], "final": run["final"][:4], "program_cases": run["program_cases"],
                       "reused_programs": run["reused_programs"]}}
    with gzip.open(os.path.join(here, "judge", name + ".json.gz"), "wt") as f:
        json.dump(fixture, f, separators=(",", ":"))
    print(name, "best", result["best"]["text"], "test", result["test"])


def driver(*args) -> dict:
    out = subprocess.run([DRIVER, *args], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def main() -> None:
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--list-only", action="store_true", help="regenerate golden/list/ only")
    ap.add_argument("--lower-only", action="store_true", help="regenerate golden/lower/ only")
    ap.add_argument("--judge-only", action="store_true", help="regenerate golden/judge/ only")
    ap.add_argument("--generational-only", action="store_true", help="regenerate golden/generational/ only")
    ap.add_argument("--init-only", action="store_true", help="regenerate golden/init/ only")
    ap.add_argument("--region-only", action="store_true", help="regenerate golden/region/ only")
    ap.add_argument("--headline", action="store_true",
                    help="regenerate golden/headline/ only (the benchmark's search, several minutes)")
    args = ap.parse_args()
    if args.headline:
        headline_fixture()
        return
    if args.lower_only:
        lower_fixtures()
        return
    if args.judge_only:
        judge_fixtures()
        return
    if args.generational_only:
        gen_fixtures()
        return
    if args.region_only:
        region_fixtures()
        return
    if args.init_only:
        init_fixtures()
        return
    if not os.path.exists(DRIVER):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    here = os.path.dirname(os.path.abspath(__file__))
    for name, workload, kwargs, extra in ([] if args.list_only else CASES):
        task = int64_edge_task(**kwargs) if workload == "int64_edges" else W.make(workload, **kwargs)
        task.search.update(extra)
        if name.endswith("exact_metric"):
            task.fitness = {"metric": "exact"}
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            tables = driver("tables", tp, "--search", sp)
            run = driver("run", tp, "--search", sp)
        fixture = {
            "name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
            "train": task.train, "test": task.test, "search": task.search,
            "tables": {k: v for k, v in tables.items() if k != "initial"},
            "initial": [rows[0] for rows in tables["initial"]],
            "run": run,
        }
        with gzip.open(os.path.join(here, name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(run["history"]), "history entries,", len(run["final"]), "final members")
    os.makedirs(os.path.join(here, "list"), exist_ok=True)
    for name, kwargs, variant in LIST_CASES:
        task = W.list_threshold(**kwargs)
        if variant:
            task.grammar = variant_grammar(variant)
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            tables = driver("tables", tp, "--search", sp)
            run = driver("run", tp, "--search", sp)
            batch = driver("batch", tp, "--search", sp, "--round-seed", str(LIST_ROUND_SEED))
        assert run["declined"] == "", (name, run["declined"])
        fixture = {
            "name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
            "train": task.train, "test": task.test, "search": task.search,
            "tables": {k: v for k, v in tables.items() if k != "initial"},
            "initial": [rows[0] for rows in tables["initial"]],
            "run": run,
            "batch": batch,
        }
        with gzip.open(os.path.join(here, "list", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(run["history"]), "history entries,", len(run["final"]), "final members")
    for name, kwargs, variant in LIST_RUNS:
        task = W.list_threshold(**kwargs)
        if variant:
            task.grammar = variant_grammar(variant)
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            run = driver("run", tp, "--search", sp)
        assert run["declined"] == "", (name, run["declined"])
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "run": run}
        with gzip.open(os.path.join(here, "list", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(run["history"]), "history entries,", len(run["final"]), "final members")
    lower_fixtures()
    judge_fixtures()
    gen_fixtures()
    init_fixtures()
    region_fixtures()


def row_digest(rows) -> str:
    """SHA-256 over the ranked rows' construction expressions and constants."""
    import hashlib
    h = hashlib.sha256()
    for r in rows:
        h.update(json.dumps([r["origins"], [c[1] for c in r["constants"]]], separators=(",", ":")).encode())
    return h.hexdigest()


def headline_fixture() -> None:
    """The benchmark's own search (large scalar regression: P = 16384, 128
    generations, 256 cases, max 64 nodes, seed 0) run whole by the reference
    CPU engine: the full history, the final ranked fitness, wrong and node
    vectors, the best 256 rows and a digest of all 16384 ranked rows."""
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "headline"), exist_ok=True)
    task = W.poly4(population=16384, generations=128, seed=0, cases=256, max_nodes=64)
    with tempfile.TemporaryDirectory() as d:
        task.write(d)
        tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
        run = driver("run", tp, "--search", sp)
    final = run["final"]
    fixture = {"name": "poly4_p16384_g128_s0", "task": {"name": task.name, "fitness": task.fitness},
               "grammar": task.grammar, "train": task.train, "test": task.test, "search": task.search,
               "run": {"declined": run["declined"], "time_ms": run["time_ms"], "program_cases": run["program_cases"],
                       "reused_programs": run["reused_programs"], "history": run["history"],
                       "final_fitness": [m["fitness"] for m in final], "final_wrong": [m["wrong"] for m in final],
                       "final_nodes": [m["nodes"] for m in final],
                       "top": [dict(m, rows=m["rows"]) for m in final[:256]],
                       "row_digest": row_digest([m["rows"][0] for m in final])}}
    with gzip.open(os.path.join(here, "headline", "poly4_p16384_g128_s0.json.gz"), "wt") as f:
        json.dump(fixture, f, separators=(",", ":"))
    print("headline", len(run["history"]), "history entries,", len(final), "final members",
          "%.1f s" % (run["time_ms"] / 1000.0))


def lower_fixtures() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "lower"), exist_ok=True)
    for name, workload, kwargs, variant in LOWER_CASES:
        if workload == "list":
            task = W.list_threshold(**kwargs)
        elif workload == "int64_edges":
            task = int64_edge_task(**kwargs)
        elif workload == "scalar_let":
            task = W.poly4(**kwargs)
            task.grammar = scalar_let_grammar()
        elif workload == "scalar_fuel":
            task = W.poly4(**kwargs)
            task.grammar = scalar_fuel_grammar()
        else:
            task = W.make(workload, **kwargs)
        if variant:
            task.grammar = variant_grammar(variant)
        with tempfile.TemporaryDirectory() as d:
            task.write(d)
            tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
            lowered = driver("lower", tp, "--search", sp, "--case-detail", "4")
        fixture = {"name": name, "task": {"name": task.name, "fitness": task.fitness}, "grammar": task.grammar,
                   "train": task.train, "test": task.test, "search": task.search, "lower": lowered}
        with gzip.open(os.path.join(here, "lower", name + ".json.gz"), "wt") as f:
            json.dump(fixture, f, separators=(",", ":"))
        print(name, len(lowered["rows"]), "rows")


if __name__ == "__main__":
    main()
