"""Deterministic synthetic GAGP tasks in the reference's file formats.

Every task is written as the reference's ``gagp-task-v1`` file set
(``spec/task.md``): a ``grammar-definition-v2`` grammar, ``fitness-cases``
train/test files and an absolute-error fitness policy, plus a
``gagp-search-config-v1`` search file.  The same files drive the reference CPU
engine (``gagp run --engine cpu``) and this engine, so both search the same
problem from the same seed.

Workloads:

* ``polynomial``  -- scalar integer regression of y = x^3 - 2x + 1; x = -10..10
  train cases, 40 test cases x ~ U[-50, 50]; grammar x (w3), constants {0,1,2}
  (w2), add/sub/mul (w1); max 31 nodes, depth 8, fuel 1000.
* ``poly4``       -- random integer polynomial of degree <= 4, coefficients
  U{-5..5} from the seed; train x ~ U{-100..100}; grammar x, constants
  -2..3, add/sub/mul/idiv0/imod0 and if(lt(E,E),E,E); max 64 nodes, depth 16,
  fuel 1000.
* ``list_threshold`` -- list programs with a loop: xs an IntList of length
  U{0..50} with elements U[-1000, 1000] and a threshold t ~ U{-100..100};
  the target is the sum of the elements above t, their count, or the
  maximum (0 for an empty list); the grammar folds xs with a traversal
  whose step (binders element, index, accumulator) adds, subtracts and
  compares.
* ``list_statements`` -- the same list cases searched by a statement
  program: a Program entry whose blocks assign grammar locals, loop with
  for_range, branch with if_stmt and return, reading xs through len and
  index.

Inputs are generated with ``random.Random(seed)``.
"""
from __future__ import annotations

import json
import math
import os
import random
from dataclasses import dataclass, field
from typing import Dict, List, Optional


def _int_case(x: int, y: int) -> dict:
    return {"inputs": {"x": {"type": "int", "value": x}}, "expected": {"type": "int", "value": y}}


def _binary(name: str) -> dict:
    return {"signature": f"{name}(Int,Int)->Int", "args": [{"ref": "Expr"}, {"ref": "Expr"}]}


@dataclass
class TaskFiles:
    """An in-memory task: grammar, cases and search documents."""

    name: str
    grammar: dict
    train: List[dict]
    test: List[dict] = field(default_factory=list)
    fitness: dict = field(default_factory=lambda: {"metric": "absolute", "case_cap": 1000})
    search: dict = field(default_factory=dict)

    def write(self, directory: str) -> str:
        """Write the task file set into ``directory``; return the task path."""
        os.makedirs(directory, exist_ok=True)
        with open(os.path.join(directory, "grammar.json"), "w") as f:
            json.dump(self.grammar, f, indent=1)
        with open(os.path.join(directory, "train.cases.json"), "w") as f:
            json.dump({"format_version": "fitness-cases", "cases": self.train}, f)
        task = {"format": "gagp-task-v1", "name": self.name, "grammar": "grammar.json",
                "train": "train.cases.json", "fitness": self.fitness}
        if self.test:
            with open(os.path.join(directory, "test.cases.json"), "w") as f:
                json.dump({"format_version": "fitness-cases", "cases": self.test}, f)
            task["test"] = "test.cases.json"
        with open(os.path.join(directory, "task.json"), "w") as f:
            json.dump(task, f, indent=1)
        if self.search:
            with open(os.path.join(directory, "search.json"), "w") as f:
                json.dump(self.search, f, indent=1)
        return os.path.join(directory, "task.json")


def search_config(population: int, generations: int, seed: int, **extra) -> dict:
    """A ``gagp-search-config-v1`` document; absent members keep gagp's defaults."""
    doc = {"format": "gagp-search-config-v1", "population_size": population,
           "generations": generations, "seed": str(seed)}
    doc.update(extra)
    return doc


def polynomial_grammar(constants=("0", "1", "2"), max_nodes: int = 31, max_depth: int = 8,
                       fuel: int = 1000) -> dict:
    return {
        "format_version": "grammar-definition-v2",
        "entry": {"nonterminal": "Expr", "type": "Int"},
        "inputs": [{"name": "x", "type": "Int"}],
        "search_limits": {"max_nodes": max_nodes, "max_depth": max_depth},
        "execution_limits": {"fuel": fuel},
        "nonterminals": [{"id": "Expr", "type": "Int", "scope": [], "alternatives": [
            {"id": "x", "weight": 3, "expression": {"input": "x"}},
            {"id": "small", "weight": 2,
             "expression": {"constant": {"type": "Int", "values": list(constants)}}},
            {"id": "add", "weight": 1, "expression": _binary("add")},
            {"id": "sub", "weight": 1, "expression": _binary("sub")},
            {"id": "mul", "weight": 1, "expression": _binary("mul")},
        ]}],
    }


def polynomial(population: int = 1024, generations: int = 64, seed: int = 0) -> TaskFiles:
    """Scalar regression of y = x^3 - 2x + 1 (21 train cases, 40 test cases)."""
    f = lambda x: x ** 3 - 2 * x + 1
    rng = random.Random(seed)
    test_x = [rng.randint(-50, 50) for _ in range(40)]
    return TaskFiles(
        name="polynomial", grammar=polynomial_grammar(),
        train=[_int_case(x, f(x)) for x in range(-10, 11)],
        test=[_int_case(x, f(x)) for x in test_x],
        search=search_config(population, generations, seed))


def poly4_grammar(max_nodes: int = 64, max_depth: int = 16, fuel: int = 1000) -> dict:
    ref = {"ref": "Expr"}
    return {
        "format_version": "grammar-definition-v2",
        "entry": {"nonterminal": "Expr", "type": "Int"},
        "inputs": [{"name": "x", "type": "Int"}],
        "search_limits": {"max_nodes": max_nodes, "max_depth": max_depth},
        "execution_limits": {"fuel": fuel},
        "nonterminals": [{"id": "Expr", "type": "Int", "scope": [], "alternatives": [
            {"id": "x", "weight": 3, "expression": {"input": "x"}},
            {"id": "c", "weight": 2, "expression": {"constant": {"type": "Int", "range": ["-2", "3"]}}},
            {"id": "add", "weight": 1, "expression": _binary("add")},
            {"id": "sub", "weight": 1, "expression": _binary("sub")},
            {"id": "mul", "weight": 1, "expression": _binary("mul")},
            {"id": "idiv0", "weight": 1, "expression": _binary("idiv0")},
            {"id": "imod0", "weight": 1, "expression": _binary("imod0")},
            {"id": "iflt", "weight": 1, "expression": {
                "signature": "if(Bool,Int,Int)->Int",
                "args": [{"signature": "lt(Int,Int)->Bool", "args": [ref, ref]}, ref, ref]}},
        ]}],
    }


def poly4(population: int = 16384, generations: int = 128, seed: int = 0, cases: int = 256,
          max_nodes: int = 64) -> TaskFiles:
    """Random degree<=4 integer polynomial regression over ``cases`` train cases."""
    rng = random.Random(seed)
    coefficients = [rng.randint(-5, 5) for _ in range(5)]
    xs = [rng.randint(-100, 100) for _ in range(cases)]
    f = lambda x: sum(c * x ** k for k, c in enumerate(coefficients))
    return TaskFiles(
        name=f"poly4-s{seed}", grammar=poly4_grammar(max_nodes=max_nodes),
        train=[_int_case(x, f(x)) for x in xs],
        search=search_config(population, generations, seed))


LIST_TARGETS = ("threshold_sum", "threshold_count", "max")


def list_threshold_grammar(max_nodes: int = 48, max_depth: int = 12, fuel: int = 4096) -> dict:
    """The list grammar: a fold of xs whose step sees the element, its index
    and the accumulator, plus the threshold input t."""
    step = {"ref": "Step"}
    cmp = lambda op: {"signature": "if(Bool,Int,Int)->Int",  # noqa: E731
                      "args": [{"signature": f"{op}(Int,Int)->Bool", "args": [step, step]}, step, step]}
    return {
        "format_version": "grammar-definition-v2",
        "entry": {"nonterminal": "Top", "type": "Int"},
        "inputs": [{"name": "xs", "type": "IntList"}, {"name": "t", "type": "Int"}],
        "search_limits": {"max_nodes": max_nodes, "max_depth": max_depth},
        "execution_limits": {"fuel": fuel},
        "nonterminals": [
            {"id": "Top", "type": "Int", "scope": [], "alternatives": [
                {"id": "fold", "weight": 3, "expression": {
                    "signature": "traverse(IntList,Int,Int,Int)->Int",
                    "args": [{"input": "xs"}, {"constant": {"type": "Int", "values": ["0"]}}, {"ref": "Leaf"}, step],
                    "bind": {"3": ["element", "index", "acc"]}}}]},
            {"id": "Leaf", "type": "Int", "scope": [], "alternatives": [
                {"id": "t", "weight": 1, "expression": {"input": "t"}},
                {"id": "k", "weight": 2, "expression": {"constant": {"type": "Int", "range": ["-1", "1"]}}},
                {"id": "len", "weight": 1, "expression": {"signature": "len(IntList)->Int",
                                                          "args": [{"input": "xs"}]}}]},
            {"id": "Step", "type": "Int",
             "scope": [{"name": "element", "type": "Int"}, {"name": "index", "type": "Int"},
                       {"name": "acc", "type": "Int"}],
             "alternatives": [
                 {"id": "element", "weight": 2, "expression": {"bound": "element"}},
                 {"id": "acc", "weight": 2, "expression": {"bound": "acc"}},
                 {"id": "t", "weight": 1, "expression": {"input": "t"}},
                 {"id": "one", "weight": 1, "expression": {"constant": {"type": "Int", "values": ["1"]}}},
                 {"id": "add", "weight": 2, "expression": {"signature": "add(Int,Int)->Int", "args": [step, step]}},
                 {"id": "sub", "weight": 1, "expression": {"signature": "sub(Int,Int)->Int", "args": [step, step]}},
                 {"id": "if_gt", "weight": 1, "expression": cmp("gt")},
                 {"id": "if_lt", "weight": 1, "expression": cmp("lt")}]},
        ],
    }


def list_target(name: str, xs: List[int], t: int) -> int:
    if name == "threshold_sum":
        return sum(e for e in xs if e > t)
    if name == "threshold_count":
        return sum(1 for e in xs if e > t)
    return max(xs) if xs else 0


def list_threshold(population: int = 8192, generations: int = 96, seed: int = 0, cases: int = 200,
                   target: str = "threshold_sum", max_nodes: int = 48) -> TaskFiles:
    rng = random.Random(seed)
    train = []
    for _ in range(cases):
        xs = [rng.randint(-1000, 1000) for _ in range(rng.randint(0, 50))]
        t = rng.randint(-100, 100)
        train.append({"inputs": {"xs": {"type": "int_list", "value": xs}, "t": {"type": "int", "value": t}},
                      "expected": {"type": "int", "value": list_target(target, xs, t)}})
    return TaskFiles(name=f"list-{target}-s{seed}", grammar=list_threshold_grammar(max_nodes=max_nodes),
                     train=train, search=search_config(population, generations, seed))


def list_statements_grammar(max_nodes: int = 64, max_depth: int = 12, fuel: int = 4096) -> dict:
    """A statement grammar over the list cases: the program assigns the
    local acc, then runs statements (assignments to acc, k or the input t,
    for_range loops counting i, if_stmt branches, returns) and ends with a
    return; expressions read t, small constants, the locals, len(xs) and
    index(xs, e)."""
    def control(key, args, **extra):
        return dict({"control": key, "type": "Int", "args": args}, **extra)

    ref = lambda n: {"ref": n}  # noqa: E731
    binary = lambda op, a, b: {"signature": f"{op}(Int,Int)->Int", "args": [ref(a), ref(b)]}  # noqa: E731
    compare = lambda op: {"signature": f"{op}(Int,Int)->Bool", "args": [ref("Value"), ref("Value")]}  # noqa: E731
    return {
        "format_version": "grammar-definition-v2",
        "entry": {"category": "Program", "nonterminal": "Main", "type": "Int"},
        "inputs": [{"name": "xs", "type": "IntList"}, {"name": "t", "type": "Int"}],
        "locals": [{"name": "acc", "type": "Int"}, {"name": "i", "type": "Int"}, {"name": "k", "type": "Int"}],
        "search_limits": {"max_nodes": max_nodes, "max_depth": max_depth},
        "execution_limits": {"fuel": fuel},
        "nonterminals": [
            {"id": "Main", "category": "Program", "type": "Int", "scope": [], "variation": False, "alternatives": [
                {"id": "main", "weight": 1, "expression": control("program(Block)->Program", [
                    control("block_cons(Statement,Block)->Block", [
                        control("assign(Int)->Statement", [ref("Value")], name="acc"), ref("Rest")])])}]},
            {"id": "Rest", "category": "Block", "type": "Int", "scope": [], "alternatives": [
                {"id": "more", "weight": 3, "expression": control("block_cons(Statement,Block)->Block",
                                                                  [ref("Stmt"), ref("Rest")])},
                {"id": "last", "weight": 1, "expression": control("block_cons(Statement,Block)->Block", [
                    control("return(Int)->Statement", [ref("Value")]),
                    control("block_nil()->Block", [])])}]},
            {"id": "Body", "category": "Block", "type": "Int", "scope": [], "alternatives": [
                {"id": "empty", "weight": 2, "expression": control("block_nil()->Block", [])},
                {"id": "cons", "weight": 2, "expression": control("block_cons(Statement,Block)->Block",
                                                                  [ref("Stmt"), ref("Body")])}]},
            {"id": "Stmt", "category": "Statement", "type": "Int", "scope": [], "alternatives": [
                {"id": "acc", "weight": 3, "expression": control("assign(Int)->Statement", [ref("Value")],
                                                                 name="acc")},
                {"id": "k", "weight": 1, "expression": control("assign(Int)->Statement", [ref("Value")], name="k")},
                {"id": "t", "weight": 1, "expression": control("assign(Int)->Statement", [ref("Value")],
                                                               input_name="t")},
                {"id": "loop", "weight": 2, "expression": control("for_range(Int,Block)->Statement",
                                                                  [ref("Bound"), ref("Body")], name="i")},
                {"id": "when", "weight": 2, "expression": control("if_stmt(Bool,Block,Block)->Statement",
                                                                  [ref("Test"), ref("Body"), ref("Body")])},
                {"id": "ret", "weight": 1, "expression": control("return(Int)->Statement", [ref("Value")])}]},
            {"id": "Bound", "type": "Int", "scope": [], "alternatives": [
                {"id": "len", "weight": 3, "expression": {"signature": "len(IntList)->Int", "args": [{"input": "xs"}]}},
                {"id": "small", "weight": 1, "expression": {"constant": {"type": "Int", "range": ["0", "3"]}}}]},
            {"id": "Value", "type": "Int", "scope": [], "alternatives": [
                {"id": "t", "weight": 2, "expression": {"input": "t"}},
                {"id": "c", "weight": 2, "expression": {"constant": {"type": "Int", "range": ["-1", "2"]}}},
                {"id": "acc", "weight": 3, "expression": {"local": "acc"}},
                {"id": "i", "weight": 1, "expression": {"local": "i"}},
                {"id": "k", "weight": 1, "expression": {"local": "k"}},
                {"id": "at", "weight": 3, "expression": {"signature": "index(IntList,Int)->Int",
                                                         "args": [{"input": "xs"}, ref("Value")]}},
                {"id": "add", "weight": 2, "expression": binary("add", "Value", "Value")},
                {"id": "sub", "weight": 1, "expression": binary("sub", "Value", "Value")}]},
            {"id": "Test", "type": "Bool", "scope": [], "alternatives": [
                {"id": "gt", "weight": 2, "expression": compare("gt")},
                {"id": "lt", "weight": 1, "expression": compare("lt")},
                {"id": "eq", "weight": 1, "expression": compare("eq")}]},
        ],
    }


def list_statements(population: int = 8192, generations: int = 96, seed: int = 0, cases: int = 200,
                    target: str = "threshold_sum", max_nodes: int = 64) -> "TaskFiles":
    """The list cases of ``list_threshold`` searched with ``list_statements_grammar``."""
    task = list_threshold(population=population, generations=generations, seed=seed, cases=cases, target=target)
    task.name = f"list-statements-{target}-s{seed}"
    task.grammar = list_statements_grammar(max_nodes=max_nodes)
    return task


def _transition(kind: str, source: int, offset: int = 0) -> dict:
    return {"kind": kind, "source_state": source, "offset": str(offset),
            "window": {"begin": {"kind": "begin", "cut": 0}, "end": {"kind": "begin", "cut": 0}}, "expression": 0}


def grid_paths_grammar(max_nodes: int = 48, max_depth: int = 12, fuel: int = 20000, frames: int = 16,
                       cells: int = 64, ambiguous: bool = False) -> dict:
    """A grammar with a bounded region: a memoized coordinate recurrence
    over (r, c) in [0, rows) x [0, columns) whose requests step to (r - 1, c)
    and (r, c - 1), and whose four phases are evolved: the base predicate
    (reads r and c), the base body (reads the captured input `columns`),
    the combine (reads both request results) and the boundary value.
    `ambiguous` adds a combine alternative add(Join, Join), which derives
    add(up, left) a second way: the reference re-derives its generated
    initial programs from their syntax trees, taking the first production
    that matches."""
    ref = lambda n: {"ref": n}  # noqa: E731
    plan = {
        "version": 1, "state_types": ["Int", "Int"], "result_type": "Int", "parameter_types": ["Int"],
        "preparations": [], "request_expression_types": [], "bound_operand_count": 2,
        "requests": [{"states": [_transition("coordinate_offset", 0, -1), _transition("coordinate_offset", 1, 0)]},
                     {"states": [_transition("coordinate_offset", 0, 0), _transition("coordinate_offset", 1, -1)]}],
        "limits": {"frames": frames, "cells": cells, "entry_fuel": 1}, "memoized": True,
        "duplicate_policy": "reject", "progress": "coordinates", "coordinate_slots": [0, 1],
        "coordinate_rank": [{"coordinate": 0, "direction": 1}, {"coordinate": 1, "direction": 1}],
        "coordinate_domains": [
            {"lower": {"kind": "literal", "literal": "0", "operand": 0},
             "upper": {"kind": "operand", "literal": "0", "operand": 2}},
            {"lower": {"kind": "literal", "literal": "0", "operand": 0},
             "upper": {"kind": "operand", "literal": "0", "operand": 3}}],
        "coordinate_endpoint": "exclusive", "sequence_state": 0}
    region = {"structured": {"family": "bounded", "plan": plan}, "captures": [{"input": "columns"}],
              "phases": [{"argument": 4, "bindings": [{"bank": "state", "slot": 0, "name": "r"},
                                                      {"bank": "state", "slot": 1, "name": "c"}]},
                         {"argument": 5, "bindings": [{"bank": "parameter", "slot": 0, "name": "p"}]},
                         {"argument": 6, "bindings": [{"bank": "result", "slot": 0, "name": "up"},
                                                      {"bank": "result", "slot": 1, "name": "left"}]},
                         {"argument": 7, "bindings": []}],
              "args": [ref("Coord"), ref("Coord"), {"input": "rows"}, {"input": "columns"}, ref("Test"),
                       ref("Base"), ref("Join"), ref("Edge")]}
    small = lambda *v: {"constant": {"type": "Int", "values": [str(x) for x in v]}}  # noqa: E731
    return {
        "format_version": "grammar-definition-v2",
        "entry": {"nonterminal": "Top", "type": "Int"},
        "inputs": [{"name": "row", "type": "Int"}, {"name": "column", "type": "Int"},
                   {"name": "rows", "type": "Int"}, {"name": "columns", "type": "Int"}],
        "search_limits": {"max_nodes": max_nodes, "max_depth": max_depth},
        "execution_limits": {"fuel": fuel},
        "nonterminals": [
            {"id": "Top", "type": "Int", "scope": [], "alternatives": [
                {"id": "paths", "weight": 3, "expression": region},
                {"id": "shift", "weight": 1, "expression": {"signature": "add(Int,Int)->Int",
                                                            "args": [ref("Top"), ref("Coord")]}},
                {"id": "one", "weight": 1, "expression": small(1)}]},
            {"id": "Coord", "type": "Int", "scope": [], "alternatives": [
                {"id": "row", "weight": 2, "expression": {"input": "row"}},
                {"id": "column", "weight": 2, "expression": {"input": "column"}},
                {"id": "k", "weight": 1, "expression": small(0, 1)},
                {"id": "add", "weight": 1, "expression": {"signature": "add(Int,Int)->Int",
                                                          "args": [ref("Coord"), ref("Coord")]}}]},
            {"id": "Test", "type": "Bool", "scope": [{"name": "r", "type": "Int"}, {"name": "c", "type": "Int"}],
             "alternatives": [
                 {"id": "r0", "weight": 2, "expression": {"signature": "eq(Int,Int)->Bool",
                                                          "args": [{"bound": "r"}, small(0, 1)]}},
                 {"id": "c0", "weight": 2, "expression": {"signature": "eq(Int,Int)->Bool",
                                                          "args": [{"bound": "c"}, small(0, 1)]}},
                 {"id": "lt", "weight": 1, "expression": {"signature": "lt(Int,Int)->Bool",
                                                          "args": [{"bound": "r"}, {"bound": "c"}]}},
                 {"id": "or", "weight": 1, "expression": {"signature": "or(Bool,Bool)->Bool",
                                                          "args": [ref("Test"), ref("Test")]}}]},
            {"id": "Base", "type": "Int", "scope": [{"name": "p", "type": "Int"}], "alternatives": [
                {"id": "one", "weight": 2, "expression": small(1, 2)},
                {"id": "p", "weight": 1, "expression": {"bound": "p"}},
                {"id": "sub", "weight": 1, "expression": {"signature": "sub(Int,Int)->Int",
                                                          "args": [ref("Base"), ref("Base")]}}]},
            {"id": "Join", "type": "Int", "scope": [{"name": "up", "type": "Int"}, {"name": "left", "type": "Int"}],
             "alternatives": [
                 {"id": "add", "weight": 2, "expression": {"signature": "add(Int,Int)->Int",
                                                           "args": [{"bound": "up"}, {"bound": "left"}]}},
                 {"id": "up", "weight": 1, "expression": {"bound": "up"}},
                 {"id": "left", "weight": 1, "expression": {"bound": "left"}},
                 {"id": "max", "weight": 1, "expression": {"signature": "max(Int,Int)->Int",
                                                           "args": [ref("Join"), ref("Join")]}},
                 {"id": "sub", "weight": 1, "expression": {"signature": "sub(Int,Int)->Int",
                                                           "args": [ref("Join"), ref("Join")]}}] +
             ([{"id": "sum", "weight": 1, "expression": {"signature": "add(Int,Int)->Int",
                                                         "args": [ref("Join"), ref("Join")]}}] if ambiguous else [])},
            {"id": "Edge", "type": "Int", "scope": [], "alternatives": [
                {"id": "k", "weight": 1, "expression": small(0, 1)}]},
        ],
    }


def grid_paths(population: int = 1024, generations: int = 32, seed: int = 0, cases: int = 40,
               size: int = 7, ambiguous: bool = False) -> "TaskFiles":
    """Lattice paths: C(row + column, row) for row, column in [0, size) on a
    size x size grid, searched with ``grid_paths_grammar``."""
    rng = random.Random(seed)
    train = []
    for _ in range(cases):
        r, c = rng.randrange(size), rng.randrange(size)
        train.append({"inputs": {"row": {"type": "int", "value": r}, "column": {"type": "int", "value": c},
                                 "rows": {"type": "int", "value": size}, "columns": {"type": "int", "value": size}},
                      "expected": {"type": "int", "value": math.comb(r + c, r)}})
    return TaskFiles(name=f"grid-paths-s{seed}", grammar=grid_paths_grammar(ambiguous=ambiguous), train=train,
                     search=search_config(population, generations, seed))


def _log_uniform_population(rng: random.Random, lo: int, hi: int) -> int:
    # floor(lo * (hi / lo) ** u), u ~ U[0, 1)
    return int(lo * (hi / lo) ** rng.random())


def mix_files(entry: dict) -> TaskFiles:
    """The task files of a mix entry: built with the mix for the scalar
    entries, on demand for the list entries (their cases, lists of up to 50
    elements, are the costly part to build)."""
    if entry["files"] is None:
        entry["files"] = make(entry["workload"], **entry["args"])
    return entry["files"]


def batch_mix(count: int = 64, generations: int = 64, max_population: int = 8192) -> List[dict]:
    """The batching workload: `count` independent searches with seeds 0..count-1,
    populations log-uniform in 256..max_population, case counts uniform in
    16..1000.  Even indices are scalar regressions of a random integer
    polynomial (the large scalar grammar); odd indices are list programs
    (``list_threshold``, the target cycling through threshold sum, threshold
    count and maximum), whose files ``mix_files`` builds on demand."""
    out = []
    for i in range(count):
        rng = random.Random(1000003 * i + 17)
        population = _log_uniform_population(rng, 256, max_population)
        cases = rng.randint(16, 1000)
        args = dict(population=population, generations=generations, seed=i, cases=cases)
        entry = {"index": i, "seed": i, "population": population, "cases": cases, "generations": generations,
                 "kind": "scalar" if i % 2 == 0 else "list", "files": None}
        if i % 2 == 0:
            entry.update(workload="poly4", args=args)
            entry["files"] = poly4(**args)
        else:
            entry.update(workload="list_threshold", args=dict(args, target=LIST_TARGETS[(i // 2) % 3]))
        out.append(entry)
    return out


def serving_mix(count: int = 2000, seed: int = 0) -> List[dict]:
    """The serving workload: `count` requests, populations log-uniform in
    256..16384, case counts uniform in 16..2000, generations uniform in
    32..128, half scalar regressions of a random integer polynomial and half
    list programs (``list_threshold``, files built on demand by
    ``mix_files``)."""
    rng = random.Random(seed)
    out = []
    for i in range(count):
        population = _log_uniform_population(rng, 256, 16384)
        cases = rng.randint(16, 2000)
        generations = rng.randint(32, 128)
        scalar = rng.random() < 0.5
        args = dict(population=population, generations=generations, seed=seed * 100003 + i, cases=cases)
        entry = {"index": i, "seed": args["seed"], "population": population, "cases": cases,
                 "generations": generations, "kind": "scalar" if scalar else "list", "files": None}
        if scalar:
            entry.update(workload="poly4", args=args)
            entry["files"] = poly4(**args)
        else:
            entry.update(workload="list_threshold", args=dict(args, target=LIST_TARGETS[i % 3]))
        out.append(entry)
    return out


WORKLOADS: Dict[str, object] = {"polynomial": polynomial, "poly4": poly4, "list_threshold": list_threshold,
                                "list_statements": list_statements, "grid_paths": grid_paths}


def make(name: str, **kwargs) -> TaskFiles:
    return WORKLOADS[name](**kwargs)
