"""Loads the golden fixtures of tests/golden (see make_golden.py)."""
from __future__ import annotations

import glob
import gzip
import json
import os
import re
import tempfile

from gagp_b200 import abi
from gagp_b200 import task as T
from gagp_b200 import workloads as W

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[: -len(".json.gz")] for p in glob.glob(os.path.join(HERE, "*.json.gz")))


def fixture(name: str) -> dict:
    with gzip.open(os.path.join(HERE, name + ".json.gz"), "rt") as f:
        return json.load(f)


# list-program fixtures (golden/list/): the reference's tables, rows and runs
# of list tasks (traversals, lets, statement programs)
LIST_HERE = os.path.join(HERE, "list")


def list_names():
    return sorted(os.path.basename(p)[: -len(".json.gz")] for p in glob.glob(os.path.join(LIST_HERE, "*.json.gz")))


def list_fixture(name: str) -> dict:
    with gzip.open(os.path.join(LIST_HERE, name + ".json.gz"), "rt") as f:
        return json.load(f)


def load_task(fx: dict) -> T.LoadedTask:
    files = W.TaskFiles(name=fx["task"]["name"], grammar=fx["grammar"], train=fx["train"], test=fx["test"],
                        fitness=fx["task"]["fitness"], search=fx["search"])
    with tempfile.TemporaryDirectory() as d:
        files.write(d)
        return T.load(os.path.join(d, "task.json"), os.path.join(d, "search.json"))


def reference_rows(rows, stride: int) -> abi.RowsBuffer:
    return abi.RowsBuffer.from_rows([(r["origins"], [c[1] for c in r["constants"]]) for r in rows], stride)


def binder_names_in_order(text: str) -> str:
    """Program text with its bound variables renamed v0, v1, ... in order of
    first appearance: the reference's export numbers them from the largest
    binder id of its prototype program, which only that numbering depends on."""
    names = {}
    return re.sub(r"\bv\d+\b", lambda m: names.setdefault(m.group(0), "v%d" % len(names)), text)


def first_match_origins(tables, origins, constants):
    """A row's derivation as the reference's import re-derives a program
    (reconstruct_derivation, cpp/src/evolution/grammar/membership.cpp:330-360):
    at each nonterminal the first production, in order, that matches the
    whole subtree."""
    from gagp_b200 import grammar as G
    ex = tables.expressions
    value, k = [], 0
    for e in origins:
        if ex[e].kind == G.EK_CONSTANT:
            value.append(constants[k])
            k += 1
        else:
            value.append(None)
    out = list(origins)

    def match(e, i):
        x = ex[e]
        if x.kind == G.EK_REFERENCE:
            off, count = tables.nonterminals[x.target][0], tables.nonterminals[x.target][1]
            for p in range(off, off + count):
                end = match(tables.productions[p][0], i)
                if end >= 0:
                    return end
            return -1
        if i >= len(origins):
            return -1
        y = ex[origins[i]]
        if x.kind != y.kind:
            return -1
        if x.kind == G.EK_CONSTANT:
            d = tables.domains[x.target]
            if d.integer_range:
                if not d.minimum <= value[i] <= d.maximum:
                    return -1
            elif value[i] not in [tables.values[d.value_offset + j][1] for j in range(d.value_count)]:
                return -1
        elif x.kind == G.EK_OPERATION:
            if (x.node_kind, x.opcode, x.operand, x.arity, x.type) != (y.node_kind, y.opcode, y.operand, y.arity,
                                                                        y.type):
                return -1
        elif x.operand != y.operand:
            return -1
        out[i] = e
        j = i + 1
        for c in range(x.arity if x.kind == G.EK_OPERATION else 0):
            j = match(x.children[c], j)
            if j < 0:
                return -1
        return j

    return out if match(tables.root_expression, 0) == len(origins) else list(origins)


def compare_result(lt: T.LoadedTask, got: dict, run: dict, label: str = "") -> None:
    """Asserts a search result equals the reference run bit for bit: history,
    final ranked population and the evaluation counters (program-case pairs
    evaluated, children that reused a completed result)."""
    ref_hist, ref_final = run["history"], run["final"]
    assert got["program_cases"] == run["program_cases"], (label, "program_cases", got["program_cases"],
                                                          run["program_cases"])
    assert got["reused_programs"] == run["reused_programs"], (label, "reused", got["reused_programs"],
                                                              run["reused_programs"])
    assert len(got["history"]) == len(ref_hist), label
    for i, (a, b) in enumerate(zip(got["history"], ref_hist)):
        text = binder_names_in_order(T.program_text(lt.tables, *a["row"]))
        b = dict(b, text=binder_names_in_order(b["text"]))
        assert a["best_fitness"] == b["best_fitness"], (label, "history", i, a["best_fitness"], b["best_fitness"])
        assert a["mean_fitness"] == float.fromhex(b["mean_fitness"]), (label, "mean", i)
        assert a["best_wrong"] == b["best_wrong"], (label, "wrong", i)
        assert a["best_nodes"] == b["best_nodes"], (label, "nodes", i)
        assert text == b["text"], (label, "champion", i, text, b["text"])
    assert len(got["final"]) == len(ref_final), label
    for i, (a, b) in enumerate(zip(got["final"], ref_final)):
        r = b["rows"][0]
        assert a["fitness"] == b["fitness"], (label, "final fitness", i, a["fitness"], b["fitness"])
        assert a["wrong"] == b["wrong"], (label, "final wrong", i)
        assert a["nodes"] == b["nodes"], (label, "final nodes", i)
        origins = list(a["row"][0])
        if origins != r["origins"]:
            # the reference exports its members as syntax trees, whose rows
            # it re-derives: a program of an ambiguous grammar compares in
            # that first-match derivation
            origins = first_match_origins(lt.tables, origins, list(a["row"][1]))
        assert origins == r["origins"], (label, "final origins", i)
        assert list(a["row"][1]) == [c[1] for c in r["constants"]], (label, "final constants", i)
