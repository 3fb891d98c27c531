"""``gagp-task-v1`` / ``gagp-search-config-v1`` loading.

Mirrors what ``gagp run`` assembles before a search
(``cpp/src/cli/run.cpp:275-300``): the built-in default search
(``run.cpp:36-49``, ``configs/search/default.json``) overlaid with the search
file, penalty = the task's ``case_cap``, fuel = the grammar's execution fuel
(a search file may only lower it), reduction lanes = 512 (``run.cpp:63``).
Inputs are ordered by name, as ``prepare_case_set`` orders them
(``cpp/src/evolution/case_set.cpp:48-55``).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import grammar as G
from .abi import CasesBlob, SearchSettings

DEFAULT_SEARCH = {
    "format": "gagp-search-config-v1", "representation": "resident", "population_size": 1024,
    "generations": 64, "selection": {"method": "tournament", "size": 2}, "elitism": 1,
    "crossover": {"probability": 0.7, "attempts": 8}, "mutation": {"probability": 0.3},
    "sites": {"scope": "uniform_phase", "draw": "counted"}, "limits": {"site_depth": 7},
    "ranking": {"tie_break": "ast_nodes"}, "schedule": {"mode": "steady_state", "replacement_size": 2},
}

_TYPE_TAGS = {"int": G.TAG_INT, "bool": G.TAG_BOOL, "int_list": G.TAG_INTLIST}


@dataclass
class LoadedTask:
    name: str
    tables: G.PhaseTables
    cases: CasesBlob
    settings: SearchSettings
    test_cases: Optional[CasesBlob] = None


def _case_values(doc: dict, names):
    """Inputs in evaluator order, their tags, expected values and tag, and the
    IntList arena: an int_list input becomes the offset of its length word in
    the arena, its elements following."""
    rows, expected, tags, etag = [], [], None, None
    lists: list = []
    for case in doc["cases"]:
        row, row_tags = [], []
        for n in names:
            v = case["inputs"][n]
            if v["type"] not in _TYPE_TAGS:
                raise G.Declined(f"input type {v['type']} is outside the resident subset")
            row_tags.append(_TYPE_TAGS[v["type"]])
            if v["type"] == "int_list":
                row.append(len(lists))
                lists.append(len(v["value"]))
                lists.extend(int(x) for x in v["value"])
            else:
                row.append(int(v["value"]))
        if tags is None:
            tags = row_tags
        elif tags != row_tags:
            raise G.Declined("mixed input types")
        e = case["expected"]
        if e["type"] not in ("int", "bool"):
            raise G.Declined(f"expected type {e['type']} is outside the resident subset")
        if etag is None:
            etag = _TYPE_TAGS[e["type"]]
        rows.append(row)
        expected.append(int(e["value"]))
    return np.array(rows, dtype=np.int64).reshape(len(expected), len(names)), tags or [], \
        np.array(expected, dtype=np.int64), etag or 0, (np.array(lists, dtype=np.int64) if lists else None)


def apply_search(settings: SearchSettings, doc: dict) -> None:
    """Overlay a ``gagp-search-config-v1`` document (spec/search_config.md)."""
    if doc.get("format") != "gagp-search-config-v1":
        raise ValueError("gagp-search-config-v1 required")
    if doc.get("representation", "resident") != "resident":
        raise G.Declined("native_ast representation is not the resident engine")
    s = settings
    if "population_size" in doc:
        s.population = int(doc["population_size"])
    if "generations" in doc:
        s.generations = int(doc["generations"])
    if "seed" in doc:
        s.seed = int(doc["seed"])
    if "selection" in doc:
        s.tournament_size = int(doc["selection"].get("size", s.tournament_size))
    if "elitism" in doc:
        s.elite_count = int(doc["elitism"])
    explicit = any(k in doc for k in ("crossover", "sites")) or "max_subtree_nodes" in doc.get("mutation", {})
    if explicit:
        s.crossover_probability, s.crossover_attempts, s.mutation_max_nodes = 1.0, 8, 0
        s.uniform_phase, s.counted_sites = False, False
    if "crossover" in doc:
        s.crossover_probability = float(doc["crossover"].get("probability", s.crossover_probability))
        s.crossover_attempts = int(doc["crossover"].get("attempts", s.crossover_attempts))
    if "mutation" in doc:
        s.mutation_probability = float(doc["mutation"].get("probability", s.mutation_probability))
        s.mutation_max_nodes = int(doc["mutation"].get("max_subtree_nodes", s.mutation_max_nodes))
    if "sites" in doc:
        s.uniform_phase = doc["sites"].get("scope", "genome") == "uniform_phase"
        s.counted_sites = doc["sites"].get("draw", "reservoir") == "counted"
    if "limits" in doc:
        s.site_depth = int(doc["limits"].get("site_depth", s.site_depth))
    if "ranking" in doc:
        s.grammar_site_ranking = doc["ranking"].get("tie_break", "ast_nodes") == "grammar_sites"
    if "fitness" in doc and "penalty" in doc["fitness"]:
        s.penalty = float(doc["fitness"]["penalty"])
    if "execution" in doc and "fuel" in doc["execution"]:
        s.fuel = min(s.fuel, int(doc["execution"]["fuel"]))
    if "schedule" in doc:
        sc = doc["schedule"]
        s.steady_state = sc.get("mode", "generational") == "steady_state"
        s.batch = int(sc.get("batch", 0))
        s.replacement_size = int(sc.get("replacement_size", 2))


def load(task_path: str, search_path: Optional[str] = None, population: Optional[int] = None,
         generations: Optional[int] = None, seed: Optional[int] = None) -> LoadedTask:
    base = os.path.dirname(os.path.abspath(task_path))
    with open(task_path) as f:
        task = json.load(f)
    if task.get("format") != "gagp-task-v1":
        raise ValueError("gagp-task-v1 required")
    grammar_doc = G.load_definition(os.path.join(base, task["grammar"]))
    with open(os.path.join(base, task["train"])) as f:
        train = json.load(f)
    search = None
    if search_path:
        with open(search_path) as f:
            search = json.load(f)
    test = None
    if task.get("test"):
        with open(os.path.join(base, task["test"])) as f:
            test = json.load(f)
    return assemble(task.get("name", os.path.basename(base)), grammar_doc, train, task["fitness"], search, test,
                    population, generations, seed)


def assemble(name: str, grammar_doc: dict, train: dict, fitness: dict, search: Optional[dict] = None,
             test: Optional[dict] = None, population: Optional[int] = None, generations: Optional[int] = None,
             seed: Optional[int] = None, table_cache: Optional[dict] = None) -> LoadedTask:
    """A loaded task from in-memory task documents (what load() reads from
    files).  `table_cache` shares compiled phase tables between tasks with
    the same grammar, inputs and site depth."""
    names = sorted({n for case in train["cases"] for n in case["inputs"]})
    settings = SearchSettings()
    settings.metric = fitness["metric"]
    settings.penalty = float(fitness.get("case_cap", 1000))
    settings.fuel = int(grammar_doc["execution_limits"]["fuel"])
    apply_search(settings, DEFAULT_SEARCH)
    if search:
        apply_search(settings, search)
    if population:
        settings.population = population
    if generations:
        settings.generations = generations
    if seed is not None:
        settings.seed = seed
    if settings.metric not in ("absolute", "exact"):
        raise G.Declined(f"metric {settings.metric} is outside the resident scalar subset")
    if settings.site_depth < 1:
        raise G.Declined("the resident engine here generates its population under a site-depth limit")
    key = (json.dumps(grammar_doc, sort_keys=True), tuple(names), settings.site_depth)
    tables = table_cache.get(key) if table_cache is not None else None
    if tables is None:
        tables = G.compile_tables(grammar_doc, names, settings.site_depth, allow_lists=True)
        if table_cache is not None:
            table_cache[key] = tables
    inputs, tags, expected, etag, lists = _case_values(train, names)
    test_blob = None
    if test:
        ti, tt, te, tet, tl = _case_values(test, names)
        test_blob = CasesBlob(ti, tt, te, tet, tl)
    return LoadedTask(name, tables, CasesBlob(inputs, tags, expected, etag, lists), settings, test_blob)


def from_files(files, table_cache: Optional[dict] = None) -> LoadedTask:
    """A loaded task straight from an in-memory ``workloads.TaskFiles``."""
    train = {"format_version": "fitness-cases", "cases": files.train}
    test = {"format_version": "fitness-cases", "cases": files.test} if files.test else None
    return assemble(files.name, files.grammar, train, files.fitness, files.search or None, test,
                    table_cache=table_cache)


def program_text(tables: G.PhaseTables, origins, constants, first_binder: int = 0) -> str:
    """Prefix program text of a phase row (``cli_detail::program_text``,
    ``cpp/src/cli/program_json.cpp:876-946``).  A traversal (or a let) shows
    its body's bound variables before the body, ``[vA vB vC] body``, numbered in prefix
    order from ``first_binder`` as the reference's export numbers them
    (``export_native_phase_layout``, phase_layout.hpp:388-396); a bound read
    prints its variable."""
    out = []
    pos = [0]
    k = [0]
    env = {}
    next_id = [first_binder]

    def node():
        e = tables.expressions[origins[pos[0]]]
        pos[0] += 1
        # statements (ProgramPrinter::node): a program prints its block, a
        # block chain prints as one (block s1 s2 ...), a named control shows
        # its target and a local read its name
        if e.node_kind == G.TK_PROGRAM and e.kind == G.EK_OPERATION:
            node()
            return
        if e.node_kind == G.TK_NIL and e.kind == G.EK_OPERATION:
            out.append("(block)")
            return
        if e.node_kind == G.TK_BLOCK and e.kind == G.EK_OPERATION:
            out.append("(block")
            while True:
                out.append(" ")
                node()
                tail = tables.expressions[origins[pos[0]]]
                pos[0] += 1
                if tail.node_kind != G.TK_BLOCK:
                    break
            out.append(")")
            return
        if e.node_kind == G.TK_VAR and e.kind == G.EK_OPERATION:
            out.append(e.label)
            return
        if e.kind == G.EK_CONSTANT:
            out.append(str(constants[k[0]]))
            k[0] += 1
            return
        if e.kind == G.EK_INPUT:
            out.append(e.name)
            return
        if e.kind == G.EK_BOUND:
            out.append("v%d" % env[e.operand])
            return
        ids, binders = None, None
        if e.node_kind == G.TK_REGION and e.kind == G.EK_OPERATION:
            # a bounded region: operands, then each phase, whose bindings
            # (binders 0.. of the phase) read as fresh variables
            plan = tables.regions[e.operand].plan
            operands = len(plan.state_types) + plan.bound_count
            out.append("(" + e.name)
            for i in range(e.arity):
                out.append(" ")
                if i < operands:
                    node()
                    continue
                bound = len(plan.phase_bindings[i - operands])
                ids = [next_id[0] + j for j in range(bound)]
                next_id[0] += bound
                saved = dict(env)
                env.clear()
                env.update(zip(range(bound), ids))
                node()
                env.clear()
                env.update(saved)
            out.append(")")
            return
        if e.node_kind == G.TK_TRAVERSE:
            binders = tables.regions[e.operand].binders
            ids = [next_id[0] + j for j in range(3)]
            next_id[0] += 3
        elif e.node_kind == G.TK_LET:
            # a let binds one variable for its body (the last argument)
            binders = [e.operand]
            ids = [next_id[0]]
            next_id[0] += 1
        out.append("(" + e.name)
        if e.node_kind in (G.TK_ASSIGN, G.TK_FOR_RANGE) and e.kind == G.EK_OPERATION:
            out.append(" " + e.label)
        for i in range(e.arity):
            out.append(" ")
            if ids is not None and i == e.arity - 1:
                out.append("[" + " ".join("v%d" % x for x in ids) + "] ")
                saved = {b: env.get(b) for b in binders}
                env.update(zip(binders, ids))
                node()
                env.update(saved)
            else:
                node()
        out.append(")")

    n = len(origins)
    kinds = [tables.expressions[o].node_kind if tables.expressions[o].kind == G.EK_OPERATION else -1
             for o in origins]
    if n >= 4 and kinds[0] == G.TK_PROGRAM and kinds[1] == G.TK_BLOCK and kinds[2] == G.TK_RETURN \
            and kinds[-1] == G.TK_NIL:
        # a program that is a single `return e` reads as just `e`
        pos[0] = 3
        node()
        if pos[0] == n - 1:
            return "".join(out)
        out.clear()
        pos[0], k[0], next_id[0] = 0, 0, first_binder
    node()
    return "".join(out)
