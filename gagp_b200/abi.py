"""ctypes mirror of ``include/gagp_b200.h`` and marshalling helpers.

The structures here are the flat data formats of the C ABI: admitted phase
tables (``gagp_grammar``), scalar cases (``gagp_cases``), the resident search
configuration (``gagp_search_config``), transport rows and search results.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .grammar import PhaseTables

MAX_ARITY = 8
MAX_LOCALS = 64

STATUS_NAMES = {0: "OK", 1: "DECLINED", 2: "INVALID_ARGUMENT", 3: "OUT_OF_MEMORY", 4: "DEVICE_ERROR",
                5: "TIMEOUT_CAP", 6: "NOT_READY", 7: "NO_EXTENSION"}

METRICS = {"legacy": 0, "absolute": 1, "exact": 2}


class Expression(C.Structure):
    _fields_ = [("kind", C.c_int32), ("node_kind", C.c_int32), ("opcode", C.c_int32), ("operand", C.c_int32),
                ("arity", C.c_int32), ("fuel", C.c_uint32), ("merge_fuel", C.c_uint32), ("type", C.c_int32),
                ("target", C.c_int32), ("scope_count", C.c_int32), ("children", C.c_int32 * MAX_ARITY),
                ("child_scope", C.c_int8 * MAX_ARITY)]


class Production(C.Structure):
    _fields_ = [("expression", C.c_int32), ("reserved", C.c_int32), ("weight", C.c_double)]


class Nonterminal(C.Structure):
    _fields_ = [("production_offset", C.c_int32), ("production_count", C.c_int32), ("scope_count", C.c_int32),
                ("normalized_weights", C.c_int32), ("fixed", C.c_int32)]


class Domain(C.Structure):
    _fields_ = [("value_offset", C.c_int32), ("value_count", C.c_int32), ("integer_range", C.c_int32),
                ("reserved", C.c_int32), ("minimum", C.c_int64), ("maximum", C.c_int64)]


class Value(C.Structure):
    _fields_ = [("i", C.c_int64), ("tag", C.c_int32), ("reserved", C.c_int32)]


class Region(C.Structure):
    _fields_ = [("traversal", C.c_int32), ("ranged", C.c_int32), ("fuel_profile", C.c_int32),
                ("binders", C.c_int32 * 3), ("operand_types", C.c_int32 * 6), ("binding_types", C.c_int32 * 3),
                ("result_type", C.c_int32), ("event_cost", C.c_uint32 * 26),
                # a bounded region (traversal 0)
                ("operands", C.c_int32), ("phases", C.c_int32), ("captures", C.c_int32),
                ("capture_kind", C.c_int32 * 8), ("capture_target", C.c_int32 * 8), ("phase_type", C.c_int32 * 8),
                ("phase_bindings", C.c_int32 * 8), ("binding_bank", (C.c_int32 * 8) * 8),
                ("binding_slot", (C.c_int32 * 8) * 8), ("phase_binding_types", (C.c_int32 * 8) * 8),
                ("state_count", C.c_int32), ("request_count", C.c_int32), ("axis_count", C.c_int32),
                ("inclusive", C.c_int32), ("memoized", C.c_int32), ("frames", C.c_uint32), ("cells", C.c_uint32),
                ("entry_fuel", C.c_uint32), ("parameter_types", C.c_int32 * 8),
                ("transition_kind", (C.c_int32 * 4) * 8), ("transition_source", (C.c_int32 * 4) * 8),
                ("axis_slot", C.c_int32 * 4), ("lower_kind", C.c_int32 * 4), ("upper_kind", C.c_int32 * 4),
                ("reserved", C.c_int32), ("transition_offset", (C.c_int64 * 4) * 8),
                ("lower", C.c_int64 * 4), ("upper", C.c_int64 * 4)]


class Grammar(C.Structure):
    _fields_ = [("expressions", C.POINTER(Expression)), ("expression_count", C.c_int32),
                ("productions", C.POINTER(Production)), ("production_count", C.c_int32),
                ("nonterminals", C.POINTER(Nonterminal)), ("nonterminal_count", C.c_int32),
                ("domains", C.POINTER(Domain)), ("domain_count", C.c_int32),
                ("values", C.POINTER(Value)), ("value_count", C.c_int32),
                ("minimum", C.POINTER(C.c_uint32)),
                ("depth_count", C.c_int32), ("logical_depth_count", C.c_int32), ("site_depth", C.c_int32),
                ("root_expression", C.c_int32), ("slot_max_depth", C.c_int32), ("slot_type", C.c_int32),
                ("local_count", C.c_int32), ("local_types", C.c_int32 * MAX_LOCALS),
                ("max_nodes", C.c_int32), ("fixed_nodes", C.c_int32), ("return_fuel", C.c_uint32),
                ("regions", C.POINTER(Region)), ("region_count", C.c_int32)]


class Cases(C.Structure):
    _fields_ = [("case_count", C.c_int32), ("input_count", C.c_int32), ("inputs", C.POINTER(C.c_int64)),
                ("input_tags", C.POINTER(C.c_int32)), ("expected", C.POINTER(C.c_int64)),
                ("expected_tag", C.c_int32), ("list_values", C.POINTER(C.c_int64)),
                ("list_value_count", C.c_int64)]


class SearchConfig(C.Structure):
    _fields_ = [("population", C.c_int32), ("generations", C.c_int32), ("seed", C.c_uint64),
                ("tournament_size", C.c_int32), ("crossover_attempts", C.c_int32),
                ("crossover_probability", C.c_double), ("mutation_probability", C.c_double),
                ("mutation_max_nodes", C.c_int32), ("counted_sites", C.c_int32), ("uniform_phase", C.c_int32),
                ("steady_state", C.c_int32), ("batch", C.c_int32), ("replacement_size", C.c_int32),
                ("elite_count", C.c_int32), ("fuel", C.c_int32), ("penalty", C.c_double), ("metric", C.c_int32),
                ("grammar_site_ranking", C.c_int32), ("reduction_lanes", C.c_int32), ("reserved", C.c_int32)]


class Rows(C.Structure):
    _fields_ = [("count", C.c_int32), ("stride", C.c_int32), ("node_counts", C.POINTER(C.c_int32)),
                ("origins", C.POINTER(C.c_int32)), ("constant_counts", C.POINTER(C.c_int32)),
                ("constants", C.POINTER(C.c_int64))]


class Verdict(C.Structure):
    """``gagp_verdict``: one program's judgement on a case set."""
    _fields_ = [("cases", C.c_int32), ("correct", C.c_int32), ("runtime_errors", C.c_int32), ("reserved", C.c_int32),
                ("loss", C.c_double)]

    def summary(self) -> dict:
        """The reference's judge object (cpp/src/cli/run.cpp:232-237)."""
        n = float(self.cases)
        return {"cases": n, "correct": float(self.correct), "wrong": n - self.correct,
                "runtime_errors": float(self.runtime_errors), "mean_loss": self.loss / n,
                "solved": self.correct == self.cases}


class SearchResult(C.Structure):
    _fields_ = [("generations", C.c_int32), ("history_best_fitness", C.POINTER(C.c_double)),
                ("history_mean_fitness", C.POINTER(C.c_double)), ("history_best_wrong", C.POINTER(C.c_int32)),
                ("history_best_nodes", C.POINTER(C.c_int32)), ("history_best", Rows),
                ("population", C.c_int32), ("final_fitness", C.POINTER(C.c_double)),
                ("final_wrong", C.POINTER(C.c_int32)), ("final_nodes", C.POINTER(C.c_int32)),
                ("final_rows", Rows), ("evaluated_programs", C.c_uint64), ("reused_programs", C.c_uint64),
                ("program_cases", C.c_uint64)]


def _ptr(array: np.ndarray, ctype):
    return array.ctypes.data_as(C.POINTER(ctype))


def fill_bounded_region(x: Region, r) -> None:
    """The bounded-region fields of a region table entry from the table
    builder's plan (grammar.BoundedPlan)."""
    p = r.plan
    x.operands = len(p.state_types) + p.bound_count
    x.phases = 4
    x.captures = len(p.captures)
    for c, (kind, target) in enumerate(p.captures):
        x.capture_kind[c], x.capture_target[c] = kind, target
    for ph in range(4):
        x.phase_type[ph] = p.phase_types[ph]
        x.phase_bindings[ph] = len(p.phase_bindings[ph])
        for b, (bank, slot, tag) in enumerate(p.phase_bindings[ph]):
            x.binding_bank[ph][b], x.binding_slot[ph][b], x.phase_binding_types[ph][b] = bank, slot, tag
    x.state_count, x.request_count, x.axis_count = len(p.state_types), len(p.requests), len(p.axes)
    x.inclusive, x.memoized = int(p.inclusive), int(p.memoized)
    x.frames, x.cells, x.entry_fuel = p.frames, p.cells, p.entry_fuel
    for k, tag in enumerate(p.parameter_types):
        x.parameter_types[k] = tag
    for q, row in enumerate(p.requests):
        for st, (kind, source, offset) in enumerate(row):
            x.transition_kind[q][st], x.transition_source[q][st], x.transition_offset[q][st] = kind, source, offset
    for a, (slot, (lk, lv), (uk, uv)) in enumerate(p.axes):
        x.axis_slot[a], x.lower_kind[a], x.lower[a], x.upper_kind[a], x.upper[a] = slot, lk, lv, uk, uv
    for k, tag in enumerate(r.operand_types[:8]):
        if k < 6:
            x.operand_types[k] = tag


class GrammarBlob:
    """Keeps the ctypes arrays of one ``gagp_grammar`` alive."""

    def __init__(self, t: PhaseTables, return_fuel: int = 1):
        self.tables = t
        n = len(t.expressions)
        self.expressions = (Expression * n)()
        for i, e in enumerate(t.expressions):
            x = self.expressions[i]
            x.kind, x.node_kind, x.opcode, x.operand, x.arity = e.kind, e.node_kind, e.opcode, e.operand, e.arity
            x.fuel, x.merge_fuel, x.type, x.target, x.scope_count = e.fuel, e.merge_fuel, e.type, e.target, e.scope_count
            for k in range(MAX_ARITY):
                x.children[k] = e.children[k]
                x.child_scope[k] = e.child_scope[k]
        self.productions = (Production * max(1, len(t.productions)))()
        for i, (x, w) in enumerate(t.productions):
            self.productions[i].expression, self.productions[i].weight = x, w
        self.nonterminals = (Nonterminal * max(1, len(t.nonterminals)))()
        for i, (off, cnt, scope, norm, fixed) in enumerate(t.nonterminals):
            nt = self.nonterminals[i]
            nt.production_offset, nt.production_count, nt.scope_count = off, cnt, scope
            nt.normalized_weights, nt.fixed = int(norm), int(fixed)
        self.domains = (Domain * max(1, len(t.domains)))()
        for i, d in enumerate(t.domains):
            x = self.domains[i]
            x.value_offset, x.value_count, x.integer_range = d.value_offset, d.value_count, int(d.integer_range)
            x.minimum, x.maximum = d.minimum, d.maximum
        self.values = (Value * max(1, len(t.values)))()
        for i, (tag, v) in enumerate(t.values):
            self.values[i].tag, self.values[i].i = tag, v
        self.minimum = np.ascontiguousarray(np.array(t.minimum, dtype=np.uint32))
        g = Grammar()
        g.expressions, g.expression_count = self.expressions, n
        g.productions, g.production_count = self.productions, len(t.productions)
        g.nonterminals, g.nonterminal_count = self.nonterminals, len(t.nonterminals)
        g.domains, g.domain_count = self.domains, len(t.domains)
        g.values, g.value_count = self.values, len(t.values)
        g.minimum = _ptr(self.minimum, C.c_uint32)
        g.depth_count, g.logical_depth_count, g.site_depth = t.depth_count, t.logical_depth_count, t.site_depth
        g.root_expression, g.slot_max_depth, g.slot_type = t.root_expression, t.slot_max_depth, t.slot_type
        g.local_count = len(t.local_types)
        for j, tag in enumerate(t.local_types):
            g.local_types[j] = tag
        g.max_nodes, g.fixed_nodes, g.return_fuel = t.max_nodes, t.fixed_nodes, return_fuel
        self.regions = (Region * max(1, len(t.regions)))()
        for i, r in enumerate(t.regions):
            x = self.regions[i]
            x.traversal, x.ranged, x.fuel_profile, x.result_type = r.traversal, int(r.ranged), 0, r.result_type
            if getattr(r, "event_cost", None):
                x.fuel_profile = 1
                for k, cost in enumerate(r.event_cost):
                    x.event_cost[k] = cost
            for k in range(3):
                x.binders[k], x.binding_types[k] = r.binders[k], r.binding_types[k]
            for k, tag in enumerate(r.operand_types[:6]):
                x.operand_types[k] = tag
            if r.plan is not None:
                fill_bounded_region(x, r)
        g.regions, g.region_count = self.regions, len(t.regions)
        self.struct = g

    def ref(self):
        return C.byref(self.struct)


class CasesBlob:
    """Case set: ``inputs[case, input]`` payloads and expected values.  An
    IntList input's payload is the index in ``list_values`` of its length
    word; its elements follow."""

    def __init__(self, inputs: np.ndarray, input_tags: Sequence[int], expected: np.ndarray, expected_tag: int = 0,
                 list_values: Optional[np.ndarray] = None):
        self.inputs = np.ascontiguousarray(np.asarray(inputs, dtype=np.int64).reshape(len(expected), -1))
        self.input_tags = np.ascontiguousarray(np.asarray(input_tags, dtype=np.int32))
        self.expected = np.ascontiguousarray(np.asarray(expected, dtype=np.int64))
        self.list_values = None if list_values is None else np.ascontiguousarray(np.asarray(list_values, dtype=np.int64))
        self.expected_tag = expected_tag
        c = Cases()
        c.case_count, c.input_count = len(self.expected), self.inputs.shape[1]
        c.inputs = _ptr(self.inputs, C.c_int64)
        c.input_tags = _ptr(self.input_tags, C.c_int32)
        c.expected = _ptr(self.expected, C.c_int64)
        c.expected_tag = expected_tag
        if self.list_values is not None and len(self.list_values):
            c.list_values, c.list_value_count = _ptr(self.list_values, C.c_int64), len(self.list_values)
        self.struct = c

    def list_at(self, case: int, input_index: int) -> List[int]:
        """The IntList value of one case input."""
        at = int(self.inputs[case, input_index])
        n = int(self.list_values[at])
        return [int(x) for x in self.list_values[at + 1:at + 1 + n]]

    def ref(self):
        return C.byref(self.struct)


@dataclass
class SearchSettings:
    """Effective ``gagp-search-config-v1`` semantics of a resident run."""

    population: int = 1024
    generations: int = 64
    seed: int = 0
    tournament_size: int = 2
    crossover_probability: float = 0.7
    crossover_attempts: int = 8
    mutation_probability: float = 0.3
    mutation_max_nodes: int = 0
    counted_sites: bool = True
    uniform_phase: bool = True
    site_depth: int = 7
    steady_state: bool = True
    batch: int = 0
    replacement_size: int = 2
    elite_count: int = 1
    fuel: int = 1000
    penalty: float = 1000.0
    metric: str = "absolute"
    grammar_site_ranking: bool = False
    reduction_lanes: int = 512

    def struct(self) -> SearchConfig:
        c = SearchConfig()
        c.population, c.generations, c.seed = self.population, self.generations, self.seed
        c.tournament_size, c.crossover_attempts = self.tournament_size, self.crossover_attempts
        c.crossover_probability, c.mutation_probability = self.crossover_probability, self.mutation_probability
        c.mutation_max_nodes = self.mutation_max_nodes
        c.counted_sites, c.uniform_phase = int(self.counted_sites), int(self.uniform_phase)
        c.steady_state, c.batch, c.replacement_size = int(self.steady_state), self.batch, self.replacement_size
        c.elite_count, c.fuel, c.penalty = self.elite_count, self.fuel, self.penalty
        c.metric, c.grammar_site_ranking = METRICS[self.metric], int(self.grammar_site_ranking)
        c.reduction_lanes = self.reduction_lanes
        return c


class RowsBuffer:
    """Caller-owned transport rows (``gagp_rows``)."""

    def __init__(self, count: int, stride: int, fill: bool = True):
        """``fill`` False leaves the arrays uninitialised, for rows the
        engine writes (a search result writes every slot of its width)."""
        self.count, self.stride = count, stride
        make = (lambda shape, dtype, value: np.full(shape, value, dtype=dtype)) if fill else \
            (lambda shape, dtype, value: np.empty(shape, dtype=dtype))
        self.node_counts = make(count, np.int32, 0)
        self.origins = make((count, stride), np.int32, -1)
        self.constant_counts = make(count, np.int32, 0)
        self.constants = make((count, stride), np.int64, 0)
        r = Rows()
        r.count, r.stride = count, stride
        r.node_counts = _ptr(self.node_counts, C.c_int32)
        r.origins = _ptr(self.origins, C.c_int32)
        r.constant_counts = _ptr(self.constant_counts, C.c_int32)
        r.constants = _ptr(self.constants, C.c_int64)
        self.struct = r

    @classmethod
    def from_rows(cls, rows: List[tuple], stride: int) -> "RowsBuffer":
        """``rows``: list of (origins, constants) sequences."""
        buf = cls(len(rows), stride)
        for i, (origins, constants) in enumerate(rows):
            buf.node_counts[i] = len(origins)
            buf.origins[i, : len(origins)] = origins
            buf.constant_counts[i] = len(constants)
            buf.constants[i, : len(constants)] = constants
        return buf

    def row(self, i: int) -> tuple:
        n, k = int(self.node_counts[i]), int(self.constant_counts[i])
        return tuple(int(x) for x in self.origins[i, :n]), tuple(int(x) for x in self.constants[i, :k])

    def ref(self):
        return C.byref(self.struct)


class ResultBuffer:
    """Caller-owned ``gagp_search_result`` arrays."""

    def __init__(self, generations: int, population: int, stride: int):
        self.history_best_fitness = np.zeros(generations, dtype=np.float64)
        self.history_mean_fitness = np.zeros(generations, dtype=np.float64)
        self.history_best_wrong = np.zeros(generations, dtype=np.int32)
        self.history_best_nodes = np.zeros(generations, dtype=np.int32)
        self.history_best = RowsBuffer(generations, stride)
        self.final_fitness = np.zeros(population, dtype=np.float64)
        self.final_wrong = np.zeros(population, dtype=np.int32)
        self.final_nodes = np.zeros(population, dtype=np.int32)
        self.final_rows = RowsBuffer(population, stride, fill=False)
        r = SearchResult()
        r.generations = generations
        r.history_best_fitness = _ptr(self.history_best_fitness, C.c_double)
        r.history_mean_fitness = _ptr(self.history_mean_fitness, C.c_double)
        r.history_best_wrong = _ptr(self.history_best_wrong, C.c_int32)
        r.history_best_nodes = _ptr(self.history_best_nodes, C.c_int32)
        r.history_best = self.history_best.struct
        r.population = population
        r.final_fitness = _ptr(self.final_fitness, C.c_double)
        r.final_wrong = _ptr(self.final_wrong, C.c_int32)
        r.final_nodes = _ptr(self.final_nodes, C.c_int32)
        r.final_rows = self.final_rows.struct
        self.struct = r

    def ref(self):
        return C.byref(self.struct)

    def summary(self) -> dict:
        g = self.struct.generations
        return {
            "history": [
                {"best_fitness": float(self.history_best_fitness[i]),
                 "mean_fitness": float(self.history_mean_fitness[i]),
                 "best_wrong": int(self.history_best_wrong[i]), "best_nodes": int(self.history_best_nodes[i]),
                 "row": self.history_best.row(i)} for i in range(g)],
            "final": [
                {"fitness": float(self.final_fitness[i]), "wrong": int(self.final_wrong[i]),
                 "nodes": int(self.final_nodes[i]), "row": self.final_rows.row(i)}
                for i in range(self.struct.population)],
            "evaluated_programs": int(self.struct.evaluated_programs),
            "reused_programs": int(self.struct.reused_programs),
            "program_cases": int(self.struct.program_cases),
        }
