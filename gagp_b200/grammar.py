"""Grammar admission: ``grammar-definition-v2`` -> resident phase tables.

This is the cold host-side step that turns a user grammar into the flat tables
the device engine searches with.  It restates, for the scalar-expression
subset of the grammar language, three reference steps:

* ``compile_grammar`` (``cpp/src/evolution/grammar/compiled.cpp:150-215``):
  nonterminals and their alternatives are taken in sorted stable-id order
  (``cpp/src/evolution/grammar/definition.cpp:104-110,434-464``) and every
  expression is numbered in post order (``compiled.cpp:391-395``), so the ids
  below equal the reference's expression ids;
* ``compile_phase_grammar`` (``cpp/src/evolution/repro/gpu/phase_grammar.hpp:102-532``):
  the per-expression generation records, the production ranges in visit order,
  constant domains and the entry expression appended last;
* the site-depth cost table (``phase_grammar.hpp:496-530``) and the static
  weight normalisation (``phase_grammar.hpp:48-67``).

Beyond scalar expressions it admits lists, lets, traversals, statement
programs, bounded regions and fuel charges (``allow_lists``).  A construct
outside the subset raises :class:`Declined`, which is the
reference's resident-admission decline (``std::invalid_argument`` at
admission, ``cpp/src/evolution/evolve.cpp:45-49``).
"""
from __future__ import annotations

import json
import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

NO_ID = 0xFFFFFFFF

# ValueTag (cpp/include/gagp/core/value.hpp:16-27)
TAG_INT, TAG_FLOAT, TAG_BOOL, TAG_INTLIST, TAG_INVALID = 0, 1, 2, 5, 9
# completion tag of a statement, never a runtime value (kPhaseStatement,
# device/phase_compile.cuh:23)
TAG_STATEMENT = 0xF0
TYPE_TAGS = {"Int": TAG_INT, "Bool": TAG_BOOL}
# with the list subset
LIST_TYPE_TAGS = {"Int": TAG_INT, "Bool": TAG_BOOL, "IntList": TAG_INTLIST}

# PhaseExpressionKind (device/phase_generate.cuh:25)
EK_OPERATION, EK_CONSTANT, EK_BOUND, EK_REFERENCE, EK_INPUT, EK_ALIAS = range(6)
# PhaseTreeKind (device/phase_compile.cuh:21)
TK_CONSTANT, TK_LOCAL, TK_OPERATION, TK_IF, TK_AND, TK_OR = range(6)
TK_PROGRAM, TK_BLOCK, TK_NIL, TK_ASSIGN, TK_RETURN, TK_FOR_RANGE, TK_VAR = range(6, 13)
TK_LET, TK_BOUND, TK_REGION, TK_TRAVERSE = 13, 14, 15, 16
# grammar locals a phase can name (kPhaseNamedLocals), open lets and loops on
# one lowering path (kPhaseLets, kPhaseLoops, kPhaseWalks) and the
# evaluator's locals (MAX_LOCALS)
NAMED_LOCALS, LOWER_LETS, LOWER_LOOPS, LOWER_WALKS, MAX_LOCALS = 16, 16, 16, 8, 64
# Opcode (cpp/include/gagp/core/opcode.hpp:8-37)
OP = {"push_const": 0, "load": 1, "store": 2, "neg": 3, "not": 4, "add": 5, "sub": 6, "mul": 7,
      "div": 8, "mod": 9, "lt": 10, "le": 11, "gt": 12, "ge": 13, "eq": 14, "ne": 15, "jmp": 16,
      "jmp_if_false": 17, "jmp_if_true": 18, "call_builtin": 19, "return": 20}
# BuiltinId (cpp/include/gagp/core/builtin.hpp:13-45)
BUILTIN = {"abs": 0, "min": 1, "max": 2, "clip": 3, "len": 4, "index": 7, "is_int": 12, "idiv0": 13,
           "imod0": 14, "trunc_div0": 28, "trunc_mod0": 29}

# Scalar primitives of the catalog (cpp/src/evolution/grammar/catalog.cpp:83-116):
# name -> (argument types, result type, tree kind, opcode, builtin operand, printed name).
def _scalar_catalog() -> Dict[str, tuple]:
    cat = {}
    for t in ("Int", "Bool"):
        cat[f"if(Bool,{t},{t})->{t}"] = (("Bool", t, t), t, TK_IF, 0, 0, "if_expr")
        cat[f"eq({t},{t})->Bool"] = ((t, t), "Bool", TK_OPERATION, OP["eq"], 0, "eq")
        cat[f"ne({t},{t})->Bool"] = ((t, t), "Bool", TK_OPERATION, OP["ne"], 0, "ne")
    for name in ("add", "sub", "mul", "mod"):
        cat[f"{name}(Int,Int)->Int"] = (("Int", "Int"), "Int", TK_OPERATION, OP[name], 0, name)
    cat["neg(Int)->Int"] = (("Int",), "Int", TK_OPERATION, OP["neg"], 0, "neg")
    for name in ("lt", "le", "gt", "ge"):
        cat[f"{name}(Int,Int)->Bool"] = (("Int", "Int"), "Bool", TK_OPERATION, OP[name], 0, name)
    cat["not(Bool)->Bool"] = (("Bool",), "Bool", TK_OPERATION, OP["not"], 0, "not")
    cat["and(Bool,Bool)->Bool"] = (("Bool", "Bool"), "Bool", TK_AND, 0, 0, "and")
    cat["or(Bool,Bool)->Bool"] = (("Bool", "Bool"), "Bool", TK_OR, 0, 0, "or")
    for name in ("min", "max"):
        cat[f"{name}(Int,Int)->Int"] = (("Int", "Int"), "Int", TK_OPERATION, OP["call_builtin"], BUILTIN[name], name)
    cat["abs(Int)->Int"] = (("Int",), "Int", TK_OPERATION, OP["call_builtin"], BUILTIN["abs"], "abs")
    for name in ("idiv0", "imod0", "trunc_div0", "trunc_mod0"):
        cat[f"{name}(Int,Int)->Int"] = (("Int", "Int"), "Int", TK_OPERATION, OP["call_builtin"], BUILTIN[name], name)
    return cat


CATALOG = _scalar_catalog()
# List primitives of the list subset: len and the forward and reverse
# traversals of an IntList with an Int or Bool state (catalog.cpp:120-141;
# the body argument binds element, index and state).  The operand of a
# traversal entry here is its direction: 1 forward, 2 reverse.
LIST_CATALOG = {
    "len(IntList)->Int": (("IntList",), "Int", TK_OPERATION, OP["call_builtin"], BUILTIN["len"], "len"),
}
# let(value, body) binds one name for its body (catalog.cpp:89-92, a
# LET_REGION whose region argument is the body)
for _bound in ("Int", "Bool"):
    for _t in ("Int", "Bool"):
        LIST_CATALOG[f"let({_bound},{_t})->{_t}"] = ((_bound, _t), _t, TK_LET, 0, 0, "let_region")
for _state in ("Int", "Bool"):
    LIST_CATALOG[f"traverse(IntList,Int,{_state},{_state})->{_state}"] = (
        ("IntList", "Int", _state, _state), _state, TK_TRAVERSE, 0, 1, "traverse")
    LIST_CATALOG[f"traverse_reverse(IntList,Int,{_state},{_state})->{_state}"] = (
        ("IntList", "Int", _state, _state), _state, TK_TRAVERSE, 0, 2, "traverse_reverse")
# index(xs, i): Python-style indexing, an error out of range (catalog.cpp:128)
LIST_CATALOG["index(IntList,Int)->Int"] = (("IntList", "Int"), "Int", TK_OPERATION, OP["call_builtin"],
                                          BUILTIN["index"], "index")


def _controls() -> Dict[str, tuple]:
    """Statement controls of the catalog (catalog.cpp:53-68): key ->
    (argument slots as (category, value type or None for the control's own
    result contract), result category, tree kind, printed name, whether it
    names a local or input target)."""
    out = {
        "program(Block)->Program": ((("Block", None),), "Program", TK_PROGRAM, "program", False),
        "block_nil()->Block": ((), "Block", TK_NIL, "block_nil", False),
        "block_cons(Statement,Block)->Block": ((("Statement", None), ("Block", None)), "Block", TK_BLOCK,
                                               "block_cons", False),
        "if_stmt(Bool,Block,Block)->Statement": ((("Expression", "Bool"), ("Block", None), ("Block", None)),
                                                 "Statement", TK_IF, "if_stmt", False),
        "for_range(Int,Block)->Statement": ((("Expression", "Int"), ("Block", None)), "Statement", TK_FOR_RANGE,
                                            "for_range", True),
    }
    for t in ("Int", "Bool", "IntList"):
        out[f"assign({t})->Statement"] = ((("Expression", t),), "Statement", TK_ASSIGN, "assign", True)
        out[f"return({t})->Statement"] = ((("Expression", t),), "Statement", TK_RETURN, "return", False)
    return out


CONTROLS = _controls()
STATEMENT_CATEGORIES = ("Program", "Block", "Statement")


class Declined(ValueError):
    """The resident engine cannot hold this grammar (an admission decline)."""


@dataclass
class Expression:
    """One phase-grammar expression (``PhaseExpression``, phase_generate.cuh:79-92)."""

    kind: int = EK_OPERATION
    node_kind: int = TK_CONSTANT
    opcode: int = 0
    operand: int = 0
    arity: int = 0
    fuel: int = 1
    merge_fuel: int = 1
    type: int = TAG_INVALID
    target: int = -1
    children: List[int] = field(default_factory=lambda: [-1] * 8)
    scope_count: int = 0
    child_scope: List[int] = field(default_factory=lambda: [-1] * 8)
    name: str = ""
    result: str = ""          # grammar result type name
    scope_map: List[int] = field(default_factory=list)  # a reference's scope positions in its environment
    binding_types: List[int] = field(default_factory=list)  # a traversal body's element/index/state tags
    category: str = "Expression"  # syntax category: Expression, or Program/Block/Statement
    label: str = ""               # the local or input an assign, a for_range or a local read names
    plan: Optional["BoundedPlan"] = None  # a bounded region's plan (front end only)
    event_cost: Optional[List[int]] = None  # a traversal's fuel profile (26 PhaseFuelEvent charges)


@dataclass
class Domain:
    value_offset: int = 0
    value_count: int = 0
    integer_range: bool = False
    minimum: int = 0
    maximum: int = 0


@dataclass
class PhaseTables:
    """Flat resident tables of one admitted search (one whole-program phase)."""

    expressions: List[Expression]
    productions: List[Tuple[int, float]]          # (expression, weight)
    nonterminals: List[Tuple[int, int, int, bool, bool]]  # offset, count, scope, normalized, fixed
    domains: List[Domain]
    values: List[Tuple[int, int]]                 # (tag, payload)
    minimum: List[int]
    root_expression: int
    depth_count: int
    logical_depth_count: int
    site_depth: int
    # slot / layout
    slot_max_depth: int
    slot_type: int
    local_types: List[int]
    input_names: List[str]
    max_nodes: int
    fixed_nodes: int
    fuel: int
    names: List[str] = field(default_factory=list)  # printed name per expression
    labels: List[str] = field(default_factory=list)  # named target per expression ("" for none)
    # the value type a program returns: slot_type for an expression entry,
    # the entry's result contract for a Program entry (slot_type is then the
    # statement completion tag)
    result_type: int = TAG_INVALID
    local_names: List[str] = field(default_factory=list)  # grammar locals in declaration order
    # traversal table (HostPhaseGrammar::regions): a Traverse node's operand
    # indexes it; see Region
    regions: List["Region"] = field(default_factory=list)


@dataclass
class Region:
    """A traversal table entry (``PhaseRegionInfo``, device/phase_compile.cuh:47-60,
    as ``compile_phase_grammar`` fills it, phase_grammar.hpp:263-285): direction
    (1 forward, 2 reverse), the binder numbers of element, index and state, the
    children's operand types, the binding types and the result type."""

    traversal: int
    binders: List[int]
    operand_types: List[int]
    binding_types: List[int]
    result_type: int
    ranged: bool = False
    # a bounded region (traversal 0): its plan and phases (BoundedPlan)
    plan: Optional["BoundedPlan"] = None
    # a traversal's fuel profile: 26 PhaseFuelEvent charges (None: every instruction costs 1)
    event_cost: Optional[List[int]] = None


# region slot banks (RegionSlotBank, cpp/include/gagp/core/region_plan.hpp:96)
BANKS = {"state": 0, "parameter": 1, "prepared": 2, "result": 3, "measure": 4}
# capture kinds (PhaseCaptureKind, device/phase_compile.cuh:42)
CAPTURE_INPUT, CAPTURE_LOCAL, CAPTURE_BOUND = 0, 1, 2


@dataclass
class BoundedPlan:
    """A bounded region with coordinate progress (``RegionPlan``,
    cpp/include/gagp/core/region_plan.hpp:64-91, and the phase layout of
    ``compile_phase_grammar``, phase_grammar.hpp:331-385): initial states and
    bound operands, four phases (base predicate, base body, combine,
    boundary), requests that copy or offset states, coordinate axes with
    literal or operand bounds, and the frame, memo-cell and entry-fuel
    limits."""

    state_types: List[int]
    bound_count: int
    parameter_types: List[int]
    requests: List[List[Tuple[int, int, int]]]       # per request, per state: (kind 0 copy/1 offset, source, offset)
    axes: List[Tuple[int, Tuple[int, int], Tuple[int, int]]]  # (state slot, (lower kind, value), (upper kind, value))
    inclusive: bool
    memoized: bool
    frames: int
    cells: int
    entry_fuel: int
    captures: List[Tuple[int, int]]                  # (kind, target)
    phase_bindings: List[List[Tuple[int, int, int]]]  # per phase: (bank, slot, type)
    phase_types: List[int]


def _parse_int(text) -> int:
    if not isinstance(text, str):
        raise Declined("Int constant must be a decimal string")
    v = int(text, 10)
    if v < -(1 << 63) or v >= (1 << 63):
        raise Declined("Int constant out of range")
    return v


def load_definition(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


class _Compiler:
    def __init__(self, doc: dict, allow_lists: bool = False):
        self.allow_lists = allow_lists
        self.tags = LIST_TYPE_TAGS if allow_lists else TYPE_TAGS
        if doc.get("format_version") != "grammar-definition-v2":
            raise Declined("grammar-definition-v2 required")
        for key in ("imports", "templates"):
            if doc.get(key):
                raise Declined(f"grammar {key} are outside the resident scalar subset")
        if doc.get("locals") and not allow_lists:
            raise Declined("grammar locals are outside the resident scalar subset")
        self.doc = doc
        self.inputs = [(b["name"], b["type"]) for b in doc.get("inputs", [])]
        # grammar locals in declaration order: a local's number is its
        # position (compiled.cpp:155, binding())
        self.locals = [(b["name"], b["type"]) for b in doc.get("locals", [])]
        if any(t not in self.tags for _, t in self.locals):
            raise Declined("only Int/Bool/IntList grammar locals are resident")
        if {n for n, _ in self.locals} & {n for n, _ in self.inputs}:
            raise Declined("local declaration conflicts with input name")
        rules = sorted(doc["nonterminals"], key=lambda r: r["id"])
        self.rules = rules
        self.nt_ids = {r["id"]: i for i, r in enumerate(rules)}
        self.exprs: List[Expression] = []
        self.domains: List[dict] = []
        self.productions: List[Tuple[int, int, float]] = []  # (nonterminal, expression, weight)
        self.nt_productions: List[List[int]] = [[] for _ in rules]

    def expression(self, value: dict, scope: List[Tuple[str, str]]) -> int:
        """Front-end expression of ``value`` under the visible names ``scope``
        (the nonterminal's scope, then the binders of enclosing traversals)."""
        e = Expression()
        nt_scope = len(scope)
        if "constant" in value:
            d = value["constant"]
            if d.get("type") != "Int":
                raise Declined("only Int constant domains are resident")
            if "range" in d:
                lo, hi = (_parse_int(x) for x in d["range"])
                dom = {"integer_range": True, "minimum": lo, "maximum": hi}
            elif "values" in d:
                dom = {"integer_range": False, "values": [_parse_int(x) for x in d["values"]]}
                if not dom["values"]:
                    raise Declined("empty constant domain")
            else:
                raise Declined("constant sequence domains are not resident")
            e.kind, e.node_kind, e.target = EK_CONSTANT, TK_CONSTANT, len(self.domains)
            e.type, e.result, e.name = TAG_INT, "Int", "const"
            self.domains.append(dom)
        elif "input" in value:
            names = [n for n, _ in self.inputs]
            if value["input"] not in names:
                raise Declined("unknown input")
            idx = names.index(value["input"])
            t = self.inputs[idx][1]
            if t not in self.tags:
                raise Declined("only Int/Bool inputs are resident")
            e.kind, e.node_kind, e.target = EK_INPUT, TK_LOCAL, idx
            e.type, e.result, e.name = self.tags[t], t, value["input"]
        elif "ref" in value:
            if value["ref"] not in self.nt_ids:
                raise Declined("unknown nonterminal")
            target = self.nt_ids[value["ref"]]
            rule = self.rules[target]
            if rule.get("scope"):
                if not self.allow_lists:
                    raise Declined("scoped nonterminals are outside the scalar subset")
                # the target's scope names select from the visible names
                # (innermost first)
                names = [n for n, _ in scope]
                for slot in rule["scope"]:
                    if slot["name"] not in names:
                        raise Declined("scope map outside its environment")
                    e.scope_map.append(len(names) - 1 - names[::-1].index(slot["name"]))
                e.scope_count = len(e.scope_map)
            e.kind, e.target, e.result = EK_REFERENCE, target, rule["type"]
            e.category = rule.get("category", "Expression")
            e.type = TAG_STATEMENT if e.category in STATEMENT_CATEGORIES else self.tags.get(rule["type"], TAG_INVALID)
        elif "bound" in value and self.allow_lists:
            names = [n for n, _ in scope]
            if value["bound"] not in names:
                raise Declined("bound reference outside its environment")
            position = len(names) - 1 - names[::-1].index(value["bound"])
            t = scope[position][1]
            e.kind, e.node_kind, e.target = EK_BOUND, TK_BOUND, position
            e.type, e.result, e.name = self.tags.get(t, TAG_INVALID), t, value["bound"]
        elif "local" in value and self.allow_lists:
            # a read of a grammar local (a Var node naming the local)
            names = [n for n, _ in self.locals]
            if value["local"] not in names:
                raise Declined("unknown grammar local")
            idx = names.index(value["local"])
            if idx >= NAMED_LOCALS:
                raise Declined("grammar local capacity")
            t = self.locals[idx][1]
            e.kind, e.node_kind, e.operand = EK_OPERATION, TK_VAR, idx
            e.type, e.result, e.name, e.label = self.tags[t], t, "var", value["local"]
        elif "control" in value and self.allow_lists:
            # a statement control (compiled.cpp:498-526): its argument slots
            # are typed expressions or statement categories carrying the
            # control's own result contract ("type")
            if value["control"] not in CONTROLS:
                raise Declined(f"control {value['control']} is outside the resident subset")
            slots, category, tree_kind, name, named = CONTROLS[value["control"]]
            contract = value.get("type")
            if contract not in self.tags:
                raise Declined("statement result contract outside Int, Bool and IntList")
            if tree_kind == TK_RETURN and slots[0][1] != contract:
                raise Declined("return type disagrees with enclosing result contract")
            e.operand = 0
            if named:
                if ("name" in value) + ("input_name" in value) != 1:
                    raise Declined("control requires exactly one name or input_name target")
                targets = self.inputs if "input_name" in value else self.locals
                target = value["input_name"] if "input_name" in value else value["name"]
                tnames = [n for n, _ in targets]
                if target not in tnames:
                    raise Declined("control target is not visible")
                idx = tnames.index(target)
                if targets[idx][1] != slots[0][1]:
                    raise Declined("control target local type mismatch")
                if "input_name" in value:
                    e.operand = ("input", idx)  # resolved to -1 - evaluator position by the table builder
                else:
                    if idx >= NAMED_LOCALS:
                        raise Declined("grammar local capacity")
                    e.operand = idx
                e.label = target
            elif "name" in value or "input_name" in value:
                raise Declined("control does not accept a target name")
            args = value.get("args", [])
            if len(args) != len(slots):
                raise Declined("control argument count mismatch")
            children = [self.expression(a, scope) for a in args]
            for c, (cat, t) in zip(children, slots):
                if self.exprs[c].category != cat or self.exprs[c].result != (t if cat == "Expression" else contract):
                    raise Declined("control argument category or type mismatch")
            e.kind, e.node_kind, e.arity, e.category = EK_OPERATION, tree_kind, len(children), category
            e.result, e.name = contract, name
            # a statement completes without a value; an assign or a return
            # carries its value's type (phase_grammar.hpp:177,327-329)
            e.type = self.tags[slots[0][1]] if tree_kind in (TK_ASSIGN, TK_RETURN) else TAG_STATEMENT
            for i, c in enumerate(children):
                e.children[i] = c
                e.child_scope[i] = len(scope)
        elif "structured" in value and self.allow_lists:
            return self.bounded_region(value, scope)
        elif "signature" in value:
            sig = value["signature"]
            if sig in CATALOG:
                entry = CATALOG[sig]
            elif self.allow_lists and sig in LIST_CATALOG:
                entry = LIST_CATALOG[sig]
            else:
                raise Declined(f"primitive {sig} is outside the resident scalar subset")
            arg_types, result, tree_kind, opcode, operand, name = entry
            args = value.get("args", [])
            if len(args) != len(arg_types):
                raise Declined("argument count mismatch")
            binds = value.get("bind", {})
            if binds and tree_kind not in (TK_TRAVERSE, TK_LET):
                raise Declined("binders outside a traversal or let are outside the table builder's list subset")
            child_scopes = [scope] * len(args)
            if tree_kind == TK_LET:
                # the body (argument 1) binds the value
                names = binds.get("1", [])
                if set(binds) != {"1"} or len(names) != 1:
                    raise Declined("let capability")
                child_scopes[1] = scope + [(names[0], arg_types[0])]
            if tree_kind == TK_TRAVERSE:
                # the body (last argument) binds element, index and state
                body = len(args) - 1
                names = binds.get(str(body), [])
                if set(binds) != {str(body)} or len(names) != 3:
                    raise Declined("traversal capability")
                child_scopes[body] = scope + [(names[0], "Int"), (names[1], "Int"), (names[2], arg_types[2])]
            children = [self.expression(a, child_scopes[k]) for k, a in enumerate(args)]
            for c, t in zip(children, arg_types):
                if self.exprs[c].result != t:
                    raise Declined("argument type mismatch")
            e.kind, e.node_kind, e.opcode, e.operand = EK_OPERATION, tree_kind, opcode, operand
            e.arity, e.type, e.result, e.name = len(children), self.tags[result], result, name
            if tree_kind == TK_TRAVERSE:
                e.binding_types = [TAG_INT, TAG_INT, self.tags[arg_types[2]]]
            for i, c in enumerate(children):
                e.children[i] = c
                e.child_scope[i] = len(child_scopes[i])
        else:
            raise Declined("expression form outside the resident scalar subset")
        if "fuel_events" in value:
            self.fuel_events(e, value["fuel_events"])
        self.exprs.append(e)
        return len(self.exprs) - 1

    # traversal fuel events by PhaseFuelEvent number (device/phase_compile.cuh:36-40)
    TRAVERSAL_EVENTS = {"store_sequence": 4, "store_start": 5, "check_start": 8, "observe_sequence": 11,
                        "set_begin": 14, "set_end": 15, "initialize_state": 16, "initialize_cursor": 17,
                        "test_cursor": 18, "read_element": 19, "bind_element": 20, "compute_index": 21,
                        "update_state": 22, "advance_cursor": 23, "repeat": 24, "result": 25}

    @staticmethod
    def fuel_events(e: "Expression", events: dict) -> None:
        """Node-level fuel charges (fuel_charges and supports_fuel_event,
        cpp/src/evolution/grammar/compiled.cpp:47-72, fuel_events.cpp:159-176,
        as compile_phase_grammar places them, phase_grammar.hpp:386-395): an
        operation's (a constant's, an input's, a bound read's) `operation`
        charge and a value if's `branch_test` are its node's fuel, a value
        if's `branch_merge` its merge fuel, a let's `bind` its STORE's fuel.
        Traversal events are declined."""
        if not isinstance(events, dict) or not events:
            raise Declined("fuel_events must be a nonempty object")
        if e.kind == EK_OPERATION and e.node_kind == TK_TRAVERSE:
            # a traversal's profile: each event's first instruction carries
            # its charge (unlisted events cost 1, phase_grammar.hpp:272-274);
            # a zero charge lets the reference alias or skip instructions,
            # which is not restated here
            e.event_cost = [1] * 26
            for name, cost in events.items():
                if name not in _Compiler.TRAVERSAL_EVENTS:
                    raise Declined(f"fuel event {name} outside a traversal's events")
                if not 1 <= int(cost) < 2 ** 31:
                    raise Declined("zero-cost traversal events are outside the resident subset")
                e.event_cost[_Compiler.TRAVERSAL_EVENTS[name]] = int(cost)
            return
        for name, cost in events.items():
            cost = int(cost)
            if not 0 <= cost < 2 ** 31:
                raise Declined("fuel event cost")
            kind = e.node_kind if e.kind == EK_OPERATION else None
            if name == "operation" and (e.kind in (EK_CONSTANT, EK_INPUT, EK_BOUND) or kind in (TK_OPERATION, TK_VAR)):
                e.fuel = cost
            elif name == "bind" and kind == TK_LET:
                e.fuel = cost
            elif name == "branch_test" and kind == TK_IF and e.type != TAG_STATEMENT:
                e.fuel = cost
            elif name == "branch_merge" and kind == TK_IF and e.type != TAG_STATEMENT:
                e.merge_fuel = cost
            else:
                raise Declined(f"fuel event {name} outside the node-level charges")

    def bounded_region(self, value: dict, scope: List[Tuple[str, str]]) -> int:
        """A bounded structured expression (compiled.cpp:538-640) in the
        subset this engine runs: coordinate progress, requests that copy or
        offset states, no preparations and no request expressions."""
        st = value["structured"]
        if st.get("family") != "bounded":
            raise Declined("structured family outside bounded regions")
        plan = st["plan"]
        if plan.get("version", 1) != 1 or plan.get("progress") != "coordinates":
            raise Declined("bounded regions other than coordinate recurrences")
        if plan.get("preparations") or plan.get("request_expression_types"):
            raise Declined("bounded region preparations and request expressions")
        state_types = [self.tags.get(t, TAG_INVALID) for t in plan["state_types"]]
        if not state_types or len(state_types) > 4 or any(t != TAG_INT for t in state_types):
            raise Declined("bounded region states other than 1..4 Int coordinates")
        bound_count = int(plan.get("bound_operand_count", 0))
        if not 0 <= bound_count <= 8:
            raise Declined("bounded region bound operands")
        result = plan["result_type"]
        if result not in ("Int", "Bool"):
            raise Declined("bounded region result type")
        parameters = plan.get("parameter_types", [])
        if len(parameters) > 8 or any(t not in self.tags for t in parameters):
            raise Declined("bounded region parameters")
        requests = []
        for r in plan["requests"]:
            row = []
            for tr in r["states"]:
                kind = {"copy_state": 0, "coordinate_offset": 1}.get(tr["kind"])
                if kind is None:
                    raise Declined("bounded region transition outside copy and coordinate offset")
                source = int(tr["source_state"])
                if not 0 <= source < len(state_types):
                    raise Declined("bounded region transition source")
                row.append((kind, source, _parse_int(tr.get("offset", "0")) if kind == 1 else 0))
            if len(row) != len(state_types):
                raise Declined("bounded region request shape")
            requests.append(row)
        if not 1 <= len(requests) <= 8:
            raise Declined("bounded region request count")
        slots = [int(x) for x in plan["coordinate_slots"]]
        domains = plan["coordinate_domains"]
        if not slots or len(slots) != len(domains) or any(not 0 <= x < len(state_types) for x in slots):
            raise Declined("bounded region coordinate axes")

        def bound(b):
            if b["kind"] == "literal":
                return (0, _parse_int(b["literal"]))
            if b["kind"] == "operand":
                k = int(b["operand"])
                if not 0 <= k < len(state_types) + bound_count:
                    raise Declined("bounded region bound operand")
                return (1, k)
            raise Declined("bounded region bound kind")
        axes = [(x, bound(d["lower"]), bound(d["upper"])) for x, d in zip(slots, domains)]
        limits = plan.get("limits", {})
        frames, cells, entry_fuel = int(limits.get("frames", 64)), int(limits.get("cells", 0)), \
            int(limits.get("entry_fuel", 1))
        if not 0 <= frames <= 128 or not 0 <= cells <= 256 or not 0 <= entry_fuel < 2 ** 31:
            raise Declined("bounded region limits")
        # captures: the caller's inputs, grammar locals or binders the
        # phases read as parameters
        captures = []
        for cap, ptype in zip(value.get("captures", []), parameters):
            if "input" in cap:
                names = [n for n, _ in self.inputs]
                if cap["input"] not in names:
                    raise Declined("bounded region capture")
                k = names.index(cap["input"])
                captures.append((CAPTURE_INPUT, k, self.inputs[k][1]))
            elif "local" in cap:
                names = [n for n, _ in self.locals]
                if cap["local"] not in names:
                    raise Declined("bounded region capture")
                k = names.index(cap["local"])
                captures.append((CAPTURE_LOCAL, k, self.locals[k][1]))
            elif "bound" in cap:
                names = [n for n, _ in scope]
                if cap["bound"] not in names:
                    raise Declined("bounded region capture")
                k = len(names) - 1 - names[::-1].index(cap["bound"])
                captures.append((CAPTURE_BOUND, k, scope[k][1]))
            else:
                raise Declined("bounded region capture")
            if captures[-1][2] != ptype:
                raise Declined("bounded region capture type mismatch")
        if len(captures) != len(parameters):
            raise Declined("bounded region capture count must match plan parameters")
        operands = len(state_types) + bound_count
        phases = value["phases"]
        if len(phases) != 4:
            raise Declined("bounded region phases")
        # phase kinds in argument order: base predicate, base body, combine,
        # boundary (bounded_region_phase_kind, region_plan.cpp:511-527)
        phase_types = [TAG_BOOL, self.tags[result], self.tags[result], self.tags[result]]
        phase_scopes, phase_bindings = [], []
        for p, ph in enumerate(phases):
            if int(ph["argument"]) != operands + p:
                raise Declined("bounded region phase argument is not canonical")
            names, bindings = [], []
            for b in ph["bindings"]:
                bank = BANKS.get(b["bank"])
                slot = int(b["slot"])
                if bank == BANKS["state"] and 0 <= slot < len(state_types):
                    t = "Int"
                elif bank == BANKS["parameter"] and 0 <= slot < len(parameters):
                    t = parameters[slot]
                elif bank == BANKS["result"] and p == 2 and 0 <= slot < len(requests):
                    t = result
                else:
                    raise Declined("bounded region binding outside the subset")
                names.append((b["name"], t))
                bindings.append((bank, slot, self.tags[t]))
            if len(bindings) > 7:
                raise Declined("bounded region phase binding capacity")
            phase_scopes.append(names)
            phase_bindings.append(bindings)
        args = value.get("args", [])
        if len(args) != operands + 4:
            raise Declined("bounded region argument count")
        arg_types = ["Int"] * operands + ["Bool", result, result, result]
        children = []
        for k, a in enumerate(args):
            children.append(self.expression(a, scope if k < operands else phase_scopes[k - operands]))
            if self.exprs[children[-1]].result != arg_types[k] or self.exprs[children[-1]].category != "Expression":
                raise Declined("bounded region argument type mismatch")
        e = Expression(kind=EK_OPERATION, node_kind=TK_REGION, arity=len(children), type=self.tags[result],
                       result=result, name="bounded_region")
        for k, ch in enumerate(children):
            e.children[k] = ch
            e.child_scope[k] = len(scope) if k < operands else len(phase_scopes[k - operands])
        fuel = value.get("fuel_events", {})
        if set(fuel) - {"operation"}:
            raise Declined("bounded region fuel profile capability")
        e.fuel = int(fuel.get("operation", 1))
        e.plan = BoundedPlan(state_types=state_types, bound_count=bound_count,
                             parameter_types=[self.tags[t] for t in parameters], requests=requests, axes=axes,
                             inclusive=plan.get("coordinate_endpoint", "exclusive") == "inclusive",
                             memoized=bool(plan.get("memoized", False)), frames=frames, cells=cells,
                             entry_fuel=entry_fuel, captures=[(k, t) for k, t, _ in captures],
                             phase_bindings=phase_bindings, phase_types=phase_types)
        self.exprs.append(e)
        return len(self.exprs) - 1

    def compile(self):
        for i, rule in enumerate(self.rules):
            category = rule.get("category", "Expression")
            if category != "Expression" and (not self.allow_lists or category not in STATEMENT_CATEGORIES):
                raise Declined("statement grammars are outside the scalar subset")
            if rule["type"] not in (self.tags if category != "Expression" else TYPE_TAGS):
                raise Declined("only Int/Bool nonterminals are resident")
            scope = [(slot["name"], slot["type"]) for slot in rule.get("scope", [])]
            if scope and (not self.allow_lists or any(t not in self.tags for _, t in scope) or len(scope) > 8):
                raise Declined("scoped nonterminals are outside the scalar subset")
            for alt in sorted(rule["alternatives"], key=lambda a: a["id"]):
                w = float(alt["weight"])
                if not (w > 0) or w == float("inf"):
                    raise Declined("production weight")
                x = self.expression(alt["expression"], scope)
                if self.exprs[x].result != rule["type"] or self.exprs[x].category != category:
                    raise Declined("production result type mismatch")
                self.nt_productions[i].append(len(self.productions))
                self.productions.append((i, x, w))


def compile_tables(doc: dict, input_names: Optional[List[str]] = None, site_depth: int = 7,
                   allow_lists: bool = False) -> PhaseTables:
    """Admit ``doc`` and build the resident tables (one whole-program slot).

    ``allow_lists`` admits the engine's whole subset beyond scalar
    expressions, as compile_phase_grammar builds it
    (``phase_grammar.hpp:94-400``): IntList inputs, len and index, forward
    and reverse traversals with their element/index/state binders, lets,
    scoped nonterminals and bound names, statement programs with grammar
    locals, bounded regions and fuel charges.  Task loading
    (``task.assemble``) always passes it."""
    c = _Compiler(doc, allow_lists)
    c.compile()
    entry = doc["entry"]
    root_nt = c.nt_ids[entry["nonterminal"]]
    # a Program entry is its own whole-program phase, without the expression
    # entry's terminator (phase_layout.hpp:118-130)
    program_entry = c.rules[root_nt].get("category", "Expression") == "Program"
    if c.rules[root_nt].get("category", "Expression") not in ("Expression", "Program"):
        raise Declined("whole-program phase requires an expression or program entry")
    limits = doc["search_limits"]
    max_depth, max_nodes = int(limits["max_depth"]), int(limits["max_nodes"])
    fuel = int(doc["execution_limits"]["fuel"])
    if not (1 <= max_depth <= 64) or max_nodes > 2048 or not (0 <= site_depth <= 15):
        raise Declined("depth/node capacity")
    grammar_inputs = [n for n, _ in c.inputs]
    names = sorted(grammar_inputs) if input_names is None else list(input_names)
    if sorted(names) != sorted(grammar_inputs) or len(names) > 64:
        raise Declined("input names must exactly cover grammar inputs")

    # compile_phase_grammar: visit from the entry nonterminal.
    n_expr = len(c.exprs)
    out_expr = [Expression() for _ in range(n_expr)]
    out_nts = [[0, 0, 0, False, False] for _ in c.rules]
    out_prods: List[Tuple[int, float]] = []
    out_domains = [Domain() for _ in c.domains]
    out_values: List[Tuple[int, int]] = []
    seen_nt, seen_expr, seen_dom = set(), set(), set()
    # lexical environments: the binder numbers visible to a nonterminal or an
    # expression (one per scope position); binders are numbered statically,
    # a traversal's three above every visible one
    nt_env: Dict[int, List[int]] = {}
    expr_env: Dict[int, List[int]] = {}
    regions: List[Region] = []

    def visit_nt(i: int, env: List[int]):
        if i in seen_nt:
            if nt_env[i] != env:
                raise Declined("nonterminal entered under two lexical environments")
            return
        seen_nt.add(i)
        nt_env[i] = env
        out_nts[i][0] = len(out_prods)
        out_nts[i][2] = len(c.rules[i].get("scope", []))
        # a nonterminal with variation disabled opens no variation site
        # (phase_variation.hpp:13)
        out_nts[i][4] = not c.rules[i].get("variation", True)
        for p in c.nt_productions[i]:
            _, x, w = c.productions[p]
            out_prods.append((x, w))
            out_nts[i][1] += 1
        for p in c.nt_productions[i]:
            visit_expr(c.productions[p][1], env)

    def visit_expr(i: int, env: List[int]):
        if i in seen_expr:
            if expr_env[i] != env:
                raise Declined("expression entered under two lexical environments")
            return
        seen_expr.add(i)
        expr_env[i] = env
        e = c.exprs[i]
        x = out_expr[i]
        x.kind, x.type, x.target, x.name, x.result = e.kind, e.type, e.target, e.name, e.result
        x.category, x.label = e.category, e.label
        if e.kind == EK_REFERENCE:
            x.scope_count, x.scope_map = e.scope_count, list(e.scope_map)
            visit_nt(e.target, [env[m] for m in e.scope_map])
            return
        x.node_kind, x.opcode, x.operand, x.arity = e.node_kind, e.opcode, e.operand, e.arity
        x.fuel, x.merge_fuel = e.fuel, e.merge_fuel
        x.children, x.child_scope = list(e.children), list(e.child_scope)
        child_env = [env] * e.arity
        if isinstance(e.operand, tuple):
            # an input target is the preset evaluator slot -1 - position
            # (phase_grammar.hpp:310-320)
            x.operand = -1 - names.index(grammar_inputs[e.operand[1]])
        if e.kind == EK_BOUND:
            x.operand = env[e.target]
        elif e.node_kind == TK_LET:
            # one binder, numbered above every visible one (phase_grammar.hpp:255-261)
            binder = max(env) + 1 if env else 0
            if binder >= 16:
                raise Declined("let capability")
            child_env[1] = env + [binder]
            x.operand = binder
        elif e.node_kind == TK_REGION:
            # a bounded region (phase_grammar.hpp:331-385): operands see the
            # surrounding environment; phase p sees only its own bindings,
            # numbered from zero
            plan = e.plan
            operands = len(plan.state_types) + plan.bound_count
            for p in range(4):
                child_env[operands + p] = list(range(len(plan.phase_bindings[p])))
                _check_phase_closed(c, e.children[operands + p])
            captures = []
            for kind, target in plan.captures:
                if kind == CAPTURE_INPUT:
                    target = names.index(grammar_inputs[target])
                elif kind == CAPTURE_BOUND:
                    target = env[target]
                elif target >= NAMED_LOCALS:
                    raise Declined("grammar local capacity")
                captures.append((kind, target))
            x.operand = len(regions)
            regions.append(Region(traversal=0, binders=[0, 0, 0],
                                  operand_types=[c.exprs[k].type for k in e.children[:operands]],
                                  binding_types=[TAG_INVALID] * 3, result_type=e.type,
                                  plan=BoundedPlan(**dict(plan.__dict__, captures=captures))))
        elif e.node_kind == TK_TRAVERSE:
            binder = max(env) + 1 if env else 0
            if binder + 2 >= 16:
                raise Declined("traversal capability")
            child_env[e.arity - 1] = env + [binder, binder + 1, binder + 2]
            x.operand = len(regions)
            regions.append(Region(traversal=e.operand, binders=[binder, binder + 1, binder + 2],
                                  operand_types=[c.exprs[k].type for k in e.children[:e.arity]],
                                  binding_types=list(e.binding_types), result_type=e.type,
                                  event_cost=list(e.event_cost) if e.event_cost else None))
        if len(env) > 15:
            raise Declined("lexical environment capacity")
        if e.kind == EK_CONSTANT and e.target not in seen_dom:
            seen_dom.add(e.target)
            d = c.domains[e.target]
            dom = out_domains[e.target]
            dom.integer_range = d["integer_range"]
            if d["integer_range"]:
                dom.minimum, dom.maximum = d["minimum"], d["maximum"]
            else:
                dom.value_offset, dom.value_count = len(out_values), len(d["values"])
                out_values.extend((TAG_INT, v) for v in d["values"])
        if e.kind == EK_INPUT:
            position = names.index(grammar_inputs[e.target])
            x.target = position
            x.operand = position
        for k in range(e.arity):
            x.child_scope[k] = len(child_env[k])
            visit_expr(e.children[k], child_env[k])

    visit_nt(root_nt, list(range(len(c.rules[root_nt].get("scope", [])))))
    # Productions may not share a root node and must resolve to a node.
    resolved = set()
    for x, _ in out_prods:
        if out_expr[x].kind == EK_REFERENCE:
            raise Declined("root aliases require native fallback")
        if x in resolved:
            raise Declined("productions sharing a root node require native fallback")
        resolved.add(x)

    depth_count = max_depth + 1
    # An expression entry runs as program(block(return e)): the phase starts at
    # AST depth 4 and keeps max_depth - 3 levels (phase_layout.hpp:131-134),
    # and the four wrapper nodes are the layout's fixed nodes.
    # A Program entry's phase is the whole tree: it starts at depth 1 and has
    # no fixed nodes.
    slot_max_depth = max_depth if program_entry else max_depth - 3
    if slot_max_depth < 1:
        raise Declined("max_depth leaves no room for the entry phase")
    entry_expr = Expression(kind=EK_REFERENCE, target=root_nt, name="", result=c.rules[root_nt]["type"],
                            category=c.rules[root_nt].get("category", "Expression"))
    root_expression = n_expr
    out_expr.append(entry_expr)
    _check_lowering_capacity(out_expr, out_nts, out_prods, seen_expr | {root_expression}, root_expression,
                             depth_count, max_depth, len(names), len(c.locals))
    logical_count = site_depth + 1 if site_depth else 1
    minimum = _minimum_table(out_expr, out_nts, out_prods, seen_expr | {root_expression}, depth_count,
                             logical_count, site_depth > 0)
    tables = PhaseTables(
        expressions=out_expr, productions=out_prods,
        nonterminals=[tuple(n) for n in out_nts], domains=out_domains, values=out_values,
        minimum=minimum, root_expression=root_expression, depth_count=depth_count,
        logical_depth_count=logical_count, site_depth=site_depth,
        slot_max_depth=slot_max_depth,
        slot_type=TAG_STATEMENT if program_entry else TYPE_TAGS[c.rules[root_nt]["type"]],
        local_types=[c.tags[dict(c.inputs)[n]] for n in names], input_names=names,
        max_nodes=max_nodes, fixed_nodes=0 if program_entry else 4, fuel=fuel,
        names=[e.name for e in out_expr], regions=regions, labels=[e.label for e in out_expr],
        result_type=c.tags[c.rules[root_nt]["type"]] if program_entry else TYPE_TAGS[c.rules[root_nt]["type"]],
        local_names=[n for n, _ in c.locals])
    _normalize_static_weights(tables)
    return tables


def _check_phase_closed(c: "_Compiler", root: int) -> None:
    """A region phase reads only its bindings: no input, grammar local,
    statement, traversal or nested region is reachable from it
    (phase_grammar.hpp:413-431)."""
    seen = set()
    stack = [root]
    while stack:
        i = stack.pop()
        if i in seen:
            continue
        seen.add(i)
        e = c.exprs[i]
        if e.kind == EK_INPUT or e.node_kind in (TK_VAR, TK_REGION, TK_TRAVERSE) and e.kind == EK_OPERATION \
                or e.category != "Expression":
            raise Declined("region phase reaches a program variable, statement, traversal or nested region")
        if e.kind == EK_REFERENCE:
            stack.extend(c.productions[p][1] for p in c.nt_productions[e.target])
        else:
            stack.extend(e.children[:e.arity])


def _check_lowering_capacity(exprs, nts, prods, reachable, root, depth_count, max_depth, inputs, named_locals):
    """Decline a grammar whose trees within the depth budget could run the
    lowering out of its fixed tables (phase_grammar.hpp:455-498): over every
    derivation, the open traversals, lets, loops and value ifs on one path and
    the temporaries they hold (nine for a traversal, one for a let or a
    loop), next to the inputs and the grammar locals."""
    plain = _minimum_table(exprs, nts, prods, reachable, depth_count, 1, False)
    TEMPS, WALKS, LETS, LOOPS, IFS = range(5)
    memo = {}

    def feasible(i, d):
        return plain[i * depth_count + d] != NO_ID

    def need(i, d):
        key = (i, d)
        if key in memo:
            return memo[key]
        e = exprs[i]
        h = [0] * 5
        if e.kind == EK_REFERENCE:
            off, count = nts[e.target][0], nts[e.target][1]
            for p in range(off, off + count):
                x = prods[p][0]
                if feasible(x, d):
                    h = [max(a, b) for a, b in zip(h, need(x, d))]
        elif d > 0:
            for k in range(e.arity):
                if feasible(e.children[k], d - 1):
                    h = [max(a, b) for a, b in zip(h, need(e.children[k], d - 1))]
            if e.node_kind == TK_TRAVERSE:
                h[TEMPS] += 9
                h[WALKS] += 1
            elif e.node_kind == TK_LET:
                h[TEMPS] += 1
                h[LETS] += 1
            elif e.node_kind == TK_FOR_RANGE:
                h[TEMPS] += 1
                h[LOOPS] += 1
            elif e.node_kind == TK_IF and e.type != TAG_STATEMENT:
                h[IFS] += 1
        memo[key] = h
        return h

    import sys
    old = sys.getrecursionlimit()
    sys.setrecursionlimit(max(old, 100000))
    try:
        h = need(root, max_depth)
    finally:
        sys.setrecursionlimit(old)
    named = min(named_locals, NAMED_LOCALS)
    if (inputs + named + h[TEMPS] > MAX_LOCALS or h[WALKS] > LOWER_WALKS or h[LETS] > LOWER_LETS
            or h[LOOPS] > LOWER_LOOPS or (h[WALKS] and h[IFS] > 16)):
        raise Declined("lowering capacity within the depth budget requires native fallback")


def _minimum_table(exprs, nts, prods, reachable, depth_count, logical_count, site_depth):
    """Minimum nodes of each (expression, depth, site budget) (phase_grammar.hpp:496-530).

    Without a site-depth limit the logical dimension has one entry and a
    reference does not consume it.
    """
    size = len(exprs) * depth_count * logical_count
    table = [NO_ID] * size
    done = [False] * size

    def cost(i: int, d: int, l: int) -> int:
        key = (i * depth_count + d) * logical_count + l
        if done[key]:
            return table[key]
        done[key] = True
        e = exprs[i]
        result = NO_ID
        if e.kind == EK_REFERENCE:
            if site_depth and not l:
                return NO_ID
            off, count = nts[e.target][0], nts[e.target][1]
            nl = l - 1 if site_depth else l
            for p in range(off, off + count):
                result = min(result, cost(prods[p][0], d, nl))
        elif d > 0:
            total = 1
            for k in range(e.arity):
                total += cost(e.children[k], d - 1, l)
            result = NO_ID if total >= NO_ID else total
        table[key] = result
        return result

    import sys
    old = sys.getrecursionlimit()
    sys.setrecursionlimit(max(old, 100000))
    try:
        for i in sorted(reachable):
            for d in range(depth_count):
                for l in range(logical_count):
                    cost(i, d, l)
    finally:
        sys.setrecursionlimit(old)
    return table


def _normalize_static_weights(t: PhaseTables) -> None:
    """Divide weights by the maximum when a maximum-weight alternative is always
    among the cheapest (phase_grammar.hpp:48-67)."""
    per = t.depth_count * t.logical_depth_count
    nts = [list(n) for n in t.nonterminals]
    prods = list(t.productions)
    for nt in nts:
        off, count = nt[0], nt[1]
        if not count:
            continue
        maximum = max(prods[off + i][1] for i in range(count))
        proven = maximum > 0
        for depth in range(per):
            if not proven:
                break
            cheapest = max_weight_cheapest = NO_ID
            for i in range(count):
                x, w = prods[off + i]
                cost = t.minimum[x * per + depth]
                cheapest = min(cheapest, cost)
                if w == maximum:
                    max_weight_cheapest = min(max_weight_cheapest, cost)
            proven = cheapest == max_weight_cheapest
        if not proven:
            continue
        for i in range(count):
            x, w = prods[off + i]
            prods[off + i] = (x, w / maximum)
        nt[3] = True
    t.nonterminals = [tuple(n) for n in nts]
    t.productions = prods


def compile_file(path: str, input_names: Optional[List[str]] = None, site_depth: int = 7) -> PhaseTables:
    return compile_tables(load_definition(path), input_names, site_depth)
