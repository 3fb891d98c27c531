"""TEST INFRASTRUCTURE ONLY -- ctypes loader of the C oracle (liboracle.so).

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gagp_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle C restatement (make -C oracle port)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "gagp_oracle.c")):
            build()
        lib = C.CDLL(LIB)
        lib.gagp_oracle_search.restype = C.c_int
        lib.gagp_oracle_search_reuse.restype = C.c_int
        lib.gagp_oracle_initial_population.restype = C.c_int
        lib.gagp_oracle_evaluate.restype = C.c_int
        lib.gagp_oracle_compile.restype = C.c_int
        lib.gagp_oracle_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def _check(rc: int):
    if rc < 0:
        raise RuntimeError("oracle: " + load().gagp_oracle_last_error().decode())


def search(grammar: abi.GrammarBlob, cases: abi.CasesBlob, settings: abi.SearchSettings,
           initial: "abi.RowsBuffer | None" = None, member_reuse: bool = False) -> dict:
    """A whole search.  `member_reuse` adds the reference's reuse of any
    identical member's result; without it only a child equal to its parent
    reuses (the rule the engine implements).  Results are the same either
    way; the evaluation counters differ."""
    lib = load()
    stride = grammar.tables.max_nodes - grammar.tables.fixed_nodes
    res = abi.ResultBuffer(settings.generations, settings.population, stride)
    cfg = settings.struct()
    _check(lib.gagp_oracle_search_reuse(grammar.ref(), cases.ref(), C.byref(cfg),
                                        initial.ref() if initial is not None else None, res.ref(),
                                        C.c_int(1 if member_reuse else 0)))
    return res.summary()


def initial_population(grammar: abi.GrammarBlob, settings: abi.SearchSettings) -> abi.RowsBuffer:
    lib = load()
    stride = grammar.tables.max_nodes - grammar.tables.fixed_nodes
    rows = abi.RowsBuffer(settings.population, stride)
    cfg = settings.struct()
    _check(lib.gagp_oracle_initial_population(grammar.ref(), C.byref(cfg), rows.ref()))
    return rows


def make_batch(grammar: abi.GrammarBlob, settings: abi.SearchSettings, selection, seed: int):
    """One make_batch over the generated initial population: the children's
    rows and their reusable parents (-1: none)."""
    lib = load()
    stride = grammar.tables.max_nodes - grammar.tables.fixed_nodes
    batch = settings.batch if settings.batch > 0 else settings.population
    rows = abi.RowsBuffer(batch, stride)
    reuse = np.full(batch, -2, dtype=np.int32)
    sel = np.ascontiguousarray(np.asarray(selection, dtype=np.float64))
    assert sel.size == settings.population
    cfg = settings.struct()
    _check(lib.gagp_oracle_make_batch(grammar.ref(), C.byref(cfg), sel.ctypes.data_as(C.POINTER(C.c_double)),
                                      C.c_uint64(seed), rows.ref(), reuse.ctypes.data_as(C.POINTER(C.c_int32))))
    return rows, reuse


def evaluate(grammar: abi.GrammarBlob, cases: abi.CasesBlob, settings: abi.SearchSettings,
             rows: abi.RowsBuffer):
    lib = load()
    fitness = np.zeros(rows.count, dtype=np.float64)
    wrong = np.zeros(rows.count, dtype=np.uint32)
    steps = C.c_uint64(0)
    cfg = settings.struct()
    _check(lib.gagp_oracle_evaluate(grammar.ref(), cases.ref(), C.byref(cfg), rows.ref(),
                                    fitness.ctypes.data_as(C.POINTER(C.c_double)),
                                    wrong.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(steps)))
    return fitness, wrong, int(steps.value)


def compile_row(grammar: abi.GrammarBlob, origins, constants):
    lib = load()
    o = np.ascontiguousarray(np.asarray(origins, dtype=np.int32))
    c = np.ascontiguousarray(np.asarray(constants if len(constants) else [0], dtype=np.int64))
    code = np.zeros(5 * 4096, dtype=np.int32)
    consts = np.zeros(1024, dtype=np.int64)
    nconst = C.c_int32(0)
    bound = C.c_int32(0)
    n = lib.gagp_oracle_compile(grammar.ref(), o.ctypes.data_as(C.POINTER(C.c_int32)), len(origins),
                                c.ctypes.data_as(C.POINTER(C.c_int64)), len(constants),
                                code.ctypes.data_as(C.POINTER(C.c_int32)), 4096,
                                consts.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(nconst), C.byref(bound))
    _check(n)
    return code[: 5 * n].reshape(n, 5).tolist(), consts[: nconst.value].tolist(), bound.value


def mt19937_64(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    load().gagp_oracle_mt19937_64(C.c_uint64(seed), out.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_int32(count))
    return out
