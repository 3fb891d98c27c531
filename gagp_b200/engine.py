"""Python front end of the C ABI (include/gagp_b200.h) over ctypes.

``Engine`` mirrors the reference's resident owner and search loop
(``NativePhasePopulation`` + ``run_phase_population_steady``): admit a search,
run it on the device, read its history and final ranked population.  The
native library must be built (``gagp_b200.build``); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import abi
from .task import LoadedTask

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgagp_b200.so")
_lib = None


class EngineError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library():
    """Loads the in-tree engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(7, f"native engine library missing: {LIB_PATH} (run gagp_b200.build)")
        lib = C.CDLL(LIB_PATH)
        lib.gagp_b200_last_error.restype = C.c_char_p
        lib.gagp_b200_version.restype = C.c_char_p
        for name in ("gagp_b200_engine_create", "gagp_b200_search_bytes", "gagp_b200_search_create",
                     "gagp_b200_search_destroy", "gagp_b200_search_run", "gagp_b200_batch_run",
                     "gagp_b200_batch_step", "gagp_b200_search_result", "gagp_b200_batch_start",
                     "gagp_b200_batch_advance", "gagp_b200_search_progress", "gagp_b200_search_counters", "gagp_b200_engine_transfers",
                     "gagp_b200_engine_profile", "gagp_b200_engine_kernel_stats", "gagp_b200_engine_timeline",
                     "gagp_b200_evaluate_rows", "gagp_b200_judge_rows",
                     "gagp_b200_evaluate_rows_static", "gagp_b200_server_create", "gagp_b200_server_submit",
                     "gagp_b200_server_step", "gagp_b200_server_poll", "gagp_b200_server_set_rounds_per_step", "gagp_b200_server_times",
                     "gagp_b200_server_result", "gagp_b200_server_cancel"):
            getattr(lib, name).restype = C.c_int32
        lib.gagp_b200_engine_destroy.restype = None
        lib.gagp_b200_server_destroy.restype = None
        _lib = lib
    return _lib


def _check(status: int):
    if status != 0:
        raise EngineError(status, load_library().gagp_b200_last_error().decode())


class Search:
    """One admitted search held by an engine."""

    def __init__(self, engine: "Engine", sid: int, task: LoadedTask, grammar: abi.GrammarBlob):
        self.engine, self.id, self.task, self.grammar = engine, sid, task, grammar

    def run(self):
        self.engine.run(self)
        return self

    def result_buffer(self) -> abi.ResultBuffer:
        """The finished search's history and ranked population, copied into numpy arrays."""
        t, s = self.task.tables, self.task.settings
        res = abi.ResultBuffer(s.generations, s.population, t.max_nodes - t.fixed_nodes)
        _check(load_library().gagp_b200_search_result(self.engine.handle, self.id, res.ref()))
        return res

    def result(self) -> dict:
        return self.result_buffer().summary()

    def close(self):
        if self.id is not None and self.engine.handle:
            _check(load_library().gagp_b200_search_destroy(self.engine.handle, self.id))
            self.id = None


class Engine:
    """A device-resident GAGP engine on one GPU."""

    def __init__(self, device: int = 0, arena_bytes: int = 0):
        lib = load_library()
        h = C.c_void_p()
        _check(lib.gagp_b200_engine_create(C.c_int32(device), C.c_uint64(arena_bytes), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            load_library().gagp_b200_engine_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def search_bytes(task: LoadedTask) -> int:
        g = abi.GrammarBlob(task.tables)
        cfg = task.settings.struct()
        out = C.c_uint64(0)
        _check(load_library().gagp_b200_search_bytes(g.ref(), task.cases.ref(), C.byref(cfg), C.byref(out)))
        return int(out.value)

    def admit(self, task: LoadedTask, initial: Optional[abi.RowsBuffer] = None) -> Search:
        """Admits a search; `initial`: rows of an imported initial population
        (its first `population` rows), else the population is generated."""
        g = abi.GrammarBlob(task.tables)
        cfg = task.settings.struct()
        sid = C.c_int32(0)
        _check(load_library().gagp_b200_search_create(self.handle, g.ref(), task.cases.ref(), C.byref(cfg),
                                                     initial.ref() if initial is not None else None, C.byref(sid)))
        return Search(self, sid.value, task, g)

    def run(self, search: Search):
        _check(load_library().gagp_b200_search_run(self.handle, C.c_int32(search.id)))

    def run_batch(self, searches: Sequence[Search]):
        ids = (C.c_int32 * len(searches))(*[s.id for s in searches])
        _check(load_library().gagp_b200_batch_run(self.handle, ids, C.c_int32(len(searches))))

    def step(self, searches: Sequence[Search]) -> List[bool]:
        ids = (C.c_int32 * len(searches))(*[s.id for s in searches])
        fin = (C.c_int32 * len(searches))()
        _check(load_library().gagp_b200_batch_step(self.handle, ids, C.c_int32(len(searches)), fin))
        return [bool(x) for x in fin]

    def start(self, searches: Sequence[Search]):
        ids = (C.c_int32 * len(searches))(*[s.id for s in searches])
        _check(load_library().gagp_b200_batch_start(self.handle, ids, C.c_int32(len(searches))))

    def advance(self, searches: Sequence[Search], rounds: int, flush_l2: bool = False) -> float:
        """Runs ``rounds`` rounds of the started searches; returns device milliseconds."""
        ids = (C.c_int32 * len(searches))(*[s.id for s in searches])
        ms = C.c_double(0)
        _check(load_library().gagp_b200_batch_advance(self.handle, ids, C.c_int32(len(searches)), C.c_int32(rounds),
                                                      C.c_int32(int(flush_l2)), C.byref(ms)))
        return ms.value

    def counters(self, search: Search) -> dict:
        out = (C.c_uint64 * 25)()
        _check(load_library().gagp_b200_search_counters(self.handle, C.c_int32(search.id), out, C.c_int32(25)))
        return {"evaluated_programs": out[0], "reused_programs": out[1], "program_cases": out[2],
                "accumulator_ops": out[3], "exact_vm_instructions": out[24],
                "place_generate_cycles": out[4], "place_stage_cycles": out[5], "place_serial_cycles": out[6],
                "place_levels": out[7], "vary_bytes": out[8], "lower_bytes": out[9],
                "vary_select_cycles": out[10], "vary_crossover_cycles": out[11], "vary_generate_cycles": out[12],
                "vary_rest_cycles": out[13], "place_level_cycles": out[14], "vary_max_child_cycles": out[15],
                "vary_max_phase_cycles": list(out[16:20]), "vary_slow_children": out[20],
                "generate_steps": out[21], "generate_max_steps": out[22], "generations": out[23]}

    def transfers(self) -> tuple:
        """(host->device, device->host) bytes copied by this engine so far."""
        h2d, d2h = C.c_uint64(), C.c_uint64()
        _check(load_library().gagp_b200_engine_transfers(self.handle, C.byref(h2d), C.byref(d2h)))
        return h2d.value, d2h.value

    def progress(self, search: Search) -> tuple:
        done, total, fin = C.c_int32(), C.c_int32(), C.c_int32()
        _check(load_library().gagp_b200_search_progress(self.handle, C.c_int32(search.id), C.byref(done),
                                                        C.byref(total), C.byref(fin)))
        return done.value, total.value, bool(fin.value)

    def profile(self, enable: bool = True):
        _check(load_library().gagp_b200_engine_profile(self.handle, C.c_int32(int(enable))))

    def kernel_stats(self) -> Dict[str, dict]:
        lib = load_library()
        out = {}
        i = 0
        while True:
            name, ms, n = C.c_char_p(), C.c_double(), C.c_int64()
            if lib.gagp_b200_engine_kernel_stats(self.handle, C.c_int32(i), C.byref(name), C.byref(ms), C.byref(n)):
                break
            out[name.value.decode()] = {"ms": ms.value, "launches": n.value}
            i += 1
        return out

    def timeline(self) -> List[tuple]:
        """(kernel name, start ms, end ms) of the timed launches of the last
        batch of rounds read back, in launch order."""
        lib = load_library()
        count = C.c_int32()
        _check(lib.gagp_b200_engine_timeline(self.handle, C.c_int32(0), None, None, None, C.byref(count)))
        n = count.value
        kernel = (C.c_int32 * max(1, n))()
        start, end = (C.c_float * max(1, n))(), (C.c_float * max(1, n))()
        _check(lib.gagp_b200_engine_timeline(self.handle, C.c_int32(n), kernel, start, end, C.byref(count)))
        names = list(self.kernel_stats())
        return [(names[kernel[i]], start[i], end[i]) for i in range(min(n, count.value))]

    def evaluate_rows(self, task: LoadedTask, rows: abi.RowsBuffer):
        """Fitness and wrong counts of transport rows on the task's cases."""
        g = abi.GrammarBlob(task.tables)
        cfg = task.settings.struct()
        fitness = np.zeros(rows.count, dtype=np.float64)
        wrong = np.zeros(rows.count, dtype=np.uint32)
        _check(load_library().gagp_b200_evaluate_rows(self.handle, g.ref(), task.cases.ref(), C.byref(cfg), rows.ref(),
                                                      fitness.ctypes.data_as(C.POINTER(C.c_double)),
                                                      wrong.ctypes.data_as(C.POINTER(C.c_uint32))))
        return fitness, wrong

    def judge_rows(self, task: LoadedTask, rows: abi.RowsBuffer, cases: Optional[abi.CasesBlob] = None) -> List[dict]:
        """The reference's judgement (cases, correct, wrong, runtime_errors,
        mean_loss, solved) of each row on `cases`, by default the task's test
        split."""
        cases = cases if cases is not None else task.test_cases
        if cases is None:
            raise ValueError("the task has no test split")
        g = abi.GrammarBlob(task.tables)
        cfg = task.settings.struct()
        out = (abi.Verdict * max(1, rows.count))()
        _check(load_library().gagp_b200_judge_rows(self.handle, g.ref(), cases.ref(), C.byref(cfg), rows.ref(), out))
        return [out[i].summary() for i in range(rows.count)]

    def judge_best(self, task: LoadedTask, result: dict) -> dict:
        """The judgement of a search result's best program on the task's test
        split, as `gagp run` reports it under "test"."""
        stride = task.tables.max_nodes - task.tables.fixed_nodes
        return self.judge_rows(task, abi.RowsBuffer.from_rows([result["final"][0]["row"]], stride))[0]


def evaluate_rows_static(task: LoadedTask, rows: abi.RowsBuffer, stream: int = 0):
    """Row evaluation that allocates no device memory, for callers that may not
    allocate: a host application whose own allocator owns all device memory,
    or a latency-critical scoring loop that cannot pay for an allocation per
    call.  All device buffers live in the library's static 32 MiB scratch;
    larger requests raise EngineError(INVALID_ARGUMENT).  `stream` is a
    cudaStream_t handle (0: the default stream).  Calls share that scratch,
    so concurrent calls must be serialized by the caller."""
    g = abi.GrammarBlob(task.tables)
    cfg = task.settings.struct()
    fitness = np.zeros(rows.count, dtype=np.float64)
    wrong = np.zeros(rows.count, dtype=np.uint32)
    _check(load_library().gagp_b200_evaluate_rows_static(
        g.ref(), task.cases.ref(), C.byref(cfg), rows.ref(), fitness.ctypes.data_as(C.POINTER(C.c_double)),
        wrong.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(stream)))
    return fitness, wrong


REQUEST_QUEUED, REQUEST_RUNNING, REQUEST_DONE, REQUEST_FAILED = 0, 1, 2, 3


class Server:
    """Continuous-batching request loop over one engine (gagp_b200_server_*).

    submit() queues a search; every step() admits queued requests in arrival
    order while their device bytes fit `memory_budget`, runs up to
    `rounds_per_step` rounds of every running search in one batched launch
    sequence (a captured round replayed) and retires the
    finished ones; result() returns a finished request's history and final
    population exactly as Search.result() does for the search run alone."""

    def __init__(self, engine: Engine, memory_budget: int = 0, max_active: int = 0, rounds_per_step: int = 1):
        h = C.c_void_p()
        _check(load_library().gagp_b200_server_create(engine.handle, C.c_uint64(memory_budget),
                                                      C.c_int32(max_active), C.byref(h)))
        self.engine, self.handle, self.tasks = engine, h, {}
        if rounds_per_step != 1:
            _check(load_library().gagp_b200_server_set_rounds_per_step(h, C.c_int32(rounds_per_step)))

    def close(self):
        if self.handle:
            load_library().gagp_b200_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, task: LoadedTask) -> int:
        g = abi.GrammarBlob(task.tables)
        cfg = task.settings.struct()
        ticket = C.c_int64(0)
        _check(load_library().gagp_b200_server_submit(self.handle, g.ref(), task.cases.ref(), C.byref(cfg),
                                                      C.byref(ticket)))
        self.tasks[ticket.value] = task
        return ticket.value

    def step(self) -> tuple:
        """(running, queued, finished in this step)"""
        running, queued, done = C.c_int32(), C.c_int32(), C.c_int32()
        _check(load_library().gagp_b200_server_step(self.handle, C.byref(running), C.byref(queued), C.byref(done)))
        return running.value, queued.value, done.value

    def poll(self, ticket: int) -> int:
        state = C.c_int32()
        _check(load_library().gagp_b200_server_poll(self.handle, C.c_int64(ticket), C.byref(state)))
        return state.value

    def times(self, ticket: int) -> tuple:
        """(submitted, admitted, finished) seconds on the server clock; negative: not yet"""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _check(load_library().gagp_b200_server_times(self.handle, C.c_int64(ticket), C.byref(a), C.byref(b),
                                                     C.byref(c)))
        return a.value, b.value, c.value

    def result_buffer(self, ticket: int) -> abi.ResultBuffer:
        t = self.tasks.pop(ticket)
        s = t.settings
        res = abi.ResultBuffer(s.generations, s.population, t.tables.max_nodes - t.tables.fixed_nodes)
        _check(load_library().gagp_b200_server_result(self.handle, C.c_int64(ticket), res.ref()))
        return res

    def result(self, ticket: int) -> dict:
        return self.result_buffer(ticket).summary()

    def cancel(self, ticket: int):
        self.tasks.pop(ticket, None)
        _check(load_library().gagp_b200_server_cancel(self.handle, C.c_int64(ticket)))
