"""The engine's lowering and exact VM compiled for the host (test harness).

``tests/native/lower_host.cu`` includes the same ``lower_program`` and
``run_program`` the device kernels run and exposes them through ctypes, so
CPU tests can compare them with the reference's own compiler output and CPU
evaluator.  The library is built with nvcc into ``tests/_build/`` on first
use; the product never loads it."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCE = os.path.join(HERE, "native", "lower_host.cu")
LIB = os.path.join(HERE, "_build", "liblower_host.so")
DEPS = [SOURCE] + [os.path.join(ROOT, "gagp_b200", "csrc", f) for f in
                   ("vm.cuh", "lower.cuh", "device_ops.cuh", "search_state.h")] + \
    [os.path.join(ROOT, "include", "gagp_b200.h")]

_lib = None


def library():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in DEPS):
        from gagp_b200.build import nvcc
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run([nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC", "-shared", SOURCE, "-o", LIB], check=True)
    lib = C.CDLL(LIB)
    lib.host_lower.restype = C.c_int
    lib.host_run.restype = C.c_int
    _lib = lib
    return lib


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def lower(grammar_blob, origins, constants, code_cap=4096, shape=False):
    """(code as an (n, 5) array, constants, locals, stack bound), or None when
    the lowering rejects the row; with `shape` also the main code's
    instructions and constants (a program with bounded regions has records
    and phase code after them)."""
    lib = library()
    o = _i32(origins)
    k = np.ascontiguousarray(np.asarray(constants, dtype=np.int64))
    code = np.zeros((code_cap, 5), dtype=np.int32)
    consts = np.zeros(code_cap, dtype=np.int64)
    out = np.zeros(6, dtype=np.int32)
    n = lib.host_lower(grammar_blob.ref(), o.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int(len(o)),
                       k.ctypes.data_as(C.POINTER(C.c_int64)), C.c_int(len(k)),
                       code.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int(code_cap),
                       consts.ctypes.data_as(C.POINTER(C.c_int64)), C.c_int(code_cap),
                       out.ctypes.data_as(C.POINTER(C.c_int32)))
    if n < 0:
        return None
    if shape:
        return code[:n].copy(), consts[:out[1]].copy(), int(out[2]), int(out[3]), int(out[4]), int(out[5])
    return code[:n].copy(), consts[:out[1]].copy(), int(out[2]), int(out[3])


def run(cases_blob, local_types, fuel, code, consts, n_locals, case):
    """(ok, value, tag, steps) of one case."""
    lib = library()
    code = np.ascontiguousarray(code, dtype=np.int32)
    consts = np.ascontiguousarray(consts, dtype=np.int64)
    lt = _i32(list(local_types) + [9] * (64 - len(local_types)))
    value, tag, steps = C.c_int64(), C.c_int32(), C.c_uint64()
    ok = lib.host_run(cases_blob.ref(), lt.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int(fuel),
                      code.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int(len(code)),
                      consts.ctypes.data_as(C.POINTER(C.c_int64)), C.c_int(n_locals), C.c_int(case),
                      C.byref(value), C.byref(tag), C.byref(steps))
    return bool(ok), value.value, tag.value, steps.value


def run_regions(grammar_blob, cases_blob, fuel, code, n_main, consts, main_consts, n_locals, case):
    """(ok, value, tag, steps) of one case of a program with bounded regions."""
    lib = library()
    lib.host_run_regions.restype = C.c_int
    code = np.ascontiguousarray(code, dtype=np.int32)
    consts = np.ascontiguousarray(consts, dtype=np.int64)
    value, tag, steps = C.c_int64(), C.c_int32(), C.c_uint64()
    ok = lib.host_run_regions(grammar_blob.ref(), cases_blob.ref(), C.c_int(fuel),
                              code.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int(len(code)), C.c_int(n_main),
                              consts.ctypes.data_as(C.POINTER(C.c_int64)), C.c_int(main_consts), C.c_int(n_locals),
                              C.c_int(case), C.byref(value), C.byref(tag), C.byref(steps))
    return bool(ok), value.value, tag.value, steps.value
