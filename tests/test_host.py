"""Host-side checks that need no GPU: the C-ABI library loads and exports
every function its header declares, and admission (gagp_b200_search_bytes,
which runs on the host only) accepts the benchmark task and turns malformed
tables into errors before any kernel could read them."""
import ctypes as C
import os
import re

import pytest

from gagp_b200 import abi, build, task as T, workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gagp_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gagp_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = C.CDLL(build.build())
    names = _declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.fixture(scope="module")
def poly_task(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("poly"))
    files = W.poly4(population=256, generations=4, seed=3, cases=32, max_nodes=40)
    return T.load(files.write(d), os.path.join(d, "search.json"))


def _bytes(lt, edit=None, settings=None):
    """Status and byte count of gagp_b200_search_bytes after `edit(blob)`."""
    from gagp_b200.engine import load_library
    blob = abi.GrammarBlob(lt.tables)
    if edit:
        edit(blob)
    cfg = (settings or lt.settings).struct()
    out = C.c_uint64(0)
    st = load_library().gagp_b200_search_bytes(blob.ref(), lt.cases.ref(), C.byref(cfg), C.byref(out))
    return st, out.value


def test_admission_accepts_the_benchmark_task(poly_task):
    st, n = _bytes(poly_task)
    assert st == 0 and n > 0


def _first(blob, kind):
    return next(i for i in range(len(blob.tables.expressions)) if blob.expressions[i].kind == kind)


@pytest.mark.parametrize("case", ["production", "reference", "child", "domain", "kind", "values"])
def test_admission_rejects_malformed_tables(poly_task, case):
    def edit(blob):
        if case == "production":
            blob.productions[0].expression = len(blob.tables.expressions) + 5
        elif case == "reference":
            blob.expressions[_first(blob, W_KINDS["reference"])].target = 999
        elif case == "child":
            e = next(i for i in range(len(blob.tables.expressions))
                     if blob.expressions[i].kind == W_KINDS["operation"] and blob.expressions[i].arity > 0)
            blob.expressions[e].children[0] = -3
        elif case == "domain":
            d = blob.domains[0]
            d.integer_range, d.minimum, d.maximum = 1, 5, 2
        elif case == "kind":
            blob.expressions[0].kind = 9
        elif case == "values":
            d = blob.domains[0]
            d.integer_range, d.value_offset, d.value_count = 0, 0, 0
    st, _ = _bytes(poly_task, edit)
    assert st == 2  # GAGP_INVALID_ARGUMENT


def test_admission_declines_outside_the_resident_subset(poly_task):
    def template(blob):
        blob.expressions[_first(blob, W_KINDS["input"])].kind = 5  # an alias (template instance)
    assert _bytes(poly_task, template)[0] == 1  # GAGP_DECLINED

    def unknown_kind(blob):
        e = next(i for i in range(len(blob.tables.expressions))
                 if blob.expressions[i].kind == W_KINDS["operation"] and blob.expressions[i].arity > 0)
        blob.expressions[e].node_kind = 17  # a tree kind beyond the reference's
    assert _bytes(poly_task, unknown_kind)[0] == 1

    # a statement belongs to a Program entry's phase: in a value phase the
    # tables are malformed
    def statement(blob):
        e = next(i for i in range(len(blob.tables.expressions))
                 if blob.expressions[i].kind == W_KINDS["operation"] and blob.expressions[i].arity > 0)
        blob.expressions[e].node_kind = 9  # Assign
    assert _bytes(poly_task, statement)[0] == 2


def test_admission_of_the_generational_schedule(poly_task):
    """The generational schedule is admitted with reproduce's elite contract
    (0 <= elites < population, phase_population_cpu.cpp:271); more elites
    than the device keeps are declined."""
    s = poly_task.settings
    old = s.steady_state, s.elite_count
    try:
        s.steady_state = False
        for elites, status in ((0, 0), (1, 0), (64, 0), (65, 1), (-1, 2), (s.population, 2)):
            s.elite_count = elites
            assert _bytes(poly_task)[0] == status, elites
    finally:
        s.steady_state, s.elite_count = old


W_KINDS = {"operation": 0, "constant": 1, "reference": 3, "input": 4}


def test_admission_rejects_a_single_member_steady_state(poly_task):
    """One member: every replacement draw is the best member, which the
    steady-state loop would redraw without end; admission refuses it."""
    s = poly_task.settings
    old = s.population, s.batch
    try:
        s.population, s.batch = 1, 0
        assert _bytes(poly_task)[0] == 2  # GAGP_INVALID_ARGUMENT
    finally:
        s.population, s.batch = old


def test_list_programs_load_with_their_traversal_table():
    """The list workload (a traversal with element/index/accumulator binders
    over an IntList input) loads into resident tables: one traversal entry,
    the IntList input as a view into the list arena."""
    for target in W.LIST_TARGETS:
        files = W.list_threshold(population=64, generations=2, seed=5, cases=12, target=target)
        lt = T.from_files(files, {})
        assert [r.binders for r in lt.tables.regions] == [[0, 1, 2]]
        xs = lt.tables.input_names.index("xs")
        for c, case in enumerate(files.train):
            assert lt.cases.list_at(c, xs) == case["inputs"]["xs"]["value"]


def test_mixes_carry_list_programs():
    """Half of the batching mix and about half of the serving mix are list
    programs, built on demand with their targets' expected values."""
    mix = W.batch_mix(8)
    lists = [m for m in mix if m["kind"] == "list"]
    assert len(lists) == 4 and all(m["files"] is None for m in lists)
    files = W.mix_files(lists[0])
    assert files.grammar["inputs"] == [{"name": "xs", "type": "IntList"}, {"name": "t", "type": "Int"}]
    for case in files.train:
        xs, t = case["inputs"]["xs"]["value"], case["inputs"]["t"]["value"]
        assert 0 <= len(xs) <= 50 and -100 <= t <= 100
        assert case["expected"]["value"] == W.list_target(lists[0]["args"]["target"], xs, t)
    kinds = [m["kind"] for m in W.serving_mix(200, seed=0)]
    assert 70 < kinds.count("list") < 130


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver")),
                    reason="the reference CPU engine is not built (make -C oracle ref)")
def test_reference_runs_list_programs_resident(tmp_path):
    """The reference engine admits the same list task to its resident path
    (no decline) and searches it."""
    import json
    import subprocess
    files = W.list_threshold(population=64, generations=2, seed=5, cases=12)
    task = files.write(str(tmp_path))
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_driver"), "run", task, "--search",
                          str(tmp_path / "search.json"), "--generations", "2"],
                         check=True, capture_output=True, text=True, timeout=120).stdout
    run = json.loads(out)
    assert run["declined"] == ""
    assert len(run["history"]) == 2 and run["program_cases"] > 0
    assert run["history"][0]["text"].startswith("(traverse xs")


def test_bench_mix_admission_counts():
    """bench.py's batching and serving workloads admit every entry of their
    mixes, scalar and list programs alike."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    mix = W.batch_mix(8)
    tasks, declined = bench._mix_tasks(mix)
    assert len(tasks) == 8 and declined == 0
    assert [t.settings.population for t in tasks] == [m["population"] for m in mix]
    assert sum(1 for t in tasks if t.tables.regions) == 4


@pytest.fixture
def list_task(tmp_path):
    files = W.list_threshold(population=64, generations=2, seed=3, cases=20)
    return T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))


def test_admission_accepts_list_programs(list_task):
    """Traversals, bound reads, scoped nonterminals and IntList inputs are
    admitted; the traversal table is uploaded with the grammar."""
    st, n = _bytes(list_task)
    assert st == 0 and n > 0
    assert len(list_task.tables.regions) == 1 and list_task.tables.regions[0].traversal == 1


@pytest.mark.parametrize("case", ["ranged", "fuel_profile", "binder", "overrun", "tags"])
def test_admission_checks_list_tables_and_cases(list_task, case):
    cases = list_task.cases

    def edit(blob):
        r = blob.regions[0]
        if case == "ranged":
            r.ranged = 1
        elif case == "fuel_profile":
            r.fuel_profile = 1
        elif case == "binder":
            r.binders[1] = 16
    saved = cases.inputs.copy(), cases.input_tags.copy()
    try:
        xs = list_task.tables.input_names.index("xs")
        if case == "overrun":
            cases.inputs[0, xs] = len(cases.list_values) - 1  # a length word with no room for its elements
            cases.list_values[-1] = 5
        if case == "tags":
            cases.input_tags[xs] = 0
        st, _ = _bytes(list_task, edit)
    finally:
        cases.inputs[:], cases.input_tags[:] = saved
    assert st == (1 if case in ("ranged", "fuel_profile") else 2), case
