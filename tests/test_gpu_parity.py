"""Device engine parity (GPU): whole searches through the C ABI are bit-identical
to the reference CPU engine's golden runs and to the oracle, alone and batched."""
import pytest

from gagp_b200 import abi, workloads as W
from oracle import oracle

import golden_util as GU

pytestmark = pytest.mark.gpu
NAMES = GU.names()


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("name", NAMES)
def test_search_matches_reference(engine, name):
    fx = GU.fixture(name)
    lt = GU.load_task(fx)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    GU.compare_result(lt, got, fx["run"], name)


def test_batched_searches_match_alone(engine):
    """Searches advanced together in one launch sequence give each alone's result."""
    names = [n for n in NAMES][:6]
    tasks = [GU.load_task(GU.fixture(n)) for n in names]
    searches = [engine.admit(t) for t in tasks]
    try:
        engine.run_batch(searches)
        results = [s.result() for s in searches]
    finally:
        for s in searches:
            s.close()
    for n, t, r in zip(names, tasks, results):
        GU.compare_result(t, r, GU.fixture(n)["run"], "batched " + n)


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_search_matches_oracle_fresh_seeds(engine, seed, tmp_path):
    files = W.poly4(population=384, generations=6, seed=seed, cases=300)
    from gagp_b200 import task as T
    lt = T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))
    want = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
    s = engine.admit(lt)
    s.run()
    got = s.result()
    s.close()
    assert got["history"] == want["history"]
    assert got["final"] == want["final"]
    assert got["evaluated_programs"] == want["evaluated_programs"]
    assert got["reused_programs"] == want["reused_programs"]


def test_result_part_and_wider_rows(engine, tmp_path):
    """Reading back only the best part of the ranked population, into rows
    wider than the engine's, gives the first rows of the full read-back (the
    population is ranked and put in transport form on the device)."""
    from gagp_b200 import task as T
    from gagp_b200.engine import _check, load_library
    files = W.poly4(population=300, generations=4, seed=21, cases=40, max_nodes=40)
    lt = T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))
    s = engine.admit(lt)
    try:
        s.run()
        full = s.result()
        width = lt.tables.max_nodes - lt.tables.fixed_nodes
        part = abi.ResultBuffer(lt.settings.generations, 100, width + 7)
        part.final_rows.origins[:] = -1
        _check(load_library().gagp_b200_search_result(engine.handle, s.id, part.ref()))
        again = s.result()
    finally:
        s.close()
    got = part.summary()
    assert got["history"] == full["history"]
    assert len(got["final"]) == 100
    assert got["final"] == full["final"][:100]
    assert again == full
    # entries past a row's counts are zero up to the engine's row width (the
    # node budget rounded up to 4 slots) and untouched beyond it
    engine_width = (width + 3) // 4 * 4
    rows = part.final_rows
    for i in range(100):
        n = int(rows.node_counts[i])
        assert (rows.origins[i, n:engine_width] == 0).all()
        assert (rows.origins[i, engine_width:] == -1).all()


@pytest.mark.parametrize("population,seed", [(4096, 31), (8192, 32)])
def test_cluster_placement_matches_oracle(engine, tmp_path, population, seed):
    """Rounds of 4096 children or more are placed by the cluster kernels (the
    placement levels found from the draws on the side stream, then applied
    level by level): the search equals the oracle's."""
    from gagp_b200 import task as T
    files = W.poly4(population=population, generations=3, seed=seed, cases=24, max_nodes=40)
    lt = T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))
    want = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
        levels = engine.counters(s)["place_levels"]
    finally:
        s.close()
    assert got["history"] == want["history"]
    assert got["final"] == want["final"]
    assert got["evaluated_programs"] == want["evaluated_programs"]
    assert levels > 0


def test_cluster_placement_batched_matches_oracle(engine, tmp_path):
    """Two searches of 4096 children per round advanced as one batch (a level
    cluster and a placement cluster each) equal the oracle's searches."""
    from gagp_b200 import task as T
    tasks, wants = [], []
    for k, seed in enumerate((41, 42)):
        d = tmp_path / str(k)
        files = W.poly4(population=4096, generations=2, seed=seed, cases=20, max_nodes=40)
        lt = T.load(files.write(str(d)), str(d / "search.json"))
        tasks.append(lt)
        wants.append(oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings))
    searches = [engine.admit(t) for t in tasks]
    try:
        engine.run_batch(searches)
        results = [s.result() for s in searches]
    finally:
        for s in searches:
            s.close()
    for got, want in zip(results, wants):
        assert got["history"] == want["history"]
        assert got["final"] == want["final"]
