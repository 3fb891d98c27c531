"""Edge shapes of the device search against the oracle (GPU): populations of
one and of odd sizes, case counts that leave partial VM tiles, a node budget
tight enough that generation and splices hit capacity, tournaments of one and
five, steady batches smaller than the population with other replacement
sizes, crossover or mutation switched off or always on, the exact metric and
the largest case count of the serving mix.  Each search must equal the
oracle's bit for bit (history, final ranked population, evaluation counts)."""
import pytest

from gagp_b200 import abi, task as T, workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    e = Engine(0)
    yield e
    e.close()


# (name, population, cases, generations, max_nodes, search-config additions, task fitness)
CASES = [
    ("population_2_one_case", 2, 1, 3, 40, {}, None),
    ("odd_population_partial_tiles", 5, 33, 5, 40, {}, None),
    ("tight_node_budget", 64, 16, 6, 8, {}, None),
    ("tournament_1", 96, 24, 4, 40, {"selection": {"method": "tournament", "size": 1}}, None),
    ("tournament_5", 96, 24, 4, 40, {"selection": {"method": "tournament", "size": 5}}, None),
    ("replacement_1_quarter_batch", 256, 20, 4, 40,
     {"schedule": {"mode": "steady_state", "batch": 64, "replacement_size": 1}}, None),
    ("replacement_3_half_batch", 256, 20, 4, 40,
     {"schedule": {"mode": "steady_state", "batch": 128, "replacement_size": 3}}, None),
    ("no_crossover", 128, 20, 4, 40, {"crossover": {"probability": 0.0, "attempts": 8}}, None),
    ("always_mutate_one_attempt", 128, 20, 4, 40,
     {"crossover": {"probability": 1.0, "attempts": 1}, "mutation": {"probability": 1.0}}, None),
    ("exact_metric", 128, 40, 4, 40, {}, {"metric": "exact", "case_cap": 1000}),
    ("largest_case_count", 64, 2000, 3, 40, {}, None),
]


@pytest.mark.parametrize("name,population,cases,generations,max_nodes,extra,fitness", CASES,
                         ids=[c[0] for c in CASES])
def test_edge_shape_matches_oracle(engine, tmp_path, name, population, cases, generations, max_nodes, extra,
                                   fitness):
    files = W.poly4(population=population, generations=generations, seed=7, cases=cases, max_nodes=max_nodes)
    files.search.update(extra)
    if fitness is not None:
        files.fitness = fitness
    lt = T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))
    want = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    assert got["history"] == want["history"], name
    assert got["final"] == want["final"], name
    assert got["evaluated_programs"] == want["evaluated_programs"], name
    assert got["reused_programs"] == want["reused_programs"], name


def test_batch_entry_points_reject_a_repeated_search(engine, tmp_path):
    """A search listed twice in one batch would have two batch members write
    its device state: every batch entry point refuses it before any launch,
    and the search still runs alone afterwards."""
    from gagp_b200.engine import EngineError
    files = W.poly4(population=64, generations=2, seed=3, cases=16, max_nodes=40)
    lt = T.load(files.write(str(tmp_path)), str(tmp_path / "search.json"))
    s = engine.admit(lt)
    try:
        for call in (lambda: engine.run_batch([s, s]), lambda: engine.step([s, s]), lambda: engine.start([s, s]),
                     lambda: engine.advance([s, s], 1)):
            with pytest.raises(EngineError) as err:
                call()
            assert err.value.status == 2 and "more than once" in str(err.value)
        s.run()
        want = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
        assert s.result()["final"] == want["final"]
    finally:
        s.close()
