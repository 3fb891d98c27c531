"""The generational schedule with elites on the device against the reference
(GPU).

tests/golden/generational/ holds whole reference CPU-engine searches under
schedule.mode generational (run_phase_population,
cpp/src/evolution/evolve.cpp:253-322, with HostPhasePopulation::reproduce and
evaluate, phase_population_cpu.cpp:243-312): elites 0..4, tournaments of 2
and 3, the absolute and the exact metric, scalar and list programs, and a
population of 4096 (the variation split into ranges).  Each device search
must reproduce the history, the final ranked population and the evaluation
counters bit for bit."""
import glob
import gzip
import json
import os

import pytest

import golden_util as GU

pytestmark = pytest.mark.gpu
GEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "generational")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(GEN_DIR, "*.json.gz")))


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with Engine(0) as e:
        yield e


def _fixture(name):
    with gzip.open(os.path.join(GEN_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


@pytest.mark.parametrize("name", NAMES)
def test_generational_search_matches_reference(engine, name):
    fx = _fixture(name)
    lt = GU.load_task(fx)
    assert not lt.settings.steady_state
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    GU.compare_result(lt, got, fx["run"], name)


def test_generational_batch_matches_alone(engine):
    """Generational searches batched together give each one's own result;
    a batch mixing schedules is refused."""
    from gagp_b200.engine import EngineError
    picks = [n for n in NAMES if n != "gen_poly4_p4096"][:3]
    fixtures = [_fixture(n) for n in picks]
    tasks = [GU.load_task(fx) for fx in fixtures]
    searches = [engine.admit(t) for t in tasks]
    try:
        engine.run_batch(searches)
        for n, t, s, fx in zip(picks, tasks, searches, fixtures):
            GU.compare_result(t, s.result(), fx["run"], "batched " + n)
    finally:
        for s in searches:
            s.close()
    steady = GU.load_task(GU.fixture(GU.names()[0]))
    mixed = [engine.admit(tasks[0]), engine.admit(steady)]
    try:
        with pytest.raises(EngineError):
            engine.run_batch(mixed)
    finally:
        for s in mixed:
            s.close()
