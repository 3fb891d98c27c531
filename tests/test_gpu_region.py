"""Bounded regions on the device against the reference (GPU).

Every recorded reference run in tests/golden/region/ (the lattice-path
workload: a memoized coordinate recurrence with evolved phases) must be
reproduced bit for bit by a whole device search through the C ABI --
history with champions, final ranked population, evaluation counters --
alone and batched with a scalar search.  The device row evaluation of the
region programs of tests/golden/lower/lower_grid_paths is checked with the
other lowering pins in test_gpu_list.py."""
import glob
import gzip
import json
import os

import pytest

import golden_util as GU

pytestmark = pytest.mark.gpu
REGION_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "region")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(REGION_DIR, "*.json.gz")))


def _fixture(name):
    with gzip.open(os.path.join(REGION_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with Engine(0) as e:
        yield e


@pytest.mark.parametrize("name", NAMES)
def test_region_search_matches_reference(engine, name):
    fx = _fixture(name)
    lt = GU.load_task(fx)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    GU.compare_result(lt, got, fx["run"], name)


def test_region_and_scalar_searches_batched_match_alone(engine):
    fixtures = [_fixture(NAMES[0]), GU.fixture("poly4_exact_metric")]
    tasks = [GU.load_task(fx) for fx in fixtures]
    searches = [engine.admit(t) for t in tasks]
    try:
        engine.run_batch(searches)
        for s, t, fx in zip(searches, tasks, fixtures):
            GU.compare_result(t, s.result(), fx["run"], fx["name"])
    finally:
        for s in searches:
            s.close()
