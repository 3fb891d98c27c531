"""List programs on the device against the reference (GPU).

Traversals over IntList inputs (forward, reverse and nested), bound reads of
their element/index/accumulator binders and len: every recorded reference
run in tests/golden/list/ -- the small list tasks, a reverse traversal and the
list-program benchmark's shape (P = 1024, 200 cases, lists of 0..50 elements,
16 generations) -- must be reproduced bit for bit by a whole device search
through the C ABI (history with champions, final ranked population with
fitness, wrong counts, node counts and rows), alone and batched with scalar
searches; and the device lowering and exact VM must score every program of
tests/golden/lower/ as the reference's CPU evaluator does."""
import gzip
import glob
import json
import os

import numpy as np
import pytest

from gagp_b200 import abi

import golden_util as GU

pytestmark = pytest.mark.gpu
NAMES = GU.list_names()
LOWER_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lower")
LOWER = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(LOWER_DIR, "*.json.gz")))


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("name", NAMES)
def test_list_search_matches_reference(engine, name):
    fx = GU.list_fixture(name)
    lt = GU.load_task(fx)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    GU.compare_result(lt, got, fx["run"], name)


def test_list_and_scalar_searches_batched_match_alone(engine):
    """List and scalar searches advanced together in one launch sequence
    give each one's reference result."""
    picks = [("list", n) for n in NAMES if not n.startswith("list_config3")] + \
        [("scalar", "poly4_genome_reservoir"), ("scalar", "poly4_exact_metric")]
    fixtures = [GU.list_fixture(n) if kind == "list" else GU.fixture(n) for kind, n in picks]
    tasks = [GU.load_task(fx) for fx in fixtures]
    searches = [engine.admit(t) for t in tasks]
    try:
        engine.run_batch(searches)
        results = [s.result() for s in searches]
    finally:
        for s in searches:
            s.close()
    for (_, n), t, r, fx in zip(picks, tasks, results, fixtures):
        GU.compare_result(t, r, fx["run"], "batched " + n)


@pytest.mark.parametrize("name", LOWER)
def test_device_row_evaluation_matches_reference(engine, name):
    with gzip.open(os.path.join(LOWER_DIR, name + ".json.gz"), "rt") as f:
        fx = json.load(f)
    lt = GU.load_task(fx)
    rows_ref = [r for r in fx["lower"]["rows"] if r["status"] == 0]
    stride = lt.tables.max_nodes - lt.tables.fixed_nodes
    rows = abi.RowsBuffer.from_rows([(r["origins"], r["constants"]) for r in rows_ref], stride)
    f, w = engine.evaluate_rows(lt, rows)
    assert list(f) == [r["fitness"] for r in rows_ref]
    assert list(w) == [r["wrong"] for r in rows_ref]
