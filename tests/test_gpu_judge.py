"""Test-split judging on the device against the reference (GPU).

tests/golden/judge/ holds, for generated programs of six tasks (int64 edge
values with a `mod` that fails on 0, the polynomial task, list programs, Bool
programs under the absolute and the exact metric, and the large scalar
grammar under the exact metric), the reference's own verdict on the task's
test split: `gagp eval TASK PROGRAM --split test` (cases, correct, wrong,
runtime errors, mean loss, solved; cpp/src/cli/run.cpp:176-238).  Every
verdict of gagp_b200_judge_rows must equal it.  The run fixture adds one
whole `gagp run` with a test split: the device search's best program, judged
on the device, must give the verdict the reference's run reports under
"test"."""
import glob
import gzip
import json
import os

import pytest

import golden_util as GU
from gagp_b200 import abi

pytestmark = pytest.mark.gpu
JUDGE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "judge")
NAMES = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(JUDGE_DIR, "judge_*.json.gz"))
               if not os.path.basename(p).startswith("judge_run_"))
RUNS = sorted(os.path.basename(p)[:-len(".json.gz")] for p in glob.glob(os.path.join(JUDGE_DIR, "judge_run_*.json.gz")))


def _fixture(name):
    with gzip.open(os.path.join(JUDGE_DIR, name + ".json.gz"), "rt") as f:
        return json.load(f)


@pytest.fixture(scope="module")
def engine():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with Engine(0) as e:
        yield e


@pytest.mark.parametrize("name", NAMES)
def test_program_verdicts_match_reference(engine, name):
    fx = _fixture(name)
    lt = GU.load_task(fx)
    stride = lt.tables.max_nodes - lt.tables.fixed_nodes
    rows = abi.RowsBuffer.from_rows([(r["origins"], r["constants"]) for r in fx["rows"]], stride)
    got = engine.judge_rows(lt, rows)
    assert len(got) == len(fx["rows"])
    for i, (a, r) in enumerate(zip(got, fx["rows"])):
        b = r["verdict"]
        assert a["cases"] == b["cases"], (name, i)
        assert a["correct"] == b["correct"], (name, i, a, b)
        assert a["wrong"] == b["wrong"], (name, i, a, b)
        assert a["runtime_errors"] == b["runtime_errors"], (name, i, a, b)
        assert a["mean_loss"] == b["mean_loss"], (name, i, a, b)
        assert a["solved"] == b["solved"], (name, i, a, b)


@pytest.mark.parametrize("name", RUNS)
def test_best_program_verdict_matches_reference_run(engine, name):
    fx = _fixture(name)
    lt = GU.load_task(fx)
    s = engine.admit(lt)
    try:
        s.run()
        got = s.result()
    finally:
        s.close()
    assert got["final"][0]["fitness"] == fx["best"]["fitness"]
    assert got["final"][0]["wrong"] == fx["best"]["wrong"]
    verdict = engine.judge_best(lt, got)
    want = fx["test_verdict"]
    for k in ("cases", "correct", "wrong", "runtime_errors", "mean_loss", "solved"):
        assert verdict[k] == want[k], (k, verdict, want)
