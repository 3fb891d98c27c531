"""Host side of test-split judging (CPU): the judgement fixtures load with
their test split, the verdict struct matches the header, and a verdict
summarises as the reference's judge object does (cpp/src/cli/run.cpp:232-237)."""
import ctypes as C
import glob
import gzip
import json
import os

import golden_util as GU
from gagp_b200 import abi

JUDGE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "judge")


def test_judge_fixtures_load_with_test_split():
    paths = sorted(glob.glob(os.path.join(JUDGE_DIR, "*.json.gz")))
    assert len(paths) >= 7
    for p in paths:
        with gzip.open(p, "rt") as f:
            fx = json.load(f)
        lt = GU.load_task(fx)
        assert lt.test_cases is not None, p
        assert lt.test_cases.struct.case_count == len(fx["test"]), p
        if "rows" in fx:
            assert fx["rows"], p
            for r in fx["rows"]:
                v = r["verdict"]
                assert v["correct"] + v["wrong"] == v["cases"] == len(fx["test"])


def test_judge_fixtures_cover_errors_and_metrics():
    seen_errors, metrics, tags = 0, set(), set()
    for p in glob.glob(os.path.join(JUDGE_DIR, "judge_*.json.gz")):
        with gzip.open(p, "rt") as f:
            fx = json.load(f)
        metrics.add(fx["task"]["fitness"]["metric"])
        tags.add(fx["test"][0]["expected"]["type"])
        seen_errors += sum(1 for r in fx.get("rows", []) if r["verdict"]["runtime_errors"])
    assert seen_errors > 0
    assert metrics == {"absolute", "exact"}
    assert tags == {"int", "bool"}


def test_verdict_layout_and_summary():
    assert C.sizeof(abi.Verdict) == 24
    v = abi.Verdict(cases=40, correct=37, runtime_errors=2, reserved=0, loss=23.0)
    s = v.summary()
    assert s == {"cases": 40.0, "correct": 37.0, "wrong": 3.0, "runtime_errors": 2.0, "mean_loss": 23.0 / 40.0,
                 "solved": False}
    assert abi.Verdict(cases=5, correct=5, runtime_errors=0, reserved=0, loss=0.0).summary()["solved"]
