"""Result reuse against the reference CPU engine (CPU).

The reference's resident owner lets a child reuse a completed result when it
equals its parent (compare_child) and otherwise when it equals any current
member (the member_hashes lookup, phase_population_cpu.cpp:318-344).  The
oracle restates both (``member_reuse=True``); its evaluation counters then
equal the reference's for a whole search, and one make_batch reuses exactly
where the reference's does.
"""
import json
import os
import subprocess

import pytest

from gagp_b200 import abi, task as T, workloads as W
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER),
                                reason="the reference CPU engine is not built (make -C oracle ref)")


def _driver(*args) -> dict:
    return json.loads(subprocess.run([DRIVER, *args], check=True, capture_output=True, text=True, timeout=300).stdout)


@pytest.mark.parametrize("population,generations,seed", [(256, 6, 1), (512, 4, 2)])
def test_member_reuse_counters_match_reference(tmp_path, population, generations, seed):
    files = W.poly4(population=population, generations=generations, seed=seed, cases=48)
    task = files.write(str(tmp_path))
    search = str(tmp_path / "search.json")
    ref = _driver("run", task, "--search", search)
    lt = T.load(task, search)
    got = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings, member_reuse=True)
    assert got["program_cases"] == ref["program_cases"]
    assert got["reused_programs"] == ref["reused_programs"]
    # parent-only reuse evaluates more programs for the same search and result
    plain = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings)
    assert plain["history"] == got["history"] and plain["final"] == got["final"]
    assert plain["evaluated_programs"] >= got["evaluated_programs"]


def test_make_batch_reuse_matches_reference(tmp_path):
    files = W.poly4(population=128, generations=2, seed=3, cases=10)
    task = files.write(str(tmp_path))
    search = str(tmp_path / "search.json")
    round_seed = 123456789
    ref = _driver("batch", task, "--search", search, "--round-seed", str(round_seed))
    lt = T.load(task, search)
    P = lt.settings.population
    selection = [float((i * 7919) % P + 1) for i in range(P)]
    rows, reuse = oracle.make_batch(abi.GrammarBlob(lt.tables), lt.settings, selection, round_seed)
    for b, child in enumerate(ref["children"]):
        origins, constants = rows.row(b)
        assert list(origins) == child["origins"], b
        assert list(constants) == [c[1] for c in child["constants"]], b
        assert (reuse[b] >= 0) == (ref["reuse"][b] >= 0), b
    assert sum(1 for r in reuse if r >= 0) > 0
