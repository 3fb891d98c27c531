"""The benchmark's own search against the reference, whole (GPU).

tests/golden/headline/ holds the reference CPU engine's run of exactly the
search bench.py times by default -- the large scalar regression, population
16384, 128 generations, 256 cases, max 64 nodes, seed 0: the full history
(best fitness, mean fitness, wrong count, node count and champion program
per generation), the final ranked fitness, wrong-count and node-count
vectors of all 16384 members, the best 256 rows, a SHA-256 digest of all
16384 ranked rows, and the evaluation counters.  The device search must
reproduce all of it bit for bit."""
import gzip
import hashlib
import json
import os

import pytest

import golden_util as GU
from gagp_b200 import task as T

pytestmark = pytest.mark.gpu
PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "headline", "poly4_p16384_g128_s0.json.gz")


def test_benchmark_search_matches_reference():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with gzip.open(PATH, "rt") as f:
        fx = json.load(f)
    lt = GU.load_task(fx)
    run = fx["run"]
    assert lt.settings.population == 16384 and lt.settings.generations == 128
    with Engine(0) as eng:
        s = eng.admit(lt)
        s.run()
        got = s.result()
        s.close()
    assert got["program_cases"] == run["program_cases"]
    assert got["reused_programs"] == run["reused_programs"]
    assert len(got["history"]) == len(run["history"]) == 128
    for i, (a, b) in enumerate(zip(got["history"], run["history"])):
        assert a["best_fitness"] == b["best_fitness"], i
        assert a["mean_fitness"] == float.fromhex(b["mean_fitness"]), i
        assert (a["best_wrong"], a["best_nodes"]) == (b["best_wrong"], b["best_nodes"]), i
        assert T.program_text(lt.tables, *a["row"]) == b["text"], i
    assert [m["fitness"] for m in got["final"]] == run["final_fitness"]
    assert [m["wrong"] for m in got["final"]] == run["final_wrong"]
    assert [m["nodes"] for m in got["final"]] == run["final_nodes"]
    for i, b in enumerate(run["top"]):
        r = b["rows"][0]
        assert list(got["final"][i]["row"][0]) == r["origins"], i
        assert list(got["final"][i]["row"][1]) == [c[1] for c in r["constants"]], i
    h = hashlib.sha256()
    for m in got["final"]:
        h.update(json.dumps([[int(x) for x in m["row"][0]], [int(x) for x in m["row"][1]]],
                            separators=(",", ":")).encode())
    assert h.hexdigest() == run["row_digest"]
