"""A short run of the large scalar-regression search for profiler captures.

    python -m gagp_b200.profiling [--rounds R] [--population P] [--seed S]

Admits one search of the benchmark workload (degree<=4 integer polynomial,
256 cases, max 64 nodes, population 16384 by default), runs its initial
evaluation and R steady-state rounds with the L2 flushed before each round,
and prints the device milliseconds.  It launches few kernels before the
rounds, so a profiler can select a round's kernels by launch index.
"""
from __future__ import annotations

import argparse
import os
import tempfile

from gagp_b200 import build, task as T, workloads as W
from gagp_b200.engine import Engine


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rounds", type=int, default=6)
    ap.add_argument("--population", type=int, default=16384)
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    build.build()
    with tempfile.TemporaryDirectory() as d:
        files = W.poly4(population=args.population, generations=max(args.rounds, 2), seed=args.seed,
                        cases=args.cases, max_nodes=64)
        files.write(d)
        lt = T.load(os.path.join(d, "task.json"), os.path.join(d, "search.json"))
        with Engine(0) as eng:
            s = eng.admit(lt)
            eng.start([s])
            ms = eng.advance([s], args.rounds, flush_l2=True)
            print("rounds %d: %.3f ms device time" % (args.rounds, ms))
            s.close()


if __name__ == "__main__":
    main()
