"""A short run of a benchmark search for profiler captures.

    python -m gagp_b200.profiling [--workload poly4|list] [--rounds R] [--population P] [--cases C] [--seed S]

Admits one search of a benchmark workload -- the large scalar regression
(degree<=4 integer polynomial, 256 cases, max 64 nodes, population 16384 by
default) or the list programs (threshold sum over IntLists of 0..50
elements, 200 cases, population 8192 by default) -- runs its initial
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
    ap.add_argument("--workload", default="poly4", choices=["poly4", "list"])
    ap.add_argument("--rounds", type=int, default=6)
    ap.add_argument("--population", type=int, default=0)
    ap.add_argument("--cases", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    build.build()
    with tempfile.TemporaryDirectory() as d:
        if args.workload == "list":
            files = W.list_threshold(population=args.population or 8192, generations=max(args.rounds, 2),
                                     seed=args.seed, cases=args.cases or 200, target="threshold_sum")
        else:
            files = W.poly4(population=args.population or 16384, generations=max(args.rounds, 2), seed=args.seed,
                            cases=args.cases or 256, max_nodes=64)
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
