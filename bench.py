#!/usr/bin/env python
"""Benchmark of the resident GAGP search path on B200.

Workloads (``--workload``):

* ``poly4`` (default): the large scalar-regression search -- a random
  degree<=4 integer polynomial, 256 train cases x ~ U{-100..100}, grammar x,
  constants -2..3, add/sub/mul/idiv0/imod0 and if(lt(E,E),E,E), max 64 nodes,
  population 16384, 128 generations, absolute error (cap 1000), gagp's
  default resident search (steady state, batch = population).
* ``list``: list programs with a loop -- IntLists of 0..50 elements in
  [-1000, 1000] and a threshold t in [-100, 100], target the sum of the
  elements above t, a traversal grammar (element/index/accumulator binders,
  comparisons, add/sub), 200 cases, population 8192, 96 generations.
* ``batch``: 64 independent searches (half scalar, half list programs) run
  as one batch, against each run alone.
* ``serve``: an open-loop Poisson stream of scalar and list search requests
  through the continuous-batching server.

For ``poly4`` and ``list`` a step is one steady-state round: one batch of
children varied, lowered, evaluated on all cases and placed.  Metric: VM
program-case evaluations per second (whole job).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload W]

Own arm: `value` is program-case evaluations per second of device time over K
rounds (CUDA events on the engine stream, L2 flushed before every round,
outside the timed region); `e2e` runs a whole search through the C ABI from
host buffers (admission upload, device loop, result download).  Reference arm
(--impl reference): the reference's own CPU engine compiled from its sources
(oracle/_ref/ref_driver) on the same task, one process per host core (as many
as host memory holds), each step the initial evaluation and the first
generation of the search, timed by the reference's own clock.  Several GPUs
run independent replica searches (one per rank, seed + rank): the path has no
data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os

# the engine's rounds run on 11 CUDA streams; more hardware work queues than
# the default 8 keep them from waiting on each other (read when the CUDA
# context is created, so before anything touches the GPU)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gagp_b200 import workloads as W  # noqa: E402
from gagp_b200 import task as T  # noqa: E402

METRIC = "VM program-case evals/s"
UNIT = "program-case evals/s"
PROFILE_ROUNDS = 3
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")

# The single-search workloads: task files from the seed, their shape and label.
SEARCH_WORKLOADS = {
    "poly4": dict(population=16384, generations=128, cases=256, max_nodes=64,
                  make=lambda seed: W.poly4(population=16384, generations=128, seed=seed, cases=256, max_nodes=64),
                  label="poly4 scalar regression (large): P=16384, G=128, C=256, max_nodes=64, seed=%d",
                  cpu_generations=4, gpu_generations=8, profile="poly4_p16384"),
    "list": dict(population=8192, generations=96, cases=200, max_nodes=48,
                 make=lambda seed: W.list_threshold(population=8192, generations=96, seed=seed, cases=200,
                                                    target="threshold_sum"),
                 label="list programs (threshold sum over IntLists of 0..50 elements, traversal grammar): "
                       "P=8192, G=96, C=200, max_nodes=48, seed=%d",
                 cpu_generations=1, gpu_generations=2, profile="list_p8192"),
}
WORKLOAD = SEARCH_WORKLOADS["poly4"]


def combine_ranks(dist, seconds: float, units: float, device: str = "cuda"):
    """Whole-job figures of a multi-rank run: the max of the ranks' times and
    the sum of their units (every rank works on its own searches; this is
    the only cross-rank exchange, outside the timed region)."""
    import torch
    t = torch.tensor([seconds, float(units)], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(tot[1])


def shard(items, rank: int, world: int):
    """The items of one rank: independent searches are split round-robin."""
    return items[rank::world]


def init_ranks(world: int, local: int):
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def make_task(seed: int, directory: str) -> str:
    return WORKLOAD["make"](seed).write(directory)


def config_block(world: int, seed: int) -> dict:
    return {"workload": WORKLOAD["label"] % seed,
            "population": WORKLOAD["population"], "generations": WORKLOAD["generations"],
            "cases": WORKLOAD["cases"], "max_nodes": WORKLOAD["max_nodes"], "batch": WORKLOAD["population"],
            "parallelism": "replicas%d" % world if world > 1 else "single-gpu",
            "l2": "256 MiB buffer written before every timed round (outside the timed region)"}


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for name, flag in zip(names, f[5:9]):
                    if flag.lower().startswith("active"):
                        reasons.add(name)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks() -> dict:
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return {"hbm_gbs": p["hbm_gbs"], "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def reference_sample(task_path: str, search_path: str, generations: int, seed=None) -> dict:
    """One reference CPU-engine search (single thread), timed by its own clock."""
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    cmd = [driver, "run", task_path, "--search", search_path, "--generations", str(generations)]
    if seed is not None:
        cmd += ["--seed", str(seed)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    d = json.loads(out)
    return {"program_cases": d["program_cases"], "ms": d["time_ms"]}


def cpu_baseline(directory: str) -> dict:
    """The reference CPU engine on a bounded sample of the workload (1 thread)."""
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    g = WORKLOAD["cpu_generations"]
    if os.path.exists(driver):
        r = reference_sample(os.path.join(directory, "task.json"), os.path.join(directory, "search.json"), g)
        return {"value": r["program_cases"] / (r["ms"] / 1000.0), "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "reference CPU engine (HostPhasePopulation, single-threaded), same task and seed, "
                          "population %d, %d generation(s) + initial evaluation (%d program-cases in %.1f s)" % (
                              WORKLOAD["population"], g, r["program_cases"], r["ms"] / 1000.0)}
    sys.path.insert(0, ROOT)
    from oracle import oracle  # noqa: WPS433 (checker only)
    from gagp_b200 import abi
    lt = T.load(os.path.join(directory, "task.json"), os.path.join(directory, "search.json"), generations=2)
    t0 = time.perf_counter()
    res = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings)
    dt = time.perf_counter() - t0
    return {"value": res["program_cases"] / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "C oracle restatement, population %d, 2 generations + initial evaluation" % WORKLOAD["population"]}


def host_memory_bytes() -> int:
    """Memory this process may use on the host: MemAvailable, capped by the
    cgroup limit when there is one."""
    avail = None
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            text = open(path).read().strip()
            if text.isdigit():
                avail = min(avail or int(text), int(text))
        except OSError:
            pass
    return avail or (8 << 30)


# resident memory of one reference CPU-engine process on each workload (its
# fixed 1024-node rows: about 4.2 GB at population 16384, 2.2 GB at 8192)
REFERENCE_PROCESS_BYTES = {"poly4": 5 << 30, "list": 3 << 30}


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "gpu", "gagp")


def reference_gpu_search(directory: str, generations=None, timeout: float = 600.0) -> dict:
    """One search of the task in `directory` by the reference's own CUDA
    engine (`gagp run --engine gpu`, the plain one-search-per-launch path),
    timed by the reference's own clock: time_ms.total is the whole
    evolve_population call (initial population, its evaluation and every
    generation), time_ms.search the part after the initial population."""
    out = os.path.join(directory, "ref_gpu_out")
    cmd = [REF_GPU, "run", os.path.join(directory, "task.json"), "--engine", "gpu", "--search",
           os.path.join(directory, "search.json"), "--out", out, "--quiet"]
    if generations:
        cmd += ["--generations", str(generations)]
    subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)
    with open(os.path.join(out, "result.json")) as f:
        r = json.load(f)
    return {"total_s": r["time_ms"]["total"] / 1000.0, "search_s": r["time_ms"]["search"] / 1000.0,
            "init_s": r["time_ms"]["initialization"] / 1000.0, "best_fitness": r["best"]["fitness"],
            "declined": r.get("resident_declined", "")}


def run_reference_gpu_arm(args, rank: int, world: int):
    """--impl reference --reference-engine gpu: the reference's own CUDA engine
    (plain path: one search per process, a host round trip per round) on the
    same single-search task, one search per step over a bounded window of
    generations.  The program-case count of that window is the reference CPU
    engine's for the identical search (same task, seed and generations),
    counted once outside the timed region."""
    if rank != 0:
        return
    if not os.path.exists(REF_GPU):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/gpu/gagp was not built (make -C oracle ref-gpu)"}))
        return
    seed, gens = 0, WORKLOAD["gpu_generations"]
    with tempfile.TemporaryDirectory() as d:
        make_task(seed, d)
        cases = reference_sample(os.path.join(d, "task.json"), os.path.join(d, "search.json"), gens)["program_cases"]
        for _ in range(args.warmup):
            reference_gpu_search(d, gens)
        runs = [reference_gpu_search(d, gens) for _ in range(args.steps)]
    secs = sum(r["total_s"] for r in runs)
    value = cases * len(runs) / secs
    line = {"impl": "reference", "engine": "reference CUDA engine (gagp run --engine gpu, sm_100a build)",
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * secs / len(runs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": dict(config_block(1, seed), generation_window="initial + %d of %d" % (gens, WORKLOAD["generations"])),
            "program_cases_per_step": cases, "best_fitness": runs[0]["best_fitness"],
            "declined": runs[0]["declined"],
            "search_s": [r["search_s"] for r in runs], "total_s": [r["total_s"] for r in runs]}
    print(json.dumps(line))


def run_reference_batch_arm(args, rank: int, world: int, serving: bool = False):
    """--impl reference --workload batch|serve: the reference's plain GPU path
    on the mix, each search alone (one `gagp run --engine gpu` process after
    another), as far as a time budget allows; searches/s from the
    reference's own clock."""
    if rank != 0:
        return
    if not os.path.exists(REF_GPU):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/gpu/gagp was not built (make -C oracle ref-gpu)"}))
        return
    mix = W.serving_mix(args.requests, seed=0) if serving else W.batch_mix(64)
    budget = args.reference_budget
    done, total_s, search_s, started = [], 0.0, 0.0, time.perf_counter()
    for m in mix:
        if time.perf_counter() - started > budget:
            break
        with tempfile.TemporaryDirectory() as d:
            W.mix_files(m).write(d)
            r = reference_gpu_search(d)
        done.append({"index": m["index"], "kind": m["kind"], "population": m["population"], "cases": m["cases"],
                     "generations": m["generations"], "total_s": r["total_s"], "declined": r["declined"]})
        total_s += r["total_s"]
        search_s += r["search_s"]
    line = {"impl": "reference", "engine": "reference CUDA engine (gagp run --engine gpu, sm_100a build), each search alone",
            "metric": "searches/s", "value": len(done) / total_s, "unit": "searches/s", "n_gpus": 1,
            "steps": len(done), "warmup": 0, "ms_per_step": 1000.0 * total_s / len(done), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": ("serving" if serving else "batching") + " mix, the first %d searches in mix order "
                                   "within a %.0f s budget" % (len(done), budget)},
            "searches": done, "kinds": {k: sum(1 for x in done if x["kind"] == k) for k in ("scalar", "list")}}
    print(json.dumps(line))


def run_reference_arm(args, rank: int, world: int):
    """--impl reference: the reference CPU engine on the host cores, same task
    and configuration as the own arm."""
    if rank != 0:
        return
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    seed = 0
    if not os.path.exists(driver):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver was not built"}))
        return
    cores = os.cpu_count() or 1
    # concurrent processes: every core, as far as host memory holds them
    procs_n = max(1, min(cores, int(0.7 * host_memory_bytes()) // REFERENCE_PROCESS_BYTES[args.workload]))
    with tempfile.TemporaryDirectory() as d:
        make_task(seed, d)
        tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
        sample_generations = 1

        def step():
            # each process: the same task with its own seed, initial
            # population, its evaluation and one generation; the step's time
            # is the slowest process's own search clock (start-up, grammar
            # load and the final JSON dump are outside it)
            procs = [subprocess.Popen([driver, "run", tp, "--search", sp, "--generations", str(sample_generations),
                                       "--seed", str(seed + i)], stdout=subprocess.PIPE, text=True)
                     for i in range(procs_n)]
            total, slowest = 0, 0.0
            for p in procs:
                out, _ = p.communicate()
                if p.returncode:
                    raise RuntimeError("reference run failed")
                r = json.loads(out)
                total += r["program_cases"]
                slowest = max(slowest, r["time_ms"] / 1000.0)
            return total, slowest

        for _ in range(args.warmup):
            step()
        cases, secs = 0, 0.0
        for _ in range(args.steps):
            c, s = step()
            cases += c
            secs += s
    value = cases / secs
    sample = ("per step: %d concurrent single-threaded reference CPU-engine searches of this task (population %d, "
              "%d cases; initial population, its evaluation and generation 1 of %d; seeds 0..%d), timed by the "
              "reference's own search clock (max over processes)" % (
                  procs_n, WORKLOAD["population"], WORKLOAD["cases"], WORKLOAD["generations"], procs_n - 1))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": dict(config_block(1, seed), generation_window="initial + 1 of %d"
                                                % WORKLOAD["generations"]),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs_n, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# Algorithmic bytes per launch of the bandwidth-bound kernels: the variation
# and lowering kernels count theirs on the device (search counters 8 and 9);
# placement reads every member key, resets and writes the placement map, and
# per child reads its key and two stream draws and writes its placement.
def algorithmic_bytes(kernel: str, delta: dict, steps: int, population: int, batch: int):
    if kernel == "k_vary":
        return delta["vary_bytes"] / steps
    if kernel == "k_lower":
        return delta["lower_bytes"] / steps
    if kernel == "k_place":
        return population * (8 + 4 + 8) + batch * (8 + 4 + 4 + 4)
    return None


def profiled_traffic(kernel: str):
    """dram bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "%s_%s.txt" % (kernel, WORKLOAD["profile"]))
    try:
        for line in open(path):
            f = line.split()
            if len(f) == 3 and f[0] == "traffic_bytes_per_launch:" and f[1] == kernel:
                return float(f[2])
    except OSError:
        pass
    return None


def roofline_entry(stats: dict, delta: dict, steps: int, peak: dict) -> dict:
    """Roofline of the kernel with the largest device time (HBM-bound)."""
    top = max(stats.items(), key=lambda kv: kv[1]["ms"])[0]
    launches = max(1, stats[top]["launches"])
    ms = stats[top]["ms"] / launches
    total = sum(v["ms"] for v in stats.values())
    per_launch = algorithmic_bytes(top, delta, launches, WORKLOAD["population"], WORKLOAD["population"])
    achieved = per_launch / (ms / 1000.0) / 1e9 if per_launch is not None else None
    return {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peak["hbm_gbs"] if achieved is not None else None,
            "traffic": profiled_traffic(top), "algorithmic_bytes_per_launch": per_launch,
            "avg_launch_ms": ms, "share": stats[top]["ms"] / max(1e-9, total),
            "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak["source"]}


def round_timeline(spans):
    """The launches of the last profiled round (each round opens with its
    member index build), as [kernel, start ms, end ms] after the round's
    first launch started, and the round's span."""
    starts = [i for i, (name, _, _) in enumerate(spans) if name == "k_member_index"]
    if not starts:
        return None
    last = spans[starts[-1]:]
    t0 = min(a for _, a, _ in last)
    return {"span_ms": max(b for _, _, b in last) - t0,
            "launches": [[name, round(a - t0, 4), round(b - t0, 4)] for name, a, b in last]}


def vm_issue_summary(workload: str):
    """Integer-issue figures of the VM kernels from the committed ncu summary
    (profiles/vm_issue_<workload>.txt): per kernel, warp instructions issued
    on the integer pipes (ALU + FMA) and in all, per launch, and the
    fraction of the SM sub-partitions' issue slots they filled."""
    path = os.path.join(ROOT, "profiles", "vm_issue_%s.txt" % workload)
    out = {}
    try:
        for line in open(path):
            f = line.split()
            if len(f) == 6 and f[0] == "vm_issue:":
                out[f[1]] = {"int_inst_per_launch": float(f[2]), "inst_per_launch": float(f[3]),
                             "int_issue_frac": float(f[4]), "issue_frac": float(f[5])}
    except OSError:
        pass
    return out


def vm_entry(stats: dict, delta: dict, clock_mhz, sm_count: int = 148) -> dict:
    """The VMs' work per second of their kernel time, and the integer-issue
    roofline: integer-pipe warp instructions per launch (ncu, committed
    summary) over the live CUDA-event launch time, against the issue peak
    (one warp instruction per cycle on each of the SMs' 4 sub-partitions)."""
    out = {}
    fast = stats.get("k_vm_fast", {"ms": 0, "launches": 0})
    exact = stats.get("k_vm_general", {"ms": 0, "launches": 0})
    if fast["ms"] > 0:
        out["fast"] = {"kernel_ms": fast["ms"], "launches": fast["launches"],
                       "accumulator_ops_per_s": delta["accumulator_ops"] / (fast["ms"] / 1000.0)}
    if exact["ms"] > 0:
        out["exact"] = {"kernel_ms": exact["ms"], "launches": exact["launches"],
                        "bytecode_instructions_per_s": delta["exact_vm_instructions"] / (exact["ms"] / 1000.0)}
    ms = fast["ms"] + exact["ms"]
    if ms > 0:
        out["program_cases_per_s"] = delta["program_cases"] / (ms / 1000.0)
    issue = vm_issue_summary(ARGS_WORKLOAD[0])
    clock = (clock_mhz or 1965.0) * 1e6
    for name, st, key in (("k_vm_fast", fast, "fast"), ("k_vm_general", exact, "exact")):
        if name in issue and st["launches"] and key in out:
            per_launch_s = st["ms"] / st["launches"] / 1000.0
            slots = sm_count * 4 * clock * per_launch_s
            out[key]["roofline"] = {
                "bound": "integer issue", "achieved_int_issue_frac": issue[name]["int_inst_per_launch"] / slots,
                "achieved_issue_frac": issue[name]["inst_per_launch"] / slots,
                "ncu_int_issue_frac": issue[name]["int_issue_frac"], "ncu_issue_frac": issue[name]["issue_frac"],
                "source": "profiles/vm_issue_%s.txt instruction counts over the live launch time at %.0f MHz"
                          % (ARGS_WORKLOAD[0], clock / 1e6)}
    return out


ARGS_WORKLOAD = ["poly4"]


def run_own_arm(args, rank: int, world: int, local: int):
    import ctypes  # noqa: F401
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    dist = init_ranks(world, local)
    build.build()
    seed = rank
    line = {}
    with tempfile.TemporaryDirectory() as d:
        make_task(seed, d)
        tp, sp = os.path.join(d, "task.json"), os.path.join(d, "search.json")
        with Engine(local if world > 1 else 0) as eng:
            # e2e: whole searches through the C ABI from host buffers (median of
            # 3; --no-e2e, for profiler captures of the timed rounds, skips it)
            runs = []
            for _ in range(0 if args.no_e2e else 3):
                lt = T.load(tp, sp)
                moved0 = eng.transfers()
                t0 = time.perf_counter()
                s = eng.admit(lt)
                t_admit = time.perf_counter()
                s.run()
                t_run = time.perf_counter()
                res = s.result_buffer()
                secs = time.perf_counter() - t0
                moved1 = eng.transfers()
                runs.append({"seconds": secs, "program_cases": int(res.struct.program_cases),
                             "parts": {"admit_s": t_admit - t0, "run_s": t_run - t_admit, "result_s": secs - (t_run - t0)},
                             "h2d": moved1[0] - moved0[0], "d2h": moved1[1] - moved0[1],
                             "place_levels": eng.counters(s).get("place_levels")})
                s.close()
            runs.sort(key=lambda r: r["seconds"])
            mid = runs[1] if runs else None
            e2e = None if mid is None else {"value": mid["program_cases"] / mid["seconds"], "unit": UNIT,
                   "h2d_bytes_per_step": mid["h2d"], "d2h_bytes_per_step": mid["d2h"], "seconds": mid["seconds"],
                   "step": "one whole search (admission + %d rounds + result); median of 3" % WORKLOAD["generations"],
                   "all_seconds": [r["seconds"] for r in runs], "parts": mid["parts"],
                   "place_levels": mid["place_levels"]}
            # device-timed rounds
            lt = T.load(tp, sp)
            s = eng.admit(lt)
            eng.start([s])
            eng.advance([s], args.warmup, flush_l2=True)
            before = eng.counters(s)
            if dist:
                import torch
                dist.barrier()
                torch.cuda.synchronize()
            with ClockSampler(local) as clocks:
                ms = eng.advance([s], args.steps, flush_l2=True)
            after = eng.counters(s)
            # per-kernel CUDA-event durations: PROFILE_ROUNDS further rounds of
            # the same search right after the timed region (timing each launch
            # needs direct launches, which the timed rounds avoid)
            eng.profile(True)
            eng.advance([s], PROFILE_ROUNDS, flush_l2=True)
            stats = eng.kernel_stats()
            timeline = round_timeline(eng.timeline())
            eng.profile(False)
            profiled = eng.counters(s)
            s.close()
    cases = after["program_cases"] - before["program_cases"]
    secs = ms / 1000.0
    if dist:
        secs, cases = combine_ranks(dist, secs, cases)
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    launches = sum(v["launches"] for v in stats.values()) * args.steps // PROFILE_ROUNDS
    clock_summary = clocks.summary()
    delta = {k: after[k] - before[k] for k in after if isinstance(after[k], int)}
    pdelta = {k: profiled[k] - after[k] for k in after if isinstance(after[k], int)}
    line = {"metric": METRIC, "value": cases / secs, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": config_block(world, seed), "e2e": e2e, "gpu_launches": launches,
            "kernels": {k: {"ms_per_step": v["ms"] / PROFILE_ROUNDS, "launches_per_step": v["launches"] / PROFILE_ROUNDS}
                        for k, v in stats.items()},
            "kernel_timing": "CUDA events per launch over %d profiled rounds right after the timed region" % PROFILE_ROUNDS,
            "round_timeline": timeline,
            "roofline": roofline_entry(stats, pdelta, PROFILE_ROUNDS, peaks()), "clocks": clock_summary,
            "counters": {"program_cases": cases, "evaluated_programs": after["evaluated_programs"] - before["evaluated_programs"],
                         "reused_programs": after["reused_programs"] - before["reused_programs"],
                         "accumulator_ops": after["accumulator_ops"] - before["accumulator_ops"],
                         "exact_vm_instructions": after["exact_vm_instructions"] - before["exact_vm_instructions"],
                         "place_cycles_per_step": {k: (after[k] - before[k]) / args.steps for k in
                                                   ("place_generate_cycles", "place_stage_cycles",
                                                    "place_serial_cycles", "place_levels", "place_level_cycles")},
                         # the variation kernel's per-child statistics are
                         # collected in the profiled rounds only
                         "vary_stats_rounds": PROFILE_ROUNDS,
                         "vary_cycles_per_child": {k: pdelta[k] / max(1, PROFILE_ROUNDS * WORKLOAD["population"])
                                                   for k in ("vary_select_cycles", "vary_crossover_cycles",
                                                             "vary_generate_cycles", "vary_rest_cycles")},
                         "vary_max_child_cycles": profiled["vary_max_child_cycles"],
                         "vary_max_phase_cycles": profiled["vary_max_phase_cycles"],
                         "vary_slow_children_per_step": pdelta["vary_slow_children"] / PROFILE_ROUNDS,
                         "generate_steps_per_generation": pdelta["generate_steps"] / max(1, pdelta["generations"]),
                         "generations_per_step": pdelta["generations"] / PROFILE_ROUNDS,
                         "generate_max_steps": profiled["generate_max_steps"]}}
    line["vm"] = vm_entry(stats, pdelta, clock_summary.get("sm_mhz"))
    if world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as d:
            make_task(seed, d)
            line["cpu_baseline"] = cpu_baseline(d)
    print(json.dumps(line))


def _mix_tasks(entries):
    """The loaded tasks of the mix entries this engine admits, and how many
    it declined at admission (none of the scalar and list tasks of the
    mixes is outside the resident subset)."""
    from gagp_b200 import grammar as G
    cache, tasks, declined = {}, [], 0
    for m in entries:
        try:
            tasks.append(T.from_files(W.mix_files(m), cache))
        except G.Declined:
            declined += 1
    return tasks, declined


def run_batch_workload(args, rank: int, world: int):
    """Batching: 64 independent searches, half scalar regressions and half
    list programs (populations log-uniform 256..8192, 16..1000 cases, 64
    generations, seeds 0..63) run as one batch (one launch sequence per
    round, rounds replayed from a CUDA graph) against the plain path (each
    search alone, one after another)."""
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    dist = init_ranks(world, rank_info()[2])
    build.build()
    mix = W.batch_mix(64)
    tasks, declined = _mix_tasks(shard(mix, rank, world))
    with Engine(rank_info()[2] if world > 1 else 0) as eng:
        # warm-up: driver and modules (two searches run), and the engine's
        # memory pool grown to the batch's size (every search admitted and
        # released unrun), so that the timed admissions reuse pool memory
        warm = [eng.admit(lt) for lt in tasks]
        eng.run_batch(warm[:2])
        for s in warm:
            s.close()
        # batched: admission, the batch, results
        t0 = time.perf_counter()
        searches = [eng.admit(lt) for lt in tasks]
        t1 = time.perf_counter()
        eng.run_batch(searches)
        t2 = time.perf_counter()
        cases = sum(int(s.result_buffer().struct.program_cases) for s in searches)
        t3 = time.perf_counter()
        for s in searches:
            s.close()
        # plain: one search at a time through the same engine
        p0 = time.perf_counter()
        plain_run = 0.0
        for lt in tasks:
            s = eng.admit(lt)
            r0 = time.perf_counter()
            s.run()
            plain_run += time.perf_counter() - r0
            s.result_buffer()
            s.close()
        p1 = time.perf_counter()
    n = len(tasks)
    batch_s, e2e_s = t2 - t1, t3 - t0
    if dist:
        batch_s, n = combine_ranks(dist, batch_s, n)
        e2e_s, _ = combine_ranks(dist, e2e_s, 0)
        plain_run, _ = combine_ranks(dist, plain_run, 0)
        dist.barrier()
        dist.destroy_process_group()
    line = {"metric": "searches/s", "value": n / batch_s, "unit": "searches/s", "n_gpus": world, "steps": 1,
            "warmup": 1, "ms_per_step": 1000.0 * (t2 - t1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "batch of a 64-search mix, half scalar regressions and half list programs "
                                   "(populations log-uniform 256..8192, 16..1000 cases, 64 generations, seeds 0..63)",
                       "searches": int(n), "declined_list_searches": declined,
                       "parallelism": "searches sharded round-robin over %d GPUs" % world if world > 1 else "single-gpu"},
            "e2e": {"value": n / e2e_s, "unit": "searches/s", "seconds": e2e_s},
            "program_cases_per_s_rank0": cases / (t2 - t1),
            "plain": {"searches_per_s": n / plain_run, "e2e_searches_per_s_rank0": len(tasks) / (p1 - p0),
                      "step": "each search alone, one after another, same engine"},
            "speedup_vs_plain": plain_run / batch_s}
    if rank == 0:
        print(json.dumps(line))


def run_serve_workload(args, rank: int, world: int):
    """Serving: an open-loop Poisson stream of the requests of a serving mix
    (half scalar regressions, half list programs; populations log-uniform
    256..16384, 16..2000 cases, 32..128 generations) through the
    continuous-batching server; searches/s and p50/p99 time-to-result against
    the plain path."""
    import random
    from gagp_b200 import build
    from gagp_b200.engine import Engine, Server
    build.build()
    mix = W.serving_mix(args.requests, seed=0)
    tasks, declined = _mix_tasks(mix)
    rng = random.Random(12345)
    arrivals, t = [], 0.0
    for _ in tasks:
        t += rng.expovariate(args.rate)
        arrivals.append(t)
    n = len(tasks)
    with Engine(0) as eng:
        warm = [eng.admit(lt) for lt in tasks[:2]]
        eng.run_batch(warm)
        for s in warm:
            s.close()
        latencies, evals = [], 0
        with Server(eng, rounds_per_step=args.rounds_per_step) as server:
            outstanding = {}
            nxt, done = 0, 0
            t0 = time.perf_counter()
            peak_running = 0
            while done < n:
                now = time.perf_counter() - t0
                while nxt < n and arrivals[nxt] <= now:
                    outstanding[server.submit(tasks[nxt])] = nxt
                    nxt += 1
                if not outstanding:
                    time.sleep(max(0.0, arrivals[nxt] - now))
                    continue
                running, queued, finished = server.step()
                peak_running = max(peak_running, running)
                if finished:
                    for ticket in list(outstanding):
                        if server.poll(ticket) >= 2:
                            sub, _adm, fin = server.times(ticket)
                            latencies.append(fin - sub)
                            evals += int(server.result_buffer(ticket).struct.program_cases)
                            del outstanding[ticket]
                            done += 1
            makespan = time.perf_counter() - t0
        # plain path: a sample of the requests, each alone
        sample = tasks[:: max(1, n // 16)][:16]
        plain_s, plain_evals = 0.0, 0
        for lt in sample:
            s = eng.admit(lt)
            r0 = time.perf_counter()
            s.run()
            plain_s += time.perf_counter() - r0
            plain_evals += int(s.result_buffer().struct.program_cases)
            s.close()
    latencies.sort()
    pct = lambda q: latencies[min(len(latencies) - 1, int(q * len(latencies)))]
    plain_rate = len(sample) / plain_s
    # the plain path under the same arrivals: one search at a time, FIFO, each
    # taking its work at the sample's measured program-case rate
    per_eval = plain_s / max(1, plain_evals)
    work = [lt.settings.population * lt.settings.generations * lt.cases.expected.shape[0] for lt in tasks]
    scale = plain_evals / max(1, sum(work[i] for i in range(0, n, max(1, n // 16))[:16]))
    clock, plain_lat = 0.0, []
    for a, w in zip(arrivals, work):
        clock = max(clock, a) + w * scale * per_eval
        plain_lat.append(clock - a)
    plain_lat.sort()
    ppct = lambda q: plain_lat[min(len(plain_lat) - 1, int(q * len(plain_lat)))]
    line = {"metric": "searches/s", "value": n / makespan, "unit": "searches/s", "n_gpus": 1, "steps": n,
            "warmup": 1, "ms_per_step": 1000.0 * makespan / n, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "open-loop Poisson stream of a %d-request serving mix, scalar regressions and "
                                   "list programs (populations log-uniform 256..16384, 16..2000 cases, 32..128 "
                                   "generations)" % args.requests,
                       "requests": n, "declined_list_requests": declined, "arrival_rate_per_s": args.rate,
                       "rounds_per_step": args.rounds_per_step,
                       "parallelism": "single-gpu"},
            "latency_s": {"p50": pct(0.5), "p99": pct(0.99), "max": latencies[-1]},
            "program_cases_per_s": evals / makespan, "peak_running": peak_running,
            "plain": {"searches_per_s": plain_rate, "sample": len(sample),
                      "latency_s_fifo_model": {"p50": ppct(0.5), "p99": ppct(0.99)},
                      "step": "each search alone through the same engine; latency from a FIFO model of the same "
                              "arrivals at the sample's measured rate"}}
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the whole-search e2e leg (profiler captures)")
    ap.add_argument("--workload", default="poly4", choices=["poly4", "list", "batch", "serve"],
                    help="poly4: the large scalar search (default); list: the list-program search; "
                         "batch: 64-search batching mix; serve: open-loop serving stream")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the mix")
    ap.add_argument("--rate", type=float, default=100.0, help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--rounds-per-step", type=int, default=8,
                    help="serve: rounds each server step runs before reading the searches' states")
    ap.add_argument("--reference-engine", default="cpu", choices=["cpu", "gpu"],
                    help="--impl reference on poly4/list: the reference CPU engine (default) or its CUDA engine")
    ap.add_argument("--reference-budget", type=float, default=240.0,
                    help="--impl reference on batch/serve: seconds of reference searches to run")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global WORKLOAD
    if args.workload in SEARCH_WORKLOADS:
        WORKLOAD = SEARCH_WORKLOADS[args.workload]
        ARGS_WORKLOAD[0] = args.workload
    if args.steps + args.warmup + PROFILE_ROUNDS > WORKLOAD["generations"]:
        raise SystemExit("steps + warmup + %d profiled rounds must not exceed the search's %d rounds"
                         % (PROFILE_ROUNDS, WORKLOAD["generations"]))
    rank, world, local = rank_info()
    if args.workload == "batch" and args.impl != "reference":
        run_batch_workload(args, rank, world)
        return
    if args.workload == "serve" and args.impl != "reference":
        run_serve_workload(args, rank, world)
        return
    if args.impl == "reference":
        if args.workload in ("batch", "serve"):
            run_reference_batch_arm(args, rank, world, serving=args.workload == "serve")
        elif args.reference_engine == "gpu":
            run_reference_gpu_arm(args, rank, world)
        else:
            run_reference_arm(args, rank, world)
    else:
        run_own_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
