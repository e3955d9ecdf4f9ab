#!/usr/bin/env python3
"""DCFR solve benchmark on B200.

Workload (default, --workload flop): the flop full tree Ks7s2d, pot 6bb,
stacks 97bb, 33%/75%/all-in bets and one 3x raise on every street, ranges
from a 169-class Dirichlet(0.5) thresholded to 68 classes (seeds 2000/2001),
f32 storage, suit isomorphism, DCFR alpha 1.5 beta 0 gamma 2. The metric is
the time to 0.5%-of-the-pot exploitability (seconds, lower is better): one
solve from a fresh solver with exploitability checks on the reference's
schedule, the final value re-checked by the FP64 best-response oracle. The
line also carries the turn subgame's DCFR iterations per second.
--workload turn | turn-narrow | river | batch | learned measure the other
configurations (iterations or spot-iterations per second).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs as one process per GPU (torchrun): every rank solves its own copy
of the spot (independent replicas, no collective on the data path; the
batched spots are partitioned across ranks instead); the timed region is
bracketed by a barrier and a device synchronize on every rank, and the job
time is the maximum over ranks.

--impl reference times the CPU restatement of the reference's solver (the
C++ oracle; the Rust reference cannot be built here) on this host's cores, on
the same workload and metric (for the flop: one full solve to the target on
the same check schedule); under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime as dt
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "time to 0.5%-pot exploitability, DCFR iters/s, % HBM roofline, vs CPU ref"
UNIT = "DCFR iters/s"
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024
CLOCK_FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

WORKLOADS = {
    "turn": ("turn subgame Ks7s2dTh: 48 river runouts, pot 20bb, stacks 90bb, bets 33%/75%/all-in + 2.5x raise "
             "on turn and river, seeded class ranges (seeds 1000/1001, 51 of 169 classes zeroed), f32 storage, "
             "DCFR alpha 1.5 beta 0 gamma 2"),
    "turn-narrow": ("turn subgame Ks7s2dTh as in the turn workload with the flop workload's narrow ranges "
                    "(Dirichlet(0.5) classes thresholded to 68 of 169, seeds 2000/2001), f32 storage, DCFR alpha 1.5 "
                    "beta 0 gamma 2"),
    "river": ("river subgame Ks7s2dTh4c: pot 20bb, stacks 90bb, bets 50%/100%/all-in + 2.5x raise, seeded class "
              "ranges (seeds 1000/1001), f32 storage, DCFR alpha 1.5 beta 0 gamma 2"),
    "batch": ("512 independent river spots in one persistent launch per block of iterations under a captured CUDA "
              "graph: 5-card boards from seed 3000, pots U[400,6000] chips, stacks U[2000,15000], menus of 1-3 sizes from "
              "{33,50,75,100,150}% plus all-in for bets and raises, trees of 15-400 nodes, seeded class ranges, f32, "
              "DCFR alpha 1.5 beta 0 gamma 2, 500 iterations each, autotuned launch shape"),
    "learned": ("learned depth-limited flop solve: the flop workload's tree cut at the turn deal, leaves valued by "
                "an MLP (2706 inputs: both ranges, board one-hot, pot and stack; 4 hidden layers of 1024 with GELU; "
                "2652 outputs: every combo's EV per player) in BF16 with FP32 accumulation on the library's tcgen05 "
                "kernels, trained on seeded turn subgames solved by the GPU solver to 0.3% of the pot; compared with "
                "the full-tree solve on time to 0.5% exploitability"),
    "flop": ("flop full tree Ks7s2d: pot 6bb, stacks 97bb, bets 33%/75%/all-in + 3x raise on every street, "
             "Dirichlet(0.5) class ranges thresholded to 68 of 169 classes (seeds 2000/2001), f32 storage, "
             "suit isomorphism, DCFR alpha 1.5 beta 0 gamma 2; solved to 0.5% of the pot"),
}


def workload_config(name: str, precision: str):
    from poker_trainer_b200 import workloads
    cfg = {"turn": workloads.turn_spot, "turn-narrow": workloads.turn_narrow_spot, "river": workloads.river_spot,
           "flop": workloads.flop_spot,
           "batch": workloads.river_spot, "learned": workloads.flop_spot}[name]()
    from poker_trainer_b200 import abi
    cfg.precision = abi.PRECISIONS[precision]
    if STORAGE == "compressed":
        cfg.storage = abi.STORAGE_COMPRESSED
    if SAMPLE is not None:
        cfg.chance = abi.CHANCE_SAMPLED
        cfg.chance_turn, cfg.chance_river, cfg.chance_seed = SAMPLE
    return cfg


# --storage: the workloads' own f32 storage, or 16-bit compressed storage
# (Storage::Compressed) on the same trees.
STORAGE = "f32"
# --chance sampled: (turn cards, river cards, seed) of ChanceMode::Sampled on
# the same spots; None deals every card.
SAMPLE = None


def chance_desc() -> str:
    if SAMPLE is None:
        return "exact"
    return f"sampled: {SAMPLE[0]} turn and {SAMPLE[1]} river cards per chance node, seed {SAMPLE[2]}"


# ----------------------------------------------------------------- CPU oracle
def oracle_lib():
    """The CPU oracle (test infrastructure): used only for the CPU baseline and
    the reference arm."""
    path = os.path.join(HERE, "oracle", "liboracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "oracle")], check=True)
    L = C.CDLL(path)
    L.oracle_create.restype = C.c_void_p
    L.oracle_create.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.oracle_destroy.argtypes = [C.c_void_p]
    L.oracle_iterate.argtypes = [C.c_void_p, C.c_uint32]
    L.oracle_set_threads.argtypes = [C.c_int]
    L.oracle_get_threads.restype = C.c_int
    L.oracle_exploitability.argtypes = [C.c_void_p]
    L.oracle_exploitability.restype = C.c_double
    return L


def time_oracle(cfg, threads: int, warmup: int, max_steps: int | None, budget_s: float | None):
    """Iterations/s of the oracle on `threads` host threads: `warmup`
    untimed iterations, then up to `max_steps` iterations or until `budget_s`
    seconds have passed."""
    L = oracle_lib()
    L.oracle_set_threads(threads)
    err = C.c_int(0)
    h = L.oracle_create(C.byref(cfg), C.byref(err))
    if not h:
        raise RuntimeError(f"oracle_create failed ({err.value})")
    try:
        if warmup:
            L.oracle_iterate(h, warmup)
        done = 0
        t0 = time.perf_counter()
        while True:
            L.oracle_iterate(h, 1)
            done += 1
            el = time.perf_counter() - t0
            if max_steps is not None and done >= max_steps:
                break
            if budget_s is not None and el >= budget_s:
                break
        return done, el, L.oracle_get_threads()
    finally:
        L.oracle_destroy(h)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of one GPU during the timed region."""

    def __init__(self, device_index: int):
        import torch
        ident = str(device_index)
        try:
            ident = "GPU-" + str(torch.cuda.get_device_properties(device_index).uuid)
        except Exception:
            pass
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={ident}", f"--query-gpu={CLOCK_FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        self.t0 = self.t1 = None

    def begin(self):
        self.t0 = dt.datetime.now()

    def end(self):
        self.t1 = dt.datetime.now()

    def close(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [ln.strip() for ln in self.file.read().splitlines() if ln.strip()]
        os.unlink(self.file.name)
        samples = []
        for ln in rows:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = dt.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                samples.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        inside = [s for s in samples if self.t0 is not None and self.t0 <= s[0] <= self.t1]
        use = inside or samples
        if not use:
            return None
        reasons = sorted({REASONS[i] for s in use for i in range(4) if s[3][i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(s[1] for s in use), "sm_max_mhz": max(s[2] for s in use),
                "reasons": reasons, "samples": len(use), "samples_in_timed_region": len(inside)}


# ----------------------------------------------------------------- helpers
def measured_peak():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    profiles/<kernel>_<workload>.md (a line 'traffic_bytes_per_launch: X')."""
    path = os.path.join(HERE, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as f:
            for ln in f:
                if ln.strip().startswith("traffic_bytes_per_launch:"):
                    return float(ln.split(":", 1)[1].strip().split()[0])
    except (OSError, ValueError):
        pass
    return None


KERNEL_NAMES = {"terminal": "fast_terminal_kernel", "down": "down_kernel", "up": "up_kernel", "other": "other"}
# The CUDA kernel behind each terminal kernel name of dcfr_terminal_kernel.
TERMINAL_FN = {"panel": "panel_terminal_kernel", "warp": "warp_terminal_kernel", "block": "fast_terminal_kernel",
               "group": "group_terminal_kernel", "exact": "terminal_kernel"}


def spawn_ranks(n: int) -> int:
    """--gpus N without a launcher: re-runs this command as N ranks, one
    process per GPU (torch.distributed.run on 127.0.0.1), and returns its
    exit status. Rank 0 prints the JSON line."""
    import socket
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------- arms
def time_oracle_solve(cfg, threads: int, max_iterations: int, target_pct: float, check_every: int):
    """Seconds of the oracle's solve (run_solve, lib.rs:594-642: DCFR
    iterations with exploitability checks on the reference's schedule) from
    a fresh solver to the target, wall clock; creation is not timed."""
    from poker_trainer_b200 import abi
    L = oracle_lib()
    L.oracle_solve.argtypes = [C.c_void_p, C.POINTER(abi.SolveOptions), abi.PROGRESS_CB, C.c_void_p,
                               C.POINTER(abi.Progress)]
    L.oracle_set_threads(threads)
    err = C.c_int(0)
    h = L.oracle_create(C.byref(cfg), C.byref(err))
    if not h:
        raise RuntimeError(f"oracle_create failed ({err.value})")
    checks = []

    def cb(p, _u):
        checks.append((p.contents.iteration, p.contents.exploitability_pct))
        return 1

    cbf = abi.PROGRESS_CB(cb)
    opts = abi.SolveOptions(max_iterations, check_every, target_pct)
    out = abi.Progress()
    try:
        t0 = time.perf_counter()
        L.oracle_solve(h, C.byref(opts), cbf, None, C.byref(out))
        secs = time.perf_counter() - t0
    finally:
        L.oracle_destroy(h)
    return secs, out.iteration, out.exploitability_pct, checks, L.oracle_get_threads()


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    from poker_trainer_b200 import abi  # noqa: F401  (config layout only)
    cfg = workload_config(args.workload, args.precision)
    threads = os.cpu_count() or 1
    if args.workload == "flop":
        secs, iters, pct, checks, used = time_oracle_solve(cfg, threads, args.max_iterations, 0.5, 10)
        sample = (f"one full solve of the flop workload to 0.5% of the pot: {iters} DCFR iterations and "
                  f"{len(checks)} exploitability checks on the reference's schedule (check every 10), ended at "
                  f"{pct:.4f}%")
        line = {
            "impl": "reference", "metric": METRIC, "value": secs, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(iters, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOADS["flop"], "parallelism": "host threads",
                       "implementation": "CPU restatement of the reference's Rust solver (oracle/, C++ with OpenMP "
                                         "over chance children); the Rust crate cannot be built here",
                       "step": "one DCFR iteration of the solve; value is the wall time of the whole solve to 0.5% "
                               "of the pot from a fresh solver (creation untimed)"},
            "time_to_target": {"seconds": secs, "iterations": iters, "checks": len(checks),
                               "exploitability_pct": pct, "target_pct": 0.5},
            "checks": checks,
            "cpu_baseline": {"value": secs, "unit": "s", "cores": used, "kind": "port", "sample": sample},
            "e2e": {"value": secs, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0
    steps, secs, used = time_oracle(cfg, threads, args.warmup, args.steps, args.reference_budget_s)
    value = steps / secs
    sample = f"{steps} DCFR iterations after {args.warmup} untimed ({args.workload} workload)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload], "parallelism": "host threads",
                   "implementation": "CPU restatement of the reference's Rust solver (oracle/, C++ with OpenMP "
                                     "over chance children); the Rust crate cannot be built here"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from poker_trainer_b200 import abi
    from poker_trainer_b200.solver import Solver

    from poker_trainer_b200.dist import Group

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    grp = Group("nccl", torch.device("cuda", local))
    barrier, reduce = grp.barrier, grp.reduce

    cfg = workload_config(args.workload, args.precision)
    K, W = args.steps, args.warmup

    # End to end through the public API: host config in, a K-iteration solve,
    # the storage (regrets and strategy sums) read back into pinned host memory.
    warm = Solver.new(cfg)  # CUDA context, module load
    n_store = warm.storage_len()
    warm.iterate(W)
    warm.close()
    pin_r = torch.empty(n_store, dtype=torch.float32, pin_memory=True)
    pin_s = torch.empty(n_store, dtype=torch.float32, pin_memory=True)
    out = (pin_r.numpy(), pin_s.numpy())
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_solver = Solver.new(cfg)
    e2e_solver.iterate(K)
    e2e_solver.download_storage(out=out)
    t1 = time.perf_counter()
    setup = e2e_solver.setup_profile()
    e2e_solver.close()
    e2e_s = reduce(t1 - t0, "max")
    h2d = C.sizeof(cfg)
    d2h = 8 * n_store

    # Device-resident solve: W warm-up iterations, then K timed iterations.
    g = Solver.new(cfg)
    g.iterate(W)
    g.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    time.sleep(0.5)
    l0 = g.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    g.synchronize()
    if sampler:
        sampler.begin()
    # The timed region: K iterations as captured graph launches, CUDA events
    # on the solver's stream around them (dcfr_last_iterate_ms).
    g.iterate(K)
    g.synchronize()
    torch.cuda.synchronize()
    if sampler:
        sampler.end()
    barrier()
    launches = reduce(float(g.kernel_launches() - l0), "sum")
    clocks = sampler.close() if sampler else None
    ms = reduce(g.last_iterate_ms(), "max")
    # The same iterations again with events between the kernel classes
    # (the per-class breakdown and the roofline of the dominant class).
    prof = g.iterate_profiled(K)
    prof_ms = reduce(prof["total_ms"], "max")
    expl = g.exploitability()
    pot = float(cfg.root.pot)
    it_bytes = g.iteration_bytes()
    tkname, _ = g.terminal_kernel()
    g.close()

    value = world * K / (ms / 1000.0)
    peak, peak_kind = measured_peak()
    classes = prof["classes"]
    dom = max(("down", "terminal", "up"), key=lambda c: classes[c]["ms"])
    dc = classes[dom]
    per_launch_ms = dc["ms"] / max(dc["launches"], 1)
    per_launch_bytes = dc["bytes"] / max(dc["launches"], 1)
    achieved = per_launch_bytes / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms > 0 else 0.0
    kernels = {c: {"launches": v["launches"], "ms": v["ms"], "share": v["ms"] / max(prof["total_ms"], 1e-12),
                   "gbs": (v["bytes"] / (v["ms"] / 1000.0) / 1e9) if v["ms"] > 0 else None}
               for c, v in classes.items()}
    if rank != 0:
        grp.close()
        return 0

    # CPU baseline: the oracle on this host's cores, a bounded sample.
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        steps, secs, used = time_oracle(cfg, threads, 2, None, args.cpu_budget_s)
        cpu = {"value": steps / secs, "unit": UNIT, "cores": used, "kind": "port",
               "sample": f"{steps} DCFR iterations of the same workload after 2 untimed, {secs:.1f} s on {used} "
                         f"host threads (C++ restatement of the reference's CPU solver)"}

    working = it_bytes
    kname = KERNEL_NAMES[dom]
    if dom == "terminal":
        kname = TERMINAL_FN[tkname]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": WORKLOADS[args.workload], "iterations_per_step": 1, "precision": args.precision,
            "storage": args.storage,
            "chance": chance_desc(),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": (f"inputs larger than L2: one iteration moves {working / 1e6:.0f} MB of rows and storage "
                   f"(> {L2_BYTES / 1e6:.0f} MB L2), no flush") if working > L2_BYTES else
                  "working set smaller than L2 (no flush; L2-resident figure)",
            "timing": "value: CUDA events on the solver's stream around K captured-graph iterations, max over "
                      "ranks; kernels and roofline: a second run of K iterations with events between the kernel "
                      "classes inside the graph",
        },
        "clocks": clocks,
        "e2e": {"value": world * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "setup_ms": setup,
                "what": "dcfr_create from the host config + K iterations + regrets and sums read back into pinned "
                        "host memory, wall clock, max over ranks; bytes are the per-solve totals / K"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": f"of {peak_kind}",
                     "traffic": ncu_traffic(kname, args.workload),
                     "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms},
        "iteration_roofline": {"bytes_per_iteration": it_bytes,
                               "achieved": it_bytes * (K / (ms / 1000.0)) / 1e9, "peak": peak, "unit": "GB/s",
                               "frac": it_bytes * (K / (ms / 1000.0)) / 1e9 / peak},
        "kernels": kernels,
        "profiled_ms_per_step": prof_ms / K,
        "exploitability_pct_after": 100.0 * expl / pot,
        "iterations_after": W + 2 * K,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    grp.close()
    return 0


def flop_paths_summary(g, pot):
    """Root strategy and EV read back through the query API (part of the
    end-to-end step: what a caller of the solve reads)."""
    q = g.query([])
    return 4 * (q.strategy.size + q.ev.size + q.reach.size)


def run_turn_secondary(args, grp, local):
    """The turn workload's DCFR iterations/s (device-timed K captured-graph
    iterations after W), reported inside the flop line."""
    from poker_trainer_b200.solver import Solver

    cfg = workload_config("turn", args.precision)
    g = Solver.new(cfg)
    g.iterate(args.warmup)
    g.synchronize()
    grp.barrier()
    g.iterate(args.steps)
    ms = grp.reduce(g.last_iterate_ms(), "max")
    prof = g.iterate_profiled(args.steps)
    kname, per_panel = g.terminal_kernel()
    it_bytes = g.iteration_bytes()
    g.close()
    peak, peak_kind = measured_peak()
    t = prof["classes"]["terminal"]
    return {"workload": WORKLOADS["turn"], "value": grp.world * args.steps / (ms / 1000.0), "unit": UNIT,
            "ms_per_iteration": ms / args.steps,
            "iteration_roofline_frac": it_bytes * args.steps / (ms / 1000.0) / 1e9 / peak,
            "terminal_kernel": TERMINAL_FN[kname], "terminals_per_panel": per_panel,
            "terminal_gbs": t["bytes"] / (t["ms"] / 1000.0) / 1e9 if t["ms"] > 0 else None,
            "terminal_frac": (t["bytes"] / (t["ms"] / 1000.0) / 1e9 / peak) if t["ms"] > 0 else None,
            "peak_kind": f"of {peak_kind}"}


def run_flop(args, world, rank, local):
    """Time to 0.5%-of-pot exploitability on the flop workload (the metric's
    first term). The timed step is the whole solve: dcfr_solve from a fresh
    solver, DCFR iterations with exploitability checks on the reference's
    schedule (check every 10 iterations, then aimed at the predicted
    iteration; lib.rs:158-172, 594-642), device-timed by CUDA events on the
    solver's stream. The final exploitability is re-checked by the FP64
    best-response oracle; K further profiled iterations give the per-class
    breakdown and the terminal kernel's roofline. With N GPUs every rank
    solves its own copy (replicas) and the job time is the maximum over
    ranks."""
    import torch
    from poker_trainer_b200.dist import Group
    from poker_trainer_b200.solver import Solver, SolveOptions

    torch.cuda.set_device(local)
    grp = Group("nccl", torch.device("cuda", local), timeout_s=1200)
    cfg = workload_config("flop", args.precision)
    pot = float(cfg.root.pot)
    # Warm-up: context, module load and clocks, on the turn workload (W
    # iterations); the flop solver itself is created inside the timed e2e.
    warm = Solver.new(workload_config("turn", args.precision))
    warm.iterate(args.warmup)
    warm.close()
    checks = []
    sampler = ClockSampler(local) if rank == 0 else None
    time.sleep(0.5)
    grp.barrier()
    torch.cuda.synchronize()
    # End to end: the host config in, dcfr_create, dcfr_solve to the target
    # (each check reads one f64 back), the root's strategy and EVs read back.
    t0 = time.perf_counter()
    g = Solver.new(cfg)
    t_create = time.perf_counter() - t0
    if sampler:
        sampler.begin()
    l0 = g.kernel_launches()
    prog = g.solve(SolveOptions(max_iterations=args.max_iterations, target_exploitability_pct=0.5, check_every=10),
                   on_progress=lambda pr: checks.append((pr.iteration, pr.exploitability_pct)) or True)
    solve_launches = g.kernel_launches() - l0
    t_solved = time.perf_counter()
    if sampler:
        sampler.end()
    d2h_query = flop_paths_summary(g, pot)
    g.synchronize()
    t_e2e = time.perf_counter() - t0
    t_solve_wall, t_query = t_solved - t0 - t_create, t_e2e - (t_solved - t0)
    solve_s = grp.reduce(g.last_solve_ms() / 1000.0, "max")
    e2e_s = grp.reduce(t_e2e, "max")
    clocks = sampler.close() if sampler else None
    setup = g.setup_profile()
    e32 = g.exploitability()
    e64, _ = g.exploitability_fp64()
    K = args.steps
    prof = g.iterate_profiled(K)
    it_bytes = g.iteration_bytes()
    kname, per_panel = g.terminal_kernel()
    g.close()
    turn = run_turn_secondary(args, grp, local) if not args.no_secondary else None
    ms = prof["total_ms"]
    peak, peak_kind = measured_peak()
    classes = prof["classes"]
    kernels = {c: {"launches": v["launches"], "ms": v["ms"], "share": v["ms"] / max(ms, 1e-12),
                   "gbs": (v["bytes"] / (v["ms"] / 1000.0) / 1e9) if v["ms"] > 0 else None}
               for c, v in classes.items()}
    dom = max(("down", "terminal", "up"), key=lambda c: classes[c]["ms"])
    dc = classes[dom]
    per_launch_ms = dc["ms"] / max(dc["launches"], 1)
    per_launch_bytes = dc["bytes"] / max(dc["launches"], 1)
    achieved = per_launch_bytes / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms > 0 else 0.0
    kfull = TERMINAL_FN[kname] if dom == "terminal" else KERNEL_NAMES[dom]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        steps, secs, used = time_oracle(cfg, threads, 1, args.cpu_flop_iters, None)
        per_it = secs / steps
        # A check is two best-response traversals: about one iteration.
        cpu_ttt = per_it * (prog.iteration + len(checks))
        cpu = {"value": cpu_ttt, "unit": "s", "cores": used, "kind": "port",
               "sample": f"{steps} DCFR iterations of the flop workload after 1 untimed, {secs:.1f} s on {used} host "
                         f"threads (C++ restatement of the reference's CPU solver), scaled to the GPU solve's "
                         f"{prog.iteration} iterations + {len(checks)} checks ({per_it:.3f} s per iteration); "
                         f"bench.py --impl reference measures the full CPU solve",
               "iters_per_s": 1.0 / per_it}
    iters = prog.iteration
    line = {
        "metric": METRIC, "value": solve_s, "unit": "s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": 1000.0 * solve_s / max(iters, 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS["flop"], "precision": args.precision, "storage": args.storage,
                   "chance": chance_desc(),
                   "parallelism": f"replicas x{world} (every rank solves the spot; job time is the max)"
                                  if world > 1 else "single GPU",
                   "step": "one DCFR iteration of the solve; value is the device time of the whole solve to 0.5% "
                           "of the pot (its iterations and exploitability checks, CUDA events on the solver's "
                           "stream), ms_per_step that time per iteration",
                   "warmup": "W DCFR iterations of the turn workload before the timed solve (context, module, "
                             "clocks)",
                   "profiled": "K DCFR iterations after the solve, with events between kernel classes",
                   "l2": f"inputs larger than L2: one iteration moves {it_bytes / 1e9:.1f} GB, no flush"},
        "time_to_target": {"seconds": solve_s, "iterations": iters, "checks": len(checks),
                           "exploitability_pct": prog.exploitability_pct, "target_pct": 0.5,
                           "iters_per_s": iters / solve_s if solve_s > 0 else None,
                           "fp64_oracle_exploitability_pct": 100.0 * e64 / pot,
                           "f32_exploitability_pct": 100.0 * e32 / pot,
                           "fp64_vs_f32_rel": abs(e64 - e32) / max(abs(e64), 1e-30)},
        "checks": checks,
        "clocks": clocks,
        "gpu_launches": int(solve_launches),
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": C.sizeof(cfg) / max(iters, 1),
                "d2h_bytes_per_step": (8.0 * len(checks) + d2h_query) / max(iters, 1),
                "create_seconds": t_create, "solve_wall_seconds": t_solve_wall, "query_seconds": t_query,
                "setup_ms": setup,
                "what": "dcfr_create from the host config + dcfr_solve to the target (each check reads one f64 "
                        "back) + the root's strategy and EVs read back, wall clock, max over ranks; bytes per "
                        "iteration"},
        "roofline": {"bound": "hbm", "kernel": kfull, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"of {peak_kind}",
                     "traffic": ncu_traffic(kfull, "flop"), "bytes_per_launch": per_launch_bytes,
                     "ms_per_launch": per_launch_ms, "terminals_per_panel": per_panel},
        "iteration_roofline": {"bytes_per_iteration": it_bytes,
                               "achieved": it_bytes * (K / (ms / 1000.0)) / 1e9, "peak": peak, "unit": "GB/s",
                               "frac": it_bytes * (K / (ms / 1000.0)) / 1e9 / peak},
        "kernels": kernels,
        "turn": turn,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    grp.close()
    return 0


def batch_configs():
    """The 512 spots of the batched workload (seed 3000). A multi-GPU run
    partitions them across ranks (poker_trainer_b200.dist.shard)."""
    from poker_trainer_b200 import workloads
    from poker_trainer_b200.solver import Solver

    def nodes(c):
        st = Solver.estimate(c)
        return st.player_nodes + st.chance_nodes + st.terminal_nodes
    return workloads.batched_river_spots(count=512, seed=3000, estimate=nodes)


def run_batch(args, world, rank, local):
    """The batched river workload: the 512 spots are partitioned across the
    ranks (each solves its contiguous share; strong scaling) and the
    per-spot exploitabilities are gathered on rank 0; a step is one DCFR
    iteration of every spot, reported as spot-iterations per second of the
    whole job."""
    import numpy as np
    import torch
    from poker_trainer_b200.solver import BatchSolver

    from poker_trainer_b200.dist import Group, shard

    torch.cuda.set_device(local)
    grp = Group("nccl", torch.device("cuda", local))

    def reduce_max(x):
        return grp.reduce(x, "max")

    all_cfgs = batch_configs()
    S_total = len(all_cfgs)
    cfgs = shard(all_cfgs, rank, world)
    S = len(cfgs)
    K, W = args.steps, args.warmup
    # End to end: create from host configs, K iterations, storage of every spot read back.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e = BatchSolver.new(cfgs)
    if args.batch_tuning:
        from poker_trainer_b200 import abi
        w_, b_, i_, l_ = (int(x) for x in args.batch_tuning.split(","))
        tuned = abi.BatchTuning(warps=w_, blocks_per_sm=b_, iterations_per_launch=i_, longest_first=l_)
        e2e.set_tuning(tuned)
    else:
        tuned = e2e.autotune(10)
    e2e.iterate(K)
    d2h = 0
    for i in range(S):
        r, sm = e2e.download_storage(i)
        d2h += r.nbytes + sm.nbytes
    t_e2e = reduce_max(time.perf_counter() - t0)
    e2e.close()
    b = BatchSolver.new(cfgs)
    b.set_tuning(tuned)
    b.iterate(W)
    sampler = ClockSampler(local) if rank == 0 else None
    time.sleep(0.5)
    l0 = b.kernel_launches()
    grp.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.begin()
    b.iterate(K)
    torch.cuda.synchronize()
    if sampler:
        sampler.end()
    clocks = sampler.close() if sampler else None
    ms = reduce_max(b.last_iterate_ms())
    launches = b.kernel_launches() - l0
    expl = b.exploitability()
    pots = np.array([c.root.pot for c in cfgs], np.float64)
    it_bytes = b.iteration_bytes()
    b.close()
    # Every spot's exploitability, gathered on rank 0 in spot order.
    expl_all = np.asarray(grp.gather_concat(list(100.0 * np.asarray(expl) / pots)), np.float64)
    it_bytes_all = grp.reduce(it_bytes, "sum")
    value = S_total * K / (ms / 1000.0)
    peak, peak_kind = measured_peak()
    # The persistent kernel is the only kernel of the timed region: its
    # algorithmic bytes per launch are every spot's B_iter times the
    # iterations per launch; the committed ncu traffic is for 10 iterations
    # per launch and scales with that count.
    ipl = max(int(tuned.iterations_per_launch), 1)
    n_launch = max(int(launches), 1)
    per_launch_ms = ms / n_launch
    per_launch_bytes = it_bytes * K / n_launch
    traffic = ncu_traffic("batch_kernel", "batch")
    roof = {"bound": "hbm", "kernel": "batch_kernel",
            "achieved": per_launch_bytes / (per_launch_ms / 1000.0) / 1e9 if per_launch_ms > 0 else 0.0,
            "peak": peak, "unit": "GB/s", "peak_kind": f"of {peak_kind}",
            "traffic": traffic * ipl / 10.0 if traffic else None,
            "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms}
    roof["frac"] = roof["achieved"] / peak
    cpu = None
    if world == 1 and not args.no_cpu_baseline and rank == 0:
        L = oracle_lib()
        L.oracle_batch_iterate.argtypes = [C.c_void_p, C.c_int, C.c_uint32, C.c_int]
        threads = os.cpu_count() or 1
        L.oracle_set_threads(1)
        err = C.c_int(0)
        hs = [L.oracle_create(C.byref(c), C.byref(err)) for c in cfgs]
        arr = (C.c_void_p * S)(*hs)
        L.oracle_batch_iterate(arr, S, 1, threads)
        n_cpu = args.cpu_batch_iters
        tc0 = time.perf_counter()
        L.oracle_batch_iterate(arr, S, n_cpu, threads)
        secs = time.perf_counter() - tc0
        for h in hs:
            L.oracle_destroy(h)
        cpu = {"value": S * n_cpu / secs, "unit": "spot-iterations/s", "cores": threads, "kind": "port",
               "sample": f"{n_cpu} DCFR iterations of each of the {S} spots after 1 untimed, {secs:.1f} s, spots spread "
                         f"over {threads} host threads (C++ restatement of the reference's CPU solver)"}
    line = {
        "metric": METRIC, "value": value, "unit": "spot-iterations/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["batch"], "spots": S_total, "spots_per_rank": S, "iterations_per_step": 1,
                   "parallelism": f"spots partitioned over {world} ranks" if world > 1 else "single GPU",
                   "tuning": {"warps": tuned.warps, "blocks_per_sm": tuned.blocks_per_sm,
                              "iterations_per_launch": tuned.iterations_per_launch,
                              "longest_first": tuned.longest_first, "candidates": tuned.candidates},
                   "l2": f"one iteration of all spots moves {it_bytes / 1e9:.2f} GB (> 126 MB L2), no flush"},
        "solve_ms": ms, "clocks": clocks,
        "e2e": {"value": S_total * K / t_e2e, "unit": "spot-iterations/s",
                "h2d_bytes_per_step": S * C.sizeof(cfgs[0]) / K, "d2h_bytes_per_step": d2h / K,
                "what": "dcfr_batch_create + autotune + K iterations + every spot's storage read back, wall clock"},
        "gpu_launches": int(launches),
        "roofline": roof,
        "iteration_roofline": {"bytes_per_iteration": it_bytes_all,
                               "achieved": it_bytes_all * K / (ms / 1000.0) / 1e9 / world,
                               "peak": peak, "unit": "GB/s",
                               "frac": it_bytes_all * K / (ms / 1000.0) / 1e9 / world / peak,
                               "peak_kind": f"of {peak_kind} (per GPU)"},
        "exploitability_pct_mean_after": float(np.mean(expl_all)) if rank == 0 else None,
        "spots_gathered": int(len(expl_all)) if rank == 0 else None,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    grp.close()
    return 0


def flop_paths(g, path=()):
    """Every decision path of a solver's flop street (stops at chance
    nodes, leaves and terminals)."""
    out = []
    if not g.is_decision(list(path)):
        return out
    out.append(list(path))
    for a in g.actions_at(list(path)):
        out += flop_paths(g, list(path) + [a])
    return out


def run_learned(args, world, rank, local):
    """Config of the learned depth-limited flop solve: data from the GPU
    solver (turn subgames solved to 0.3% of the pot), networks trained on
    growing prefixes of the data on the library's tensor-core kernels
    (held-out error against training-set size), the depth-limited solve with
    the largest network against the full-tree solve, and the depth-limited
    flop strategy evaluated inside the full tree by the FP64 best-response
    oracle. Data generation and training are reported as a one-time cost:
    the same network serves every flop of this shape. With N GPUs the
    subgames are partitioned across ranks (each solves its share) and the
    network trains data-parallel; rank 0 runs the solves and reports."""
    import numpy as np
    import torch
    from poker_trainer_b200 import leafdata
    from poker_trainer_b200.dist import Group
    from poker_trainer_b200.mlp import LeafNet, gemm_time
    from poker_trainer_b200.solver import Solver, SolveOptions
    from poker_trainer_b200.train_leaf import masked_mse, predict, train

    torch.cuda.set_device(local)
    grp = Group("nccl", torch.device("cuda", local), timeout_s=3600)
    cfg = workload_config("flop", "fast")
    pot = float(cfg.root.pot)
    sizes = sorted({int(x) for x in args.learned_sizes.split(",")} | {args.learned_samples}) \
        if args.learned_sizes else [args.learned_samples]
    sizes = [n for n in sizes if n <= args.learned_samples]
    t0 = time.perf_counter()
    X, Y, M, _, iters = leafdata.make_dataset(args.learned_samples, seed=4000, target_pct=0.3, max_iterations=400,
                                              workers=args.learned_workers, part=(rank, world))
    torch.cuda.synchronize()
    t_data = grp.reduce(time.perf_counter() - t0, "max")
    Xh, Yh, Mh, Eh, _ = leafdata.make_dataset(args.learned_heldout, seed=5000, target_pct=0.3, max_iterations=400,
                                              with_equity=True, workers=args.learned_workers)
    per_hand_mean = None
    curve = []
    net = None
    t_train = 0.0
    for n in sizes:
        # The first n subgames of the seeded sequence (this rank's share of
        # them under N ranks: samples r, r + N, ...).
        k = len(range(rank, n, world))
        steps = max(args.learned_steps, int(args.learned_steps * n / sizes[-1])) if n == sizes[-1] else \
            max(1000, int(args.learned_steps * n / sizes[-1]))
        t0 = time.perf_counter()
        net_n, losses = train(X[:k], Y[:k], M[:k], hidden=1024, layers=4, steps=steps, batch=256, lr=1e-3, seed=0,
                              group=grp if world > 1 else None, local=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        pred = predict(net_n, Xh)
        mean = (Y[:k] * M[:k]).sum(0) / np.maximum(M[:k].sum(0), 1.0)
        curve.append({"training_subgames": n, "steps": steps, "train_seconds": dt,
                      "heldout_mse": masked_mse(pred, Yh, Mh),
                      "heldout_mse_per_hand_mean": masked_mse(mean[None, :], Yh, Mh),
                      "loss_last": float(np.mean(losses[-20:]))})
        if n == sizes[-1]:
            net, t_train, per_hand_mean = net_n, dt, masked_mse(mean[None, :], Yh, Mh)
    if rank != 0:
        grp.close()
        return 0
    # The solve's network: same weights, batch room for every leaf x card.
    dlnet = LeafNet(leafdata.IN_DIM, 1024, 4, leafdata.OUT_DIM, max_batch=8192, seed=0)
    dlnet.set_params(net.params())
    # Tensor-core throughput of the network's GEMM at the solve's shape class
    # (CUDA events around back-to-back launches on one stream).
    gemm_s = gemm_time(4096, 1024, 2816, reps=50) * 1e-3
    gemm_tflops = 2.0 * 4096 * 2816 * 1024 / gemm_s / 1e12
    opts = SolveOptions(max_iterations=args.max_iterations, target_exploitability_pct=0.5, check_every=10)
    full = Solver.new(cfg)
    pf = full.solve(opts)
    t_full = full.last_solve_ms() / 1000.0
    e_full, _ = full.exploitability_fp64()
    dl = Solver.new_depth_limited(cfg, dlnet)
    pd = dl.solve(opts)
    t_dl = dl.last_solve_ms() / 1000.0
    # Check: the depth-limited flop strategy inside the full tree.
    paths = flop_paths(dl)
    diffs = []
    for path in paths:
        q = dl.query(path)
        qf = full.query(path)
        full.write_node(path, sums=q.strategy)
        w = np.asarray(qf.reach, np.float64)
        rs = lambda st: (np.asarray(st, np.float64) * w[None, :]).sum(1) / max(w.sum(), 1e-30)
        diffs.append(float(np.max(np.abs(rs(q.strategy) - rs(qf.strategy)))))
    e_comb, _ = full.exploitability_fp64()
    full.close()
    # Check 2: the depth-limited flop strategy locked into the full tree and
    # the turn and river re-solved around it. Its regrets are written as
    # 1e20 x its probabilities: regret matching keeps playing it exactly
    # (what one iteration adds is below f32 resolution of those regrets, and
    # DCFR discounts all of a node's positive regrets by the same factor).
    # The re-solve stops at the full solve's FP64 exploitability (or its
    # iteration cap): equal quality, and the time that takes.
    lk = Solver.new(cfg)
    for path in paths:
        st = np.asarray(dl.query(path).strategy, np.float64)
        lk.write_node(path, regrets=(1e20 * st).astype(np.float32))
    target = max(100.0 * e_full / pot, 0.5)
    plk = lk.solve(SolveOptions(max_iterations=args.lock_iterations, target_exploitability_pct=target,
                                check_every=50))
    t_lock = lk.last_solve_ms() / 1000.0
    e_lock, _ = lk.exploitability_fp64()
    lk.close()
    # One turn subgame re-solved on the path played (check-check, then the
    # As), the work a player of the depth-limited strategy does per turn
    # reached: both ranges as they arrive at the cut under the depth-limited
    # flop strategy, solved to 0.5% of the pot.
    turn_resolve = None
    try:
        dlp = dl.ranges_after(["check", "check"])
    except Exception:
        dlp = None
    if dlp is not None:
        sub = leafdata.config_of(leafdata.abi.parse_cards("Ks7s2dAs"), int(pot), int(cfg.root.stack[0]),
                                 [np.asarray(dlp[0], np.float32), np.asarray(dlp[1], np.float32)])
        ts = Solver.new(sub)
        pts = ts.solve(SolveOptions(max_iterations=1000, target_exploitability_pct=0.5, check_every=10))
        turn_resolve = {"path": ["check", "check", "As"], "seconds": ts.last_solve_ms() / 1000.0,
                        "iterations": pts.iteration, "exploitability_pct": pts.exploitability_pct}
        ts.close()
    dl.close()
    peak = 1672.6
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        pass
    line = {
        "metric": METRIC, "value": t_dl, "unit": "s", "n_gpus": world, "steps": pd.iteration,
        "warmup": 0, "ms_per_step": 1000.0 * t_dl / max(pd.iteration, 1), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 solve, bf16 network (fp32 accumulation)",
        "data": "synthetic", "config": {"workload": WORKLOADS["learned"], "training_samples": args.learned_samples,
                                        "training_steps": args.learned_steps, "sizes": sizes},
        "time_to_target": {"full_tree_s": t_full, "full_tree_iterations": pf.iteration,
                           "full_tree_exploitability_pct_fp64": 100.0 * e_full / pot,
                           "depth_limited_s": t_dl, "depth_limited_iterations": pd.iteration,
                           "depth_limited_game_exploitability_pct": pd.exploitability_pct,
                           "speedup": t_full / t_dl,
                           "depth_limited_flop_strategy_in_full_tree_exploitability_pct_fp64": 100.0 * e_comb / pot,
                           "flop_nodes": len(paths), "max_range_strategy_diff": max(diffs) if diffs else None,
                           "locked_resolve_target_pct": target,
                           "depth_limited_flop_strategy_locked_resolve_exploitability_pct_fp64": 100.0 * e_lock / pot,
                           "locked_resolve_iterations": plk.iteration, "locked_resolve_s": t_lock,
                           "turn_resolve_on_path": turn_resolve},
        "one_time_cost": {"data_seconds": t_data, "train_seconds": t_train, "heldout_subgames": args.learned_heldout,
                          "subgames": args.learned_samples, "solve_iterations_mean": float(np.mean(iters)),
                          "note": "paid once for every flop of this shape; not part of a solve"},
        "training": {"curve": curve, "heldout_mse_showdown_equity": masked_mse(Eh, Yh, Mh),
                     "heldout_mse_per_hand_mean": per_hand_mean},
        "roofline": {"bound": "tensor", "kernel": "gemm_bf16_tc_kernel (4096 x 1024 x 2816)", "achieved": gemm_tflops,
                     "peak": peak, "unit": "TFLOP/s", "frac": gemm_tflops / peak, "peak_kind": "of measured",
                     "traffic": None},
    }
    print(json.dumps(line), flush=True)
    grp.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="flop")
    ap.add_argument("--precision", choices=["fast", "exact"], default="fast")
    ap.add_argument("--storage", choices=["f32", "compressed"], default="f32",
                    help="turn, river, flop: f32 (the workloads' storage) or 16-bit compressed storage")
    ap.add_argument("--chance", choices=["exact", "sampled"], default="exact",
                    help="turn, river, flop: every card, or ChanceMode::Sampled with --sample")
    ap.add_argument("--sample", default="8,6,3", metavar="TURN,RIVER,SEED",
                    help="--chance sampled: cards dealt per turn and river chance node, and the seed")
    ap.add_argument("--cpu-budget-s", type=float, default=10.0)
    ap.add_argument("--reference-budget-s", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="flop: skip the turn workload's iters/s field")
    ap.add_argument("--max-iterations", type=int, default=2000, help="flop: iteration cap of the timed solve")
    ap.add_argument("--cpu-flop-iters", type=int, default=3, help="flop: oracle iterations timed for the CPU figure")
    ap.add_argument("--cpu-batch-iters", type=int, default=20, help="batch: oracle iterations per spot timed")
    ap.add_argument("--learned-samples", type=int, default=1024, help="learned: solved turn subgames to train on")
    ap.add_argument("--learned-steps", type=int, default=2000, help="learned: training steps (largest size)")
    ap.add_argument("--learned-sizes", default=None, metavar="N1,N2,...",
                    help="learned: also train on these prefixes of the data (held-out error against size)")
    ap.add_argument("--learned-workers", type=int, default=4, help="learned: host threads solving subgames")
    ap.add_argument("--learned-heldout", type=int, default=64, help="learned: held-out subgames (seed 5000)")
    ap.add_argument("--batch-tuning", default=None, metavar="WARPS,BLOCKS_PER_SM,ITERS_PER_LAUNCH,LONGEST_FIRST",
                    help="batch: a fixed launch shape instead of the autotuner's")
    ap.add_argument("--lock-iterations", type=int, default=300,
                    help="learned: iterations of the full-tree re-solve around the locked flop strategy")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    global STORAGE, SAMPLE
    STORAGE = args.storage
    if args.chance == "sampled":
        t, r, sd = (int(x) for x in args.sample.split(","))
        if t < 1 or r < 1:
            ap.error("--sample deals at least one card per street")
        SAMPLE = (t, r, sd)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    world, rank, local = dist_setup(args.gpus)
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; running {world} rank(s)", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload == "flop":
        return run_flop(args, world, rank, local)
    if args.workload == "batch":
        return run_batch(args, world, rank, local)
    if args.workload == "learned":
        return run_learned(args, world, rank, local)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
