#!/usr/bin/env python
"""Benchmark of the river-subtree CFR hot path on the fixed-flop limit game.

One step = one river pass (CFR regret update, alternating the updating player step by step)
over all 27,783 river subgames of the reference's fixed-flop game, with uniform opponent
ranges over the hands the 4-card board does not block (the reference's Vector::ones).
Metric: river node visits per second (27,783 subgames x 48 rivers x 27 nodes per pass, the
count the reference's evaluate_river walks).

  value        device-resident pass (inputs already in HBM), timed with CUDA events
  e2e          the same pass through the reference-facing C ABI with host buffers:
               upload of every range to the staging, evaluate_cuda (host->device copy,
               kernel, device->host copy), download of every result
  roofline     algorithmic HBM bytes of the pass / kernel time vs measured HBM peak
  cpu_baseline the oracle (CPU restatement of the reference path) on a bounded sample

--impl reference times the reference's CPU implementation of the path (the oracle port;
the reference itself is Rust and cannot be built here) on the same workload.
With torchrun (N > 1) every rank runs its own full pass (replicas, weak scaling).
The line also carries one summary per further configuration (batched general subgames, the
adjoint pair, the value network, the full game with general bets); --traces adds their
exploitability trajectories and loss curves.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SUBGAMES = 27783                 # 63 * 49 * 9 river roots (interface.cu:17)
REFERENCE_FLOP = 0b111           # cards {0, 1, 2} = 2c 3c 4c, the reference's fixed flop
NODES_PER_SUBGAME = 48 * 27      # 48 river cards x 27 states below the river root
METRIC = "river-subtree CFR throughput, fixed-flop game (river node visits/s)"
UNIT = "nodes/s"
WORKLOAD = "fixed-flop limit hold'em, all 27783 river subgames, one CFR pass per step"


# DRAM bytes of one full river launch (27,783 subgames), read + write, from a single-pass ncu
# capture of this program (dram__bytes_read.sum + dram__bytes_write.sum)
TRAFFIC_PER_LAUNCH = 1063193600 + 509289984
# The on-chip bound of the river pass: its shared-memory data pipe's share of peak
# (l1tex__data_pipe_lsu_wavefronts_mem_shared.avg.pct_of_peak_sustained_elapsed) and
# wavefronts per subgame-river card, from an ncu capture of the 4096-subgame case
SMEM_PIPE_FRAC = 0.674
SMEM_WAVEFRONTS_PER_RIVER_CARD = 2289425218 / (4096 * 48)


def algorithmic_bytes(n):
    # ranges in + values out (1326 f32 each), regrets read (26 x 256 f32) and written
    # (the updater's 13 edges), tables once per pass (1176 boards x 11632 B).
    return n * (2 * 1326 * 4 + 26 * 1024 + 13 * 1024) + 1176 * 11632


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tensor_peaks():
    """Measured BF16 dense peaks (burst, sustained) in TFLOP/s, else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("bf16_tflops", 1590.0)), float(d.get("bf16_tflops_sustained", 1400.0))
    return 1590.0, 1400.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 6:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def uniform_ranges(order, boards):
    """Opponent ranges of the stated workload: 1 on every hand the 4-card board does not
    block, 0 on the others (the reference's Vector::ones, game.rs:37-38, masked)."""
    r = np.ones((len(boards), 1326), dtype=np.float32)
    r[(order[None, :] & boards[:, None]) != 0] = 0.0
    return r


def bench_config(n, world):
    """The workload description both arms print."""
    return {"workload": WORKLOAD, "subgames": n, "flop": "2c3c4c (reference cards 0,1,2)",
            "ranges": "uniform over the hands the 4-card board does not block",
            "l2": "inputs larger than L2 (ranges+results+regrets ~1.04 GB)",
            "parallelism": f"replicas x{world}"}


def cpu_sample(boards, bets, ranges, tables, nthreads, subgames):
    """Times the oracle's river pass on `subgames` roots; returns nodes/s."""
    from oracle import oracle as O
    e, _, a = tables
    idx = np.linspace(0, len(boards) - 1, subgames).astype(np.int64)
    reg = np.zeros((subgames, 26, 256), np.float32)
    t0 = time.perf_counter()
    O.river_batch(O.REFERENCE_FLOP, e, a, boards[idx], bets[idx], ranges[idx], reg, 0, False, nthreads)
    dt = time.perf_counter() - t0
    return subgames * NODES_PER_SUBGAME / dt, dt


def sized_sample(boards, bets, ranges, tables, nthreads, seconds):
    """Number of roots whose oracle pass takes about `seconds` on these host threads, from a
    timed probe of 4 roots per thread."""
    probe = max(4 * nthreads, 32)
    _, dt = cpu_sample(boards, bets, ranges, tables, nthreads, probe)
    return int(min(len(boards), max(probe, probe * seconds / max(dt, 1e-6))))


BATCH_SUBGAMES = 4096
BATCH_ITERATIONS = 500


def batch_section(P, rank, peak, cpu_threads, with_cpu, traces):
    """General river subgames (4096 seeded boards, pots, stacks and bet trees): per-hand CFR
    iterations through the batched solver, its HBM roofline, iterations / seconds until the
    mean FP64 exploitability of the average strategies is at most 0.5 % of the pot, and the
    stated 500-iteration solve end to end through the C ABI (host specs and ranges in, host
    average sums out)."""
    specs, ranges = P.random_subgames(BATCH_SUBGAMES, seed=4321 + rank)
    b = P.Batch(specs, ranges)
    b.enable_average()
    b.iterate(2)  # the first iteration runs eagerly, then one iteration is captured as a graph
    tuned = b.tune()
    steps = 20
    t0 = time.perf_counter()
    b.iterate(steps)
    it_s = (time.perf_counter() - t0) / steps
    nbytes = b.iteration_bytes()
    edges = sum(b.shape(i)[1] for i in range(b.count))
    cfgs = [b.config(c) for c in range(2)]
    out = {
        "workload": f"{BATCH_SUBGAMES} river subgames, 5-card seeded boards, pot U{{2..200}}, stack U{{pot..10 pot}}, "
                    "bets from {0.5 pot, pot, all-in}, 1-3 raises, ranges U(0,1) with 25 % zeroed",
        "iteration_ms": it_s * 1e3, "edges": edges,
        "hand_edge_updates_per_s": edges * 1081 * 2 / it_s,
        "roofline": {"bound": "hbm", "achieved": nbytes / it_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": nbytes / it_s / 1e9 / peak, "bytes_per_iteration": nbytes},
        "tuned_pass_ms": [round(float(x), 4) for x in tuned],
        "configs": [f"K{c['K']}x{c['per_sm']}/o{c['order']}/{c['count']}" for c in cfgs],
    }
    b.close()
    # convergence: restart from zero regrets, average sums weighted by the iteration number,
    # check every 25 iterations
    b2 = P.Batch(specs, ranges)
    b2.enable_average()
    b2.set_linear_average(True)
    for c in range(2):
        b2.set_config(c, cfgs[c]["K"], cfgs[c]["per_sm"], cfgs[c]["order"])
    done, t_solve, reached = 0, 0.0, None
    trace = []
    while done < 1000:
        t0 = time.perf_counter()
        b2.iterate(25)
        t_solve += time.perf_counter() - t0
        done += 25
        _, _, ex = b2.exploitability(use_average=True, fp64=True)
        pct = float(np.mean(ex / specs["pot"]) * 100.0)
        trace.append((done, round(pct, 4)))
        if pct <= 0.5:
            reached = {"iterations": done, "solve_s": round(t_solve, 4)}
            break
    if traces:
        out["exploitability_pct_pot"] = trace
    out["time_to_0.5pct_pot"] = reached
    out["averaging"] = "linear (iteration t weighs t)"
    b2.close()
    # end to end: the stated solve (500 iterations) from host specs and ranges to host average
    # sums, through pr_batch_new / pr_batch_iterate / pr_batch_get_all
    import torch
    torch.cuda.synchronize()
    host_avg = np.zeros((edges, 1326), np.float32)
    t0 = time.perf_counter()
    b3 = P.Batch(specs, ranges)
    b3.enable_average()
    for c in range(2):
        b3.set_config(c, cfgs[c]["K"], cfgs[c]["per_sm"], cfgs[c]["order"])
    t1 = time.perf_counter()
    b3.iterate(BATCH_ITERATIONS)
    t2 = time.perf_counter()
    b3.all_rows(1, host_avg)
    t3 = time.perf_counter()
    e2e_s = t3 - t0
    b3.close()
    out["e2e"] = {"solve_s": e2e_s, "iterations": BATCH_ITERATIONS,
                  "iteration_ms": e2e_s / BATCH_ITERATIONS * 1e3,
                  "setup_s": t1 - t0, "iterate_s": t2 - t1, "download_s": t3 - t2,
                  "h2d_bytes": int(specs.nbytes + ranges.nbytes), "d2h_bytes": int(host_avg.nbytes),
                  "note": "batch set-up, 500 CFR iterations and the download of every average sum"}
    if with_cpu:
        out["cpu_baseline"] = batch_cpu_sample(specs, ranges, cpu_threads)
    return out


def adjoint_section(P, peak, cpu_threads, with_cpu):
    """The adjoint pair on 1024 general river subgames at their average strategies
    after 100 CFR iterations. Forward V = r0^T U(sigma) r1 (pr_batch_value), backward dV/dr0,
    dV/dr1 and dV/dsigma at the root (pr_batch_value_grad), both through the C ABI with their
    host outputs; algorithmic bytes sum_s (2 E_s 1081 4 + 4 1081 4) per forward + backward."""
    specs, ranges = P.random_subgames(1024, seed=777)
    b = P.Batch(specs, ranges)
    b.enable_average()
    b.set_linear_average(True)
    b.iterate(100)
    edges = sum(b.shape(i)[1] for i in range(b.count))
    b.value(use_average=True)
    b.value_grad(use_average=True)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        b.value(use_average=True)
    fwd = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        b.value_grad(use_average=True)
    bwd = (time.perf_counter() - t0) / reps
    # the backward with device outputs (no host copies of the gradients)
    import torch
    d0 = torch.zeros((b.count, 1326), dtype=torch.float64, device="cuda")
    d1 = torch.zeros_like(d0)
    ds = torch.zeros((b.count, 8, 1326), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    b.value_grad_device(d0, d1, ds, use_average=True)
    t0 = time.perf_counter()
    for _ in range(reps):
        b.value_grad_device(d0, d1, ds, use_average=True)
    bwd_dev = (time.perf_counter() - t0) / reps
    nbytes = 2.0 * edges * 1081 * 4 + b.count * 4.0 * 1081 * 4
    out = {"workload": "1024 general river subgames (random_subgames: pots 2-200, 1-3 bets and raises), average strategies after 100 CFR iterations",
           "forward_ms": fwd * 1e3, "backward_ms": bwd * 1e3, "backward_device_outputs_ms": bwd_dev * 1e3,
           "roofline": {"bound": "hbm", "achieved": nbytes / (fwd + bwd_dev) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": nbytes / (fwd + bwd_dev) / 1e9 / peak, "bytes_fwd_bwd": nbytes,
                        "note": "forward + backward with device outputs; backward_ms adds the host copies "
                                "of the gradients ([1024][10][1326] doubles)"}}
    if with_cpu:
        out["cpu_baseline"] = adjoint_cpu_sample(b, specs, ranges, cpu_threads)
    b.close()
    return out


def adjoint_cpu_sample(b, specs, ranges, threads):
    """The oracle's double-precision strategy evaluation of both players (the values the
    forward and backward pair return) from the device's average sums, on a sample of the
    subgames sized to about 10 s, scaled to the batch."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O

    def timed(idx):
        subs = []
        for s in idx:
            sp = specs[s]
            o = O.Subgame(int(sp["board"]), float(sp["pot"]), float(sp["stack"]), int(sp["sizes"]),
                          int(sp["max_raises"]), ranges[s, 0], ranges[s, 1])
            o.average = b.average(int(s))
            subs.append(o)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda o: (o.value(0, True), o.value(1, True)), subs))
        return time.perf_counter() - t0

    probe = max(threads, 8)
    dt = timed(range(probe))
    n = int(min(b.count, max(probe, probe * 10.0 / max(dt, 1e-6))))
    dt = timed(range(n))
    return {"fwd_bwd_ms": dt * b.count / n * 1e3, "cores": threads, "kind": "port",
            "sample": f"{n} of {b.count} subgames, both players' FP64 evaluations, {dt:.2f} s, scaled"}


def full_game_section(P, traces):
    """The full fixed-flop game with general bets (flop and turn sweeps over batched river
    subgames): CFR iteration time, river subgames solved per second, iterations / solver
    seconds until the FP64 exploitability of the average strategies is at most 0.5 % of the
    starting pot, and the iteration time with value-network leaves (untrained network: the
    time does not depend on the weights)."""
    from pokerrust_b200 import full_solve as FS
    spec, ranges = FS.seeded_game("small", 7)
    pot = FS.CONFIGS["small"]["pot"]
    g = P.FullGame(spec, ranges)
    g.tune()
    g.iterate(3)  # the first iteration runs eagerly, then one iteration is captured as a graph
    steps = 20
    t0 = time.perf_counter()
    g.iterate(steps)
    it_s = (time.perf_counter() - t0) / steps
    out = {
        "workload": "fixed flop (seed 7), pot 10, stacks 100, flop and turn bets 0.75 pot / all-in with one "
                    "bet or raise per street, river subgames with 0.5 / 1 pot bets and two raises; ranges "
                    "U(0,1) with 30 % zeroed",
        "nodes": g.nodes, "leaves": g.leaves, "river_subgames": g.bet_subgames + g.allin_subgames,
        "iteration_ms": it_s * 1e3,
        "river_subgame_solves_per_s": 2 * (g.bet_subgames + g.allin_subgames) / it_s,
    }
    g.reset()
    pts, reached = FS.trajectory(g, 300, 50, pot, 0.5)
    if traces:
        out["exploitability_pct_pot"] = [(p["iterations"], round(p["pct_pot"], 4)) for p in pts]
    out["time_to_0.5pct_pot"] = reached
    net = P.ValueNet(rows=512, seed=1)
    g.set_net(net)
    g.iterate(2)
    t0 = time.perf_counter()
    g.iterate(steps)
    out["net_leaf_iteration_ms"] = (time.perf_counter() - t0) / steps * 1e3
    g.set_net(None)
    net.close()
    g.close()
    return out


def torch_gemm_baseline(P, rows):
    """Library context for the training step: torch's BF16 matmuls (cuBLAS) of the step's 15
    GEMM shapes (5 forward, 5 + 5 backward), with no element-wise work, timed with CUDA
    events."""
    import torch
    shapes = [P.ValueNet.layer_shape(l) for l in range(5)]  # (out, in)
    g = torch.Generator(device="cuda").manual_seed(0)
    mk = lambda *sh: torch.randn(*sh, device="cuda", dtype=torch.bfloat16, generator=g)
    xs = [mk(rows, i) for o, i in shapes]
    ws = [mk(o, i) for o, i in shapes]
    dys = [mk(rows, o) for o, i in shapes]

    def step():
        for x, w in zip(xs, ws):
            torch.matmul(x, w.t())
        for x, w, dy in zip(xs, ws, dys):
            torch.matmul(dy, w)
            torch.matmul(dy.t(), x)

    for _ in range(3):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 20


def value_net_section(P, peak_tflops, peak_sustained, traces):
    """The turn-leaf value network: tensor-core throughput of training steps at batch 4096
    (random inputs; 6 x 8.64 M x 4096 FLOP per step), torch's BF16 GEMMs of the same shapes as
    library context, and a small train / held-out run on river-solver data against the
    baselines it replaces."""
    import torch
    from pokerrust_b200 import train_value_net as T
    rows = 4096
    net = P.ValueNet(rows=rows, seed=11)
    g = torch.Generator(device="cuda").manual_seed(5)
    ranges = torch.rand((rows, 2, 1326), device="cuda", generator=g) / 600.0
    boards = torch.randint(0, 1 << 20, (rows,), device="cuda", dtype=torch.int64, generator=g)
    scalars = torch.rand((rows, 2), device="cuda", generator=g)
    targets = torch.randn((rows, 2652), device="cuda", generator=g) * 0.1
    for _ in range(3):
        net.train_step(ranges, boards, scalars, targets, 1e-4)
    torch.cuda.synchronize()
    steps = 20
    t0 = time.perf_counter()
    for _ in range(steps):
        net.train_step(ranges, boards, scalars, targets, 1e-4)
    step_s = (time.perf_counter() - t0) / steps
    params = sum(o * i + o for o, i in (P.ValueNet.layer_shape(l) for l in range(5)))
    flops = 6.0 * params * rows
    net.close()
    lib_ms = torch_gemm_baseline(P, rows)
    small = T.run(train_n=768, test_n=256, iterations=60, cheap=3, epochs=40, batch=256, lr=1e-3, seed=1)
    if not traces:
        small["train"].pop("loss_curve", None)
    return {
        "train_step_ms": step_s * 1e3, "batch": rows, "parameters": params,
        "tensor": {"achieved_tflops": flops / step_s / 1e12, "peak": peak_sustained,
                   "frac": flops / step_s / 1e12 / peak_sustained,
                   "note": "whole training step (15 GEMMs + element-wise kernels) over the measured sustained "
                           "BF16 peak"},
        "library_context": {"torch_bf16_gemms_ms": lib_ms, "tflops": flops / (lib_ms / 1e3) / 1e12,
                            "note": "torch.matmul (cuBLAS) of the step's 15 GEMM shapes only, no bias, GELU, "
                                    "loss or Adam: a lower bound for a library-built step"},
        "heldout": small,
    }


def batch_cpu_sample(specs, ranges, threads):
    """The oracle's per-hand CFR (one thread per subgame) on a sample of the subgames, one
    iteration each, scaled to the whole batch."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    def timed(n):
        subs = [O.Subgame(int(s["board"]), float(s["pot"]), float(s["stack"]), int(s["sizes"]),
                          int(s["max_raises"]), r[0], r[1]) for s, r in zip(specs[:n], ranges[:n])]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda o: o.iterate(1), subs))
        return time.perf_counter() - t0

    # a probe of one subgame per thread, then a sample sized to about 10 s
    probe = max(threads, 8)
    dt = timed(probe)
    n = int(min(len(specs), max(probe, probe * 10.0 / max(dt, 1e-6))))
    dt = timed(n)
    per_iter = dt * len(specs) / n
    return {"iteration_ms": per_iter * 1e3, "cores": threads, "kind": "port",
            "sample": f"{n} of {len(specs)} subgames, one iteration, {dt:.2f} s, scaled"}


def max_over_ranks(x, world, device):
    """The largest of the ranks' values (the slowest rank's time); the value itself at N = 1."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, max_seconds):
    """Whole-job throughput of N replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / max_seconds


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O  # the reference's CPU path (restated), timed here
    nthreads = os.cpu_count() or 1
    game = O.Game(O.REFERENCE_FLOP, nthreads)
    boards, bets = game.river_roots()
    ranges = uniform_ranges(O.card_order(), boards)
    tables = O.pack_flop_tables(O.REFERENCE_FLOP, nthreads)
    # each timed step is a bounded sample (about 10 s, less for long runs) of the pass
    per_step = min(10.0, 150.0 / max(1, args.steps))
    sample = sized_sample(boards, bets, ranges, tables, nthreads, per_step)
    for _ in range(args.warmup):
        cpu_sample(boards, bets, ranges, tables, nthreads, max(nthreads, 8))
    rates, times = [], []
    for _ in range(args.steps):
        r, dt = cpu_sample(boards, bets, ranges, tables, nthreads, sample)
        rates.append(r)
        times.append(dt)
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": bench_config(SUBGAMES, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"each timed step is {sample} of the {SUBGAMES} river subgames "
                                   f"({float(np.mean(times)):.2f} s of wall time, ms_per_step); value = "
                                   "their node visits / that time"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch_profile(args):
    """The batched solver alone (for profiling): args.batch_profile subgames, warm-up and
    timed CFR iterations, one JSON line."""
    import torch
    rank, _, local = dist_env()
    torch.cuda.set_device(local)
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(args.batch_profile, seed=4321 + rank)
    b = P.Batch(specs, ranges)
    b.enable_average()
    if args.batch_config:
        K, per_sm = (int(x) for x in args.batch_config.split(","))
        for c in range(2):
            if b.config(c)["count"]:
                b.set_config(c, K, per_sm, 0)
    b.iterate(max(2, args.warmup))
    t0 = time.perf_counter()
    b.iterate(args.steps)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    nbytes = b.iteration_bytes()
    print(json.dumps({"batch_profile": True, "subgames": args.batch_profile, "iteration_ms": dt * 1e3,
                      "achieved_gbs": nbytes / dt / 1e9, "bytes_per_iteration": nbytes}), flush=True)
    b.close()
    return 0


def run_full_profile(args):
    """The full fixed-flop game alone (for profiling): the bench's full game, warm-up and
    timed CFR iterations (one CUDA graph each), one JSON line."""
    import torch
    _, _, local = dist_env()
    torch.cuda.set_device(local)
    import pokerrust_b200 as P
    from pokerrust_b200 import full_solve as FS
    spec, ranges = FS.seeded_game("small", 7)
    g = P.FullGame(spec, ranges)
    g.tune()
    g.iterate(max(2, args.warmup))
    t0 = time.perf_counter()
    g.iterate(args.steps)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    print(json.dumps({"full_profile": True, "nodes": g.nodes, "river_subgames": g.bet_subgames + g.allin_subgames,
                      "iteration_ms": dt * 1e3}), flush=True)
    g.close()
    return 0


def run_net_profile(args):
    """The value network alone (for profiling): training steps at batch 4096 on random data."""
    import torch
    _, _, local = dist_env()
    torch.cuda.set_device(local)
    import pokerrust_b200 as P
    rows = 4096
    net = P.ValueNet(rows=rows, seed=11)
    g = torch.Generator(device="cuda").manual_seed(5)
    ranges = torch.rand((rows, 2, 1326), device="cuda", generator=g) / 600.0
    boards = torch.randint(0, 1 << 20, (rows,), device="cuda", dtype=torch.int64, generator=g)
    scalars = torch.rand((rows, 2), device="cuda", generator=g)
    targets = torch.randn((rows, 2652), device="cuda", generator=g) * 0.1
    for _ in range(args.warmup):
        net.train_step(ranges, boards, scalars, targets, 1e-4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.train_step(ranges, boards, scalars, targets, 1e-4)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    print(json.dumps({"net_profile": True, "batch": rows, "train_step_ms": dt * 1e3}), flush=True)
    net.close()
    return 0


def run_gpu(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import pokerrust_b200 as P

    # the game, its river roots and its hand-rank tables, all built by the library
    game = P.Game(REFERENCE_FLOP)
    boards, bets = game.river_roots()
    tables = game.tables
    if args.subgames:
        boards, bets = boards[:args.subgames], bets[:args.subgames]
        builder = P.Builder()
        for cards, bt in zip(boards, bets):
            builder.add(int(cards), float(bt))
    else:
        builder = P.Builder.wrap(game.builder)   # owned by the game
    n = len(boards)
    ranges = uniform_ranges(P.card_order(), boards)
    stride = P.RANGE_STRIDE
    d_ranges = torch.zeros((n, stride), dtype=torch.float32, device=dev)
    d_ranges[:, :1326] = torch.from_numpy(ranges).to(dev)
    d_results = torch.zeros((n, stride), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(dev)  # a real stream handle: the library launches on it
    torch.cuda.set_stream(stream)

    def step(i):
        builder.evaluate_device(tables, i % 2, False, d_ranges.data_ptr(), d_results.data_ptr(),
                                stream.cuda_stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    for i in range(args.warmup):
        step(i)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    kernel_ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(kernel_ms, world, dev)
    value = replica_rate(n * NODES_PER_SUBGAME, world, ms / 1e3)

    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "subgames": n, "kernel_ms": kernel_ms,
                              "value": value, "unit": UNIT}), flush=True)
        if args.subgames:
            builder.close()
        game.close()
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # end to end through the C ABI with host buffers (the caller's input and output rows are
    # allocated once and reused every pass)
    host_in = np.ascontiguousarray(ranges)
    out = np.zeros((n, 1326), np.float32)
    for i in range(max(1, args.warmup // 2)):
        builder.upload_all(host_in)
        P.evaluate_gpu(builder.ptr, tables, i % 2, False)
        builder.download_all(out)
    barrier()
    e_steps = max(2, min(args.steps, 10))
    t0 = time.perf_counter()
    for i in range(e_steps):
        builder.upload_all(host_in)
        P.evaluate_gpu(builder.ptr, tables, i % 2, False)
        builder.download_all(out)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e_steps, world, dev)
    assert np.all(np.isfinite(out))

    # whole-game CFR iterations through the library's game driver (game.rs:68-119): the
    # upper tree on the device (one CUDA graph per iteration), then on the host through the
    # reference's upload / evaluate_cuda / download protocol
    torch.cuda.synchronize(dev)
    game.set_device_tree(True)
    game.iterate(2)  # first iteration eager, then the graph is captured
    t0 = time.perf_counter()
    game.iterate(4)
    dev_iter_s = (time.perf_counter() - t0) / 4
    game.set_device_tree(False)
    game.iterate(1)
    h0, d0 = game.timings()
    t0 = time.perf_counter()
    game.iterate(2)
    iter_s = (time.perf_counter() - t0) / 2
    h1, d1 = game.timings()
    game.set_device_tree(True)

    cpu_threads = os.cpu_count() or 1
    batch = batch_section(P, rank, measured_peaks()[0], cpu_threads, rank == 0, args.traces)
    tp = tensor_peaks()
    vnet = value_net_section(P, tp[0], tp[1], args.traces)
    full = full_game_section(P, args.traces)
    adj = adjoint_section(P, measured_peaks()[0], cpu_threads, rank == 0)

    line = None
    if rank == 0:
        from oracle import oracle as O  # CPU baseline only
        peak, peak_kind = measured_peaks()
        ab = algorithmic_bytes(n)
        achieved = ab / (kernel_ms / 1e3) / 1e9
        tables_host = O.pack_flop_tables(O.REFERENCE_FLOP, cpu_threads)
        cpu_n = sized_sample(boards, bets, ranges, tables_host, cpu_threads, 10.0)
        cpu_rate, cpu_dt = cpu_sample(boards, bets, ranges, tables_host, cpu_threads, cpu_n)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(n, world),
            "e2e": {"value": world * n * NODES_PER_SUBGAME / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": int(n * 1328 * 4), "d2h_bytes_per_step": int(n * 1328 * 4),
                    "ms_per_step": e2e_s * 1e3},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": TRAFFIC_PER_LAUNCH if n == SUBGAMES else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one full "
                                           "launch of this program",
                         "peak_source": peak_kind,
                         "note": "algorithmic bytes per pass / kernel time; the pass is bound "
                                 "on-chip (shared memory and issue), not by HBM",
                         "onchip": {"bound": "shared-memory data pipe", "frac": SMEM_PIPE_FRAC,
                                    "wavefronts_per_river_card": round(SMEM_WAVEFRONTS_PER_RIVER_CARD),
                                    "source": "ncu l1tex__data_pipe_lsu_wavefronts_mem_shared, "
                                              "one 4096-subgame CFR pass"}},
            "cpu_baseline": {"value": cpu_rate, "unit": UNIT, "cores": cpu_threads, "kind": "port",
                             "sample": f"{cpu_n} of {n} river subgames, one pass, "
                                       f"{cpu_dt:.2f} s, scaled to nodes/s"},
            "gpu_launches": args.steps,
            "clocks": clk,
            "batch_subgames": batch,
            "value_network": vnet,
            "full_game": full,
            "adjoint": adj,
            "game_iteration": {"ms": dev_iter_s * 1e3,
                               "note": "one full CFR iteration of the fixed-flop game (both players): "
                                       "upper tree and river passes on the device, one CUDA graph",
                               "host_tree": {"ms": iter_s * 1e3, "host_ms": (h1 - h0) / 2 * 1e3,
                                             "device_ms": (d1 - d0) / 2 * 1e3,
                                             "note": "upper tree on the host, river passes through "
                                                     "upload_c / evaluate_cuda / download_c"}},
        }
        print(json.dumps(line), flush=True)
    if args.subgames:
        builder.close()
    game.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch-profile", type=int, default=0,
                    help="only the batched general subgames: this many, a few timed iterations")
    ap.add_argument("--batch-config", default="",
                    help="with --batch-profile: hands per thread and CTAs per SM for both shape classes, e.g. 4,3")
    ap.add_argument("--net-profile", action="store_true",
                    help="only the value network: warm-up and timed training steps at batch 4096")
    ap.add_argument("--full-profile", action="store_true",
                    help="only the full fixed-flop game with general bets: warm-up and timed CFR iterations")
    ap.add_argument("--subgames", type=int, default=0,
                    help="use the first N river roots only (profiling runs); 0 = all 27783")
    ap.add_argument("--profile", action="store_true",
                    help="kernel timing only: skip the end-to-end and CPU-baseline legs")
    ap.add_argument("--traces", action="store_true",
                    help="add exploitability trajectories and loss curves to the JSON line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.batch_profile:
        return run_batch_profile(args)
    if args.net_profile:
        return run_net_profile(args)
    if args.full_profile:
        return run_full_profile(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
