#!/usr/bin/env python
"""Benchmark of the BIA pair step: pair-updates/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload coulomb_cube_32768] [--method alg|rkf]

A step is one BIA step of the workload (all N(N-1)/2 pairs, reduction, drift and state
update).  Default workload: the plain FP64 BIA step of the Coulomb system, N = 32768,
charges +-1, unit cube, Maxwellian sigma = 1, dt = 1e-5 (seeded synthetic input).  One
JSON line is printed by rank 0.

  value     pair-updates/s with the state resident in HBM: K steps, each bracketed by
            CUDA events on the solver's stream, an untimed 256 MB L2 flush between steps
  e2e       the same through the host-buffer call (bia_run_host): every step copies the
            state and charges from pinned host memory and the state back
  roofline  FP64 roofline of the dominant kernel (bia_pair_tiles_kernel): algorithmic
            FP64 flops per launch (per-branch counts of this run times the per-pair flop
            model below) over the kernel's event-timed duration, against the DFMA peak
            measured on the same GPU by bia_measure_fp64_peak
  cpu_baseline  the CPU oracle (a C restatement of the reference's CPU path), OpenMP
            on all host cores, on a seeded sample of rows i (all j > i) of the workload

--impl reference times the reference's CPU implementation of the path: its Fortran
sources cannot be compiled on this image (no Fortran compiler), so the C restatement
runs in its place, on all host cores, a bounded row sample per step.
Multi-GPU (torchrun): every rank runs its own replica of the workload (the reference
runs on one GPU; replicas only), timing is the max over ranks.
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# Algorithmic FP64 flops per pair (convention: + - * / sqrt = 1, FMA = 2, each libm
# transcendental = 20, sincos = 40), counted from the reference's formulas:
# base cost per pair of each branch (frame + classification + solve set-up + finish +
# half-displacement + accumulation) and the cost of one solver iteration.
FLOPS = {
    "hyperbola": (661, 125),   # per pair, per main-loop Newton iteration
    "ellipse": (447, 47),      # per pair, per Kepler Newton step
    "parabola": (429, 76),     # per pair, per Barker Newton step
    "rkf": (147, 758),         # per pair, per accepted RKF45 step (3 Fehlberg stages sets)
    "universal": (145, 74),    # per pair, per universal-variable Newton iteration
}

# DRAM traffic per launch of bia_pair_tiles_kernel at the default workload, from the
# ncu capture summarised in profiles/ (None until captured).
TRAFFIC_BYTES_PER_LAUNCH = None


def pair_flops(stats, method):
    h, e, p, r = FLOPS["hyperbola"], FLOPS["ellipse"], FLOPS["parabola"], FLOPS["rkf"]
    u = FLOPS["universal"]
    deg_rkf = stats["degenerate"] if method == 0 else 0
    deg_uv = stats["degenerate"] - deg_rkf
    return (stats["hyperbola"] * h[0] + stats["iter_hyperbola"] * h[1] +
            stats["ellipse"] * e[0] + stats["iter_ellipse"] * e[1] +
            stats["parabola"] * p[0] + stats["iter_parabola"] * p[1] +
            (stats["rkf"] + deg_rkf) * r[0] + stats["rkf_steps"] * r[1] +
            (stats["universal"] + deg_uv) * u[0] + stats["iter_universal"] * u[1])


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="coulomb_cube_32768")
    ap.add_argument("--n", type=int, default=None, help="override the particle count")
    ap.add_argument("--method", choices=("alg", "rkf", "universal"), default="alg")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_sample(state, eps, q, dt, method, seconds, seed=0):
    """Time the oracle on a seeded row sample sized to about `seconds` of host work."""
    import oracle
    n = state.shape[1]
    rng = np.random.default_rng(seed)
    threads = os.cpu_count() or 1
    rows = rng.choice(n - 1, size=min(n - 1, max(threads, 8)), replace=False)
    t0 = time.perf_counter()
    _, pairs, _ = oracle.bia_rows(state, eps, dt, rows, method=method, q=q, nthreads=threads)
    rate = pairs / max(time.perf_counter() - t0, 1e-9)
    mean_pairs = n / 2
    nrows = int(min(n - 1, max(threads, rate * seconds / mean_pairs)))
    rows = rng.choice(n - 1, size=nrows, replace=False)
    t0 = time.perf_counter()
    _, pairs, _ = oracle.bia_rows(state, eps, dt, rows, method=method, q=q, nthreads=threads)
    el = time.perf_counter() - t0
    return pairs / el, threads, f"{nrows} seeded rows i (all j > i), {pairs} pairs, {el:.1f} s"


def run_reference(args, rank, world):
    """The reference's CPU path (C restatement of its Fortran) on all host cores."""
    if rank != 0:
        return
    from bia_3d_gpu_b200 import initial
    state, eps, q, dt, steps_cfg = initial.make(args.workload, n=args.n)
    method = {"rkf": 0, "alg": 1, "universal": 2}[args.method]
    steps = args.steps if args.steps is not None else steps_cfg
    per_step = max(0.5, min(3.0, 120.0 / max(1, steps + args.warmup)))
    for w in range(args.warmup):
        cpu_sample(state, eps, q, dt, method, per_step * 0.3, seed=1000 + w)
    rates = []
    info = None
    for k in range(steps):
        r, cores, info = cpu_sample(state, eps, q, dt, method, per_step, seed=k)
        rates.append(r)
    value = float(np.median(rates))
    n = state.shape[1]
    line = {
        "metric": "BIA pair-updates/s (plain FP64 step)", "impl": "reference",
        "value": value, "unit": "pair-updates/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "n": n, "pairs_per_step": n * (n - 1) // 2,
                   "dt": dt, "method": args.method},
        "cpu_baseline": {"value": value, "unit": "pair-updates/s", "cores": cores, "kind": "port",
                         "sample": f"per step: {info}; the reference's Fortran CPU path "
                                   "cannot be compiled here, its C restatement runs instead"},
        "e2e": {"value": value, "unit": "pair-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    from bia_3d_gpu_b200 import BIASolver, default_config, initial, measure_fp64_peak

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    state, eps, q, dt, steps_cfg = initial.make(args.workload, n=args.n)
    n = state.shape[1]
    pairs = n * (n - 1) // 2
    steps = args.steps if args.steps is not None else steps_cfg
    method = {"rkf": 0, "alg": 1, "universal": 2}[args.method]
    cfg = default_config(eps_th=eps, dt=dt, method=method)
    dev = torch.device("cuda", local)
    solver = BIASolver(device=local)
    stream = solver.stream
    d_state = torch.tensor(state, device=dev)
    d_q = torch.tensor(q, device=dev) if q is not None else None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    # warm-up (untimed): kernels loaded, buffers allocated
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            solver.step(d_state, cfg, q=d_q, stats=False)
    solver.counters(reset=True)
    solver.set_timing(True)
    solver.kernel_ms()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()                      # untimed L2 flush (256 MB > 126 MB L2)
            ev[k][0].record(stream)
            solver.step(d_state, cfg, q=d_q, stats=False)
            ev[k][1].record(stream)
    barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    kern_ms, kern_launches = solver.kernel_ms()
    solver.set_timing(False)
    stats = solver.counters(reset=True)
    if dist is not None:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * steps * pairs / (total_ms * 1e-3)

    # end-to-end through the host-buffer call with pinned host memory
    e2e = None
    if not args.no_e2e:
        h_state = torch.tensor(state).pin_memory()
        h_q = torch.tensor(q).pin_memory() if q is not None else None
        hs = h_state.numpy()
        hq = h_q.numpy() if h_q is not None else None
        solver.run_host(hs, cfg, 1, q=hq)      # warm: host-path graph built
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(steps):
            solver.run_host(hs, cfg, 1, q=hq)
        e1.record(stream)
        barrier()
        wall = time.perf_counter() - t0
        e2e_ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        h2d = 6 * n * 8 + (n * 8 if q is not None else 0)
        e2e = {"value": world * steps * pairs / (e2e_ms * 1e-3), "unit": "pair-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 6 * n * 8,
               "wall_s": wall}

    # roofline of the pair kernel
    flops_total = pair_flops(stats, method)
    per_launch_flops = flops_total / max(kern_launches, 1)
    per_launch_s = kern_ms * 1e-3 / max(kern_launches, 1)
    peak = measure_fp64_peak(local)
    achieved = per_launch_flops / per_launch_s / 1e12
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "traffic": TRAFFIC_BYTES_PER_LAUNCH,
                "peak_source": "measured live: bia_measure_fp64_peak DFMA loop on this GPU",
                "flops_per_launch": per_launch_flops, "kernel_ms_per_launch": per_launch_s * 1e3,
                "kernel": "bia_pair_tiles_kernel<true>"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample = cpu_sample(state, eps, q, dt, method, args.cpu_seconds)
        cpu = {"value": v, "unit": "pair-updates/s", "cores": cores, "kind": "port",
               "sample": sample}

    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": "BIA pair-updates/s (plain FP64 step)", "value": value,
            "unit": "pair-updates/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": total_ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "n": n, "pairs_per_step": pairs, "dt": dt,
                       "method": args.method, "reduction": "deterministic",
                       "l2": "256 MB buffer written between timed steps (untimed)",
                       "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": 2 * steps,
            "stats": {k: v for k, v in stats.items()},
            "iterations_per_classical_pair": stats["iterations"] / max(
                1, stats["hyperbola"] + stats["ellipse"] + stats["parabola"]),
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
