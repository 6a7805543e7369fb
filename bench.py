#!/usr/bin/env python
"""Benchmark of the BIA pair step: pair-updates/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plummer_32768] [--method learned|alg|universal|rkf]

A step is one BIA step of the workload (all N(N-1)/2 pairs, reduction, drift and state
update).  Default: the learned mixed-precision form (METHOD_LEARNED) on the Plummer sphere,
N = 32768, G = M = 1, equal masses, dt = 1e-4 (seeded synthetic input), beside the plain
FP64 form (the reference's ALG algorithm) timed the same way in the same run.  One JSON
line is printed by rank 0.

  value     pair-updates/s with the state resident in HBM: K steps, each from the seeded
            state, each bracketed by CUDA events on the solver's stream, an untimed 256 MB
            L2 flush between steps
  e2e       the same through the host-buffer call (bia_run_host): K consecutive steps from
            the seeded state, every step copying the state (and charges) from pinned host
            memory and the new state back
  plain_fp64  the plain FP64 ALG form on the same workload, its speed-up ratio, and the
            one-step distance of the measured form from it (global relative, positions and
            velocities)
  roofline  FP64 roofline of the dominant kernel: algorithmic FP64 flops per launch
            (per-branch counts of this run times the per-pair flop model below) over the
            kernel's event-timed duration, against the DFMA peak measured on the same GPU
            by bia_measure_fp64_peak
  cpu_baseline  the CPU oracle (a C restatement of the reference's CPU ALG path), OpenMP
            on all host cores, on a seeded sample of rows i (all j > i) of the workload

Other workloads (own JSON line each):
  --workload plummer_ensemble_4096  4096 independent Plummer systems, N_s uniform in
            [32, 1024] (seeded), eps_s = -2/N_s, dt = 1e-4, 200 steps captured in one CUDA
            graph: systems-steps/s, pair-updates/s and per-system energy drift
  --workload dim_lattice_1332  the direct-integration reference solver (dim/rkf_kernel.cu
            rebuilt) on a seeded 1332-particle lattice, eps = -3e-7, t = 0 -> 1 (the
            reference's own DIM run of this size took 2.946 s on a TITAN V, README.md:41)

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
    # universal variables (this library's solver, not the reference's), counted from the
    # dimensionless series form every exact pair takes: differences 6, prepare 20 (|r|^2,
    # r.g, |g|^2, rsqrt as sqrt + division, beta), series with its exactness test 41,
    # composition with the three-term Stumpff series and the series of r0/r 63, accumulation
    # 12 per pair; 43 per Newton iteration (almost none at the benchmark steps)
    "universal": (142, 43),
    "learned": (330, 0),       # per learned pair: elements, FP64 Halley step, composition
}
# BF16 tensor-core flops per learned pair: 2 x (16 x 64 + 64 x 64 + 64 x 64) multiply-adds
LEARNED_TENSOR_FLOPS = 2 * (16 * 64 + 64 * 64 + 64 * 64)
METHODS = {"rkf": 0, "alg": 1, "universal": 2, "learned": 3}

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the dominant pair
# kernel, from one ncu capture at n = 16384 of the same workload and method, scaled by the
# pairs per launch (both the partial sums and any local-memory traffic grow with the pairs):
#   (workload, method, learned layout) -> (pairs in the capture, bytes in the capture)
# The learned step's dominant kernel is the rest kernel (it writes every partial slot; the head
# and finish kernels move under 1 MB at this size on this workload).
TRAFFIC = {
    ("plummer_32768", 3, "split"): (16384 * 16383 // 2, 1.049e6 + 345.274e6),
    ("coulomb_cube_32768", 1, None): (16384 * 16383 // 2, 3.880e6 + 2105.114e6),  # phase-locked ALG
}


def pair_flops(stats, method):
    """Algorithmic FP64 flops of the counted pairs (learned pairs: their FP64 part; a
    learned pair that fell back is also counted with the universal-variable iterations
    it ran)."""
    h, e, p, r = FLOPS["hyperbola"], FLOPS["ellipse"], FLOPS["parabola"], FLOPS["rkf"]
    u = FLOPS["universal"]
    if method == 3:
        return (stats["learned"] * FLOPS["learned"][0] + stats["universal"] * u[0] +
                stats["degenerate"] * u[0] + stats["iter_universal"] * u[1])
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
    ap.add_argument("--workload", default="plummer_32768")
    ap.add_argument("--n", type=int, default=None, help="override the particle count")
    ap.add_argument("--dt", type=float, default=None, help="override the workload's step length")
    ap.add_argument("--method", choices=("learned", "alg", "rkf", "universal"), default="learned")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--systems", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-universal", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--no-oracle-check", action="store_true", help="skip error_vs_oracle")
    ap.add_argument("--shard", action="store_true",
                    help="split the one system over the ranks (its pairs in shards, the per-particle sums "
                         "all-reduced over NCCL) instead of one replica per rank")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations timed beside the main line")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the library's built-in kernel-shape rules instead of timing the shapes first "
                         "(for profiler runs, whose serialised launches would mislead the autotuner)")
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


def cpu_sample(state, eps, q, dt, method, seconds, seed=0, threads=None):
    """Time the oracle on a seeded row sample sized to about `seconds` of host work, on
    `threads` host threads (default: all cores)."""
    import oracle
    n = state.shape[1]
    rng = np.random.default_rng(seed)
    threads = threads or os.cpu_count() or 1
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
    # the reference has no learned form or universal-variable solver: its CPU ALG path is
    # the reference arm for every method but RKF
    method = {"rkf": 0, "alg": 1, "universal": 1, "learned": 1}[args.method]
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
        "metric": metric_name(args.method), "impl": "reference",
        "value": value, "unit": "pair-updates/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_keys(args.workload, n, dt, "rkf" if method == 0 else "alg", world,
                              reduction="host loop in pair order (bia/bia.f90:141-196)",
                              precision="FP64", l2="host CPU (no GPU)",
                              state="the seeded state for every sampled row"),
        "cpu_baseline": {"value": value, "unit": "pair-updates/s", "cores": cores, "kind": "port",
                         "sample": f"per step: {info}; the reference's Fortran CPU path "
                                   "cannot be compiled here, its C restatement runs instead"},
        "e2e": {"value": value, "unit": "pair-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_keys(workload, n, dt, method, world, reduction, precision, l2, state, autotuned=None, shard=False):
    """The config object of a bench line; both arms print the same keys."""
    return {"workload": workload, "n": n, "pairs_per_step": n * (n - 1) // 2, "dt": dt,
            "method": method, "reduction": reduction, "precision": precision, "l2": l2,
            "state": state, "parallelism": (f"pair shards x{world}, NCCL all-reduce of 6n FP64 per step"
                                            if shard else f"replicas x{world}"),
            "autotuned": autotuned}


def metric_name(method):
    if method == "learned":
        return "BIA pair-updates/s: learned-guess form vs plain FP64, at <=1e-12 pos. error"
    return "BIA pair-updates/s (plain FP64 step)"


def _init_dist(world):
    """The replicas' process group (NCCL on GPUs; gloo where there is none, for the host-only
    checks of the replica timing); None for one process."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist


def _max_over_ranks(dist, value, dev):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ensemble_forms(solver, nsys, steps, warmup, forms, dist=None, dev=None, sample_clocks=False, autotune=True):
    """The batched ensemble (Plummer systems, N_s uniform in [32, 1024], seeded), each form
    in `forms` ((label, method) pairs) autotuned on these systems, then `steps` steps from
    the seeded state replayed from one CUDA graph.  Returns ({label: result}, clocks of the
    first form, system sizes, pairs per step)."""
    import torch

    from bia_3d_gpu_b200 import default_config, initial
    sizes = initial.ensemble_sizes(nsys, 32, 1024, seed=4)
    states = [initial.plummer(int(n), seed=10000 + k)[0] for k, n in enumerate(sizes)]
    eps = -2.0 / sizes.astype(np.float64)
    host = np.ascontiguousarray(np.concatenate(states, axis=1))
    dt = 1e-4
    pairs = int(sum(int(n) * (int(n) - 1) // 2 for n in sizes))
    ens = solver.ensemble(sizes, eps)
    d = torch.tensor(host, device=dev)
    ke0, pe0 = ens.energy(d)
    out, clocks = {}, None
    for k, (label, method) in enumerate(forms):
        c = default_config(dt=dt, method=method)
        tuned = None
        if autotune:
            shape, tms = ens.autotune(d, c)
            tuned = {"shape": shape, "ms": tms}
        with torch.cuda.stream(solver.stream):
            ens.run(d, c, warmup, graph=False, stats=False)     # warm-up (untimed)
        d.copy_(torch.tensor(host, device=dev))
        ens.run(d, c, steps, graph=True, stats=False)              # capture the graph
        d.copy_(torch.tensor(host, device=dev))
        torch.cuda.synchronize()
        solver.counters(reset=True)
        sampler = ClockSampler(dev.index if dev is not None else 0) if (sample_clocks and k == 0) else None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        e0.record(solver.stream)
        ens.run(d, c, steps, graph=True, stats=False)
        e1.record(solver.stream)
        torch.cuda.synchronize()
        if sampler:
            clocks = sampler.stop()
        t_ms = _max_over_ranks(dist, e0.elapsed_time(e1), dev)
        counters = solver.counters(reset=True)
        ke1, pe1 = ens.energy(d)
        dr = np.abs((ke1 + pe1) / (ke0 + pe0) - 1)
        d.copy_(torch.tensor(host, device=dev))
        out[label] = {"ms_per_step": t_ms / steps, "systems_steps_per_s": nsys * steps / (t_ms * 1e-3),
                      "pair_updates_per_s": pairs * steps / (t_ms * 1e-3), "autotuned": tuned,
                      "newton_iterations": newton_per_pair(counters, method),
                      "energy_drift": {"max": float(dr.max()), "median": float(np.median(dr)),
                                       "p99": float(np.quantile(dr, 0.99))},
                      "stats": counters}
    ens.close()
    return out, clocks, sizes, pairs


def run_ensemble(args, rank, world, local):
    """The batched ensemble: 4096 independent Plummer systems of uneven size, 200 steps in
    one CUDA graph (one pair-kernel launch per step over all systems, two for the learned
    form), each form's launch shape chosen by the ensemble autotuner first."""
    import torch

    from bia_3d_gpu_b200 import BIASolver
    dist = _init_dist(world)
    dev = torch.device("cuda", local)
    nsys = args.systems
    steps = args.steps if args.steps is not None else 200
    method = METHODS[args.method]
    solver = BIASolver(device=local)
    solver.load_heads()
    forms = [(args.method, method)]
    if not args.no_plain:
        forms += [(lbl, m) for lbl, m in (("alg", 1), ("universal", 2), ("learned", 3)) if m != method]
    res, clocks, sizes, pairs = ensemble_forms(solver, nsys, steps, args.warmup, forms, dist, dev,
                                               sample_clocks=True, autotune=not args.no_autotune)
    main_r = res[args.method]
    ms = main_r["ms_per_step"] * steps
    if rank == 0:
        line = {
            "metric": "BIA ensemble systems-steps/s (%s step)" % args.method,
            "value": world * nsys * steps / (ms * 1e-3), "unit": "systems-steps/s",
            "pair_updates_per_s": world * pairs * steps / (ms * 1e-3), "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "plummer_ensemble_4096", "systems": nsys,
                       "n_min": int(sizes.min()), "n_max": int(sizes.max()),
                       "particles": int(sizes.sum()), "pairs_per_step": pairs, "dt": 1e-4,
                       "method": args.method, "graph": True,
                       "l2": "per-step working set (partials %.1f GB) exceeds the 126 MB L2"
                             % (sum(6 * 32 * ((int(n) + 31) // 32) ** 2 for n in sizes) * 8e-9),
                       "parallelism": f"replicas x{world}", "autotuned": main_r["autotuned"]},
            "forms": {k: {kk: vv for kk, vv in v.items() if kk != "stats"} for k, v in res.items()},
            "energy_drift": main_r["energy_drift"],
            "clocks": clocks, "gpu_launches": (4 if method == 3 else 2) * steps,
            "stats": main_r["stats"]}
        if "learned" in res:
            best = min(v["ms_per_step"] for k, v in res.items() if k in ("alg", "universal"))
            line["learned_vs_best_plain"] = best / res["learned"]["ms_per_step"]
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


def run_dim(args, rank, world, local):
    """The direct-integration reference solver on the reference's DIM run shape."""
    import torch

    from bia_3d_gpu_b200 import BIASolver, initial
    dist = _init_dist(world)
    dev = torch.device("cuda", local)
    s, _ = initial.lattice(NL=5, seed=0)
    eps = -3e-7
    solver = BIASolver(device=local)
    d = torch.tensor(s, device=dev)
    solver.dim_integrate(d, eps, 0.0, 0.05)                       # warm-up (untimed)
    d.copy_(torch.tensor(s, device=dev))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = solver.dim_integrate(d, eps, 0.0, 1.0)
    torch.cuda.synchronize()
    wall = _max_over_ranks(dist, time.perf_counter() - t0, dev)
    inv0 = solver.invariance(torch.tensor(s, device=dev), 2 * eps)
    inv1 = solver.invariance(d, 2 * eps)
    e0, e1 = inv0["KE"] + inv0["PE"], inv1["KE"] + inv1["PE"]
    if rank == 0:
        print(json.dumps({
            "metric": "DIM RKF45 wall-clock, t = 0 -> 1", "value": wall, "unit": "s",
            "n_gpus": world, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice)",
            "config": {"workload": "dim_lattice_1332", "n": s.shape[1], "eps_th": eps,
                       "relerr": 0.0, "abserr": 1e-16},
            "accepted_steps": st["accepted"], "rejected_steps": st["rejected"],
            "derivative_evaluations": st["nde"], "energy_error": e1 / e0 - 1,
            "reference_published": {"value": 2.946, "unit": "s", "hardware": "TITAN V",
                                    "source": "README.md:41"}}), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


class StepTimer:
    """Times BIA steps of one configuration on the solver's stream: every step starts from
    the seeded state (untimed device copy) after an untimed write of a 256 MB buffer (L2
    flush), and is bracketed by CUDA events on the solver's stream; max over ranks."""

    def __init__(self, solver, dist, dev, local):
        import torch
        self.torch = torch
        self.solver = solver
        self.dist = dist
        self.dev = dev
        self.local = local
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier(self):
        self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()
            self.torch.cuda.synchronize()

    def time(self, d_init, cfg, d_q, k_steps, warmup, sample_clocks=False, step=None):
        """Returns (total ms over k_steps, clocks, counters, (kernel ms, kernel launches)).
        step (optional): the step call, step(state, cfg, q); default BIASolver.step."""
        torch, solver = self.torch, self.solver
        stream = solver.stream
        if step is None:
            def step(st, c, q):
                solver.step(st, c, q=q, stats=False)
        d_state = d_init.clone()
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                d_state.copy_(d_init)
                step(d_state, cfg, d_q)
        solver.counters(reset=True)
        solver.set_timing(True)
        solver.kernel_ms()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k_steps)]
        sampler = ClockSampler(self.local) if sample_clocks else None
        self.barrier()
        if sampler:
            sampler.start()
        with torch.cuda.stream(stream):
            for k in range(k_steps):
                d_state.copy_(d_init)              # untimed: every step starts from the seeded state
                self.flush.zero_()                 # untimed L2 flush (256 MB > 126 MB L2)
                ev[k][0].record(stream)
                step(d_state, cfg, d_q)
                ev[k][1].record(stream)
        self.barrier()
        clk = sampler.stop() if sampler else None
        total = float(sum(a.elapsed_time(b) for a, b in ev))
        kern = solver.kernel_ms()
        solver.set_timing(False)
        counters = solver.counters(reset=True)
        return _max_over_ranks(self.dist, total, self.dev), clk, counters, kern

    def graph_run(self, d_init, cfg, d_q, steps):
        """`steps` consecutive steps (a trajectory) replayed from one CUDA graph; returns
        (ms, counters)."""
        torch, solver = self.torch, self.solver
        stream = solver.stream
        t = d_init.clone()
        with torch.cuda.stream(stream):
            solver.run(t, cfg, steps, q=d_q, graph=True, stats=False)   # capture and warm
            t.copy_(d_init)
        solver.counters(reset=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.barrier()
        with torch.cuda.stream(stream):
            e0.record(stream)
            solver.run(t, cfg, steps, q=d_q, graph=True, stats=False)
            e1.record(stream)
        self.barrier()
        return _max_over_ranks(self.dist, e0.elapsed_time(e1), self.dev), solver.counters(reset=True)


def newton_per_pair(st, method):
    """Newton iterations per pair of each solver a step of `method` ran (from its counters)."""
    classical = st["hyperbola"] + st["ellipse"] + st["parabola"]
    uv_pairs = st["universal"] + st["degenerate"] + st["learned_fallbacks"]
    return {
        "classical_per_pair": st["iterations"] / classical if classical else None,
        "universal_per_pair": st["iter_universal"] / uv_pairs if uv_pairs else None,
        "learned_fp32_per_learned_pair": (st["learned_fp32_steps"] / st["learned"]
                                          if method == 3 and st["learned"] else None),
        "learned_fp64_per_learned_pair": (1.0 if method == 3 and st["learned"] else None),
        "learned_pairs": st["learned"] if method == 3 else None,
    }


def error_vs_oracle(solver, cfg, d_init, d_q, state, eps, q, dt, nsel=16, nquad=6, seed=17):
    """One step of `cfg` from the seeded state, outside any timed region.  The displacement
    of `nsel` seeded particles against the oracle (the reference's FP64 CPU ALG path; max
    error over max|x| and max|v|), and `nquad` of them against the quad-precision oracle (the
    same algorithm without rounding: the exact step), as relative errors of the interaction
    displacement dX - U dt and of the kick dV, each against its own norm.  The FP64 oracle's
    own interaction errors are given beside them."""
    import torch

    import oracle
    t = d_init.clone()
    d = torch.zeros_like(t)
    with torch.cuda.stream(solver.stream):
        solver.step(t, cfg, q=d_q, disp=d, stats=False)
    torch.cuda.synchronize()
    disp = d.cpu().numpy()
    n = state.shape[1]
    sel = np.random.default_rng(seed).choice(n, nsel, replace=False)
    got = disp[:, sel].T
    ref = oracle.particle_disp(state, eps, dt, sel, q=q)
    refq = oracle.particle_disp(state, eps, dt, sel[:nquad], q=q, quad=True)
    drift = state[3:, sel[:nquad]].T * dt

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    return {
        "sample": f"{nsel} seeded particles against the FP64 oracle, {nquad} of them against the quad oracle",
        "pos_max_err_over_max_x": float(np.abs(got[:, :3] - ref[:, :3]).max() / np.abs(state[:3]).max()),
        "vel_max_err_over_max_v": float(np.abs(got[:, 3:] - ref[:, 3:]).max() / np.abs(state[3:]).max()),
        "interaction_dx_rel_err_vs_exact": rel(got[:nquad, :3] - drift, refq[:, :3] - drift),
        # dX = U dt + interaction is stored in FP64, so the interaction part is resolved to
        # half an ulp of dX, not better: an error of 0 means below this
        "interaction_dx_fp64_resolution": float(np.linalg.norm(np.spacing(refq[:, :3]) / 2)
                                                / np.linalg.norm(refq[:, :3] - drift)),
        "dv_rel_err_vs_exact": rel(got[:nquad, 3:], refq[:, 3:]),
        "fp64_oracle_interaction_dx_rel_err_vs_exact": rel(ref[:nquad, :3] - drift, refq[:, :3] - drift),
        "fp64_oracle_dv_rel_err_vs_exact": rel(ref[:nquad, 3:], refq[:, 3:]),
    }


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
    if args.workload == "plummer_ensemble_4096":
        run_ensemble(args, rank, world, local)
        return
    if args.workload == "dim_lattice_1332":
        run_dim(args, rank, world, local)
        return
    dist = _init_dist(world)

    state, eps, q, dt, steps_cfg = initial.make(args.workload, n=args.n)
    if args.dt is not None:
        dt = args.dt
    n = state.shape[1]
    pairs = n * (n - 1) // 2
    steps = args.steps if args.steps is not None else steps_cfg
    method = METHODS[args.method]
    cfg = default_config(eps_th=eps, dt=dt, method=method)
    dev = torch.device("cuda", local)
    solver = BIASolver(device=local)
    solver.load_heads()
    stream = solver.stream
    d_init = torch.tensor(state, device=dev)
    d_state = d_init.clone()
    d_q = torch.tensor(q, device=dev) if q is not None else None
    timer = StepTimer(solver, dist, dev, local)

    # the ALG pair-kernel shape for this size, chosen by the autotuner on this GPU
    tuned = None
    if (method == 1 or (method != 1 and not args.no_plain)) and not args.no_autotune:
        cfg_alg = default_config(eps_th=eps, dt=dt, method=1)
        var, tms = solver.autotune(d_state, cfg_alg, q=d_q)
        tuned = {"alg_shape": ("tiles8", "phase32_lane", "phase32")[var], "ms": tms}
    if method == 3 and not args.no_autotune:
        lvar, lms = solver.autotune(d_state, cfg, q=d_q)
        tuned = dict(tuned or {}, learned_layout=("one_kernel", "split")[lvar], learned_ms=lms)
    shard = args.shard and world > 1
    step_fn = None
    if shard:
        def step_fn(st, c, q):
            solver.step_distributed(st, c, q=q)
    total_ms, clocks, stats, (kern_ms, kern_launches) = timer.time(d_init, cfg, d_q, steps, args.warmup,
                                                                   sample_clocks=True, step=step_fn)
    # replicas: every rank advances its own copy of the system; shards: the ranks split one
    value = (1 if shard else world) * steps * pairs / (total_ms * 1e-3)

    # end-to-end through the host-buffer call with pinned host memory
    e2e = None
    if not args.no_e2e and not shard:
        h_state = torch.tensor(state).pin_memory()
        h_q = torch.tensor(q).pin_memory() if q is not None else None
        hs = h_state.numpy()
        hq = h_q.numpy() if h_q is not None else None
        solver.run_host(hs, cfg, 1, q=hq)      # warm: host-path graph built
        np.copyto(hs, state)                   # the timed run starts from the seeded state
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        timer.barrier()
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(steps):
            # a host-driven trajectory: every step copies the host state in and the new
            # state back (the call's own copies, timed)
            solver.run_host(hs, cfg, 1, q=hq)
        e1.record(stream)
        timer.barrier()
        wall = time.perf_counter() - t0
        e2e_ms = _max_over_ranks(dist, e0.elapsed_time(e1), dev)
        h2d = 6 * n * 8 + (n * 8 if q is not None else 0)
        e2e = {"value": world * steps * pairs / (e2e_ms * 1e-3), "unit": "pair-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 6 * n * 8,
               "wall_s": wall}

    # roofline of the pair kernel: the learned kernel for the learned form; the ALG step
    # takes the phase-locked kernel once there are two or more of its 32-warp CTAs per SM
    # (as bia_step.cu decides)
    nb_blocks = (n + 31) // 32
    nwb = nb_blocks * (nb_blocks + 1) // 2
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    if tuned and "learned_layout" in tuned:
        split = tuned["learned_layout"] == "split"
    else:  # the library's rule: the learned step splits at every size
        split = method == 3
    if method == 3:
        kernel_name = ("bia_pair_rest_kernel<true> + bia_pair_learned_head_kernel + "
                       "bia_pair_learned_finish_kernel<true> (one timed interval)"
                       if split else "bia_pair_learned_kernel<true>")
    elif method == 1 and tuned is not None:
        kernel_name = {"tiles8": "bia_pair_tiles_kernel<true, 1>",
                       "phase32_lane": "bia_pair_phase_kernel<true, 32, 1, false>",
                       "phase32": "bia_pair_phase_kernel<true, 32, 1, true>"}[tuned["alg_shape"]]
    elif method == 1 and (nwb + 31) // 32 >= 2 * sms:
        kernel_name = "bia_pair_phase_kernel<true, 32, 1>"
    else:
        kernel_name = "bia_pair_tiles_kernel<true, %d>" % method
    flops_total = pair_flops(stats, method)
    per_launch_flops = flops_total / max(kern_launches, 1)
    per_launch_s = kern_ms * 1e-3 / max(kern_launches, 1)
    peak = measure_fp64_peak(local)
    achieved = per_launch_flops / per_launch_s / 1e12
    traffic = None
    tkey = (args.workload, method, ("split" if split else "one_kernel") if method == 3 else None)
    if args.n is None and args.dt is None and tkey in TRAFFIC:
        tp, tb = TRAFFIC[tkey]
        traffic = tb * pairs / tp
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": traffic,
                "traffic_note": "ncu capture of the dominant kernel on the same workload at n = 16384, "
                                "scaled by pairs per launch" if traffic else None,
                "algorithmic_bytes_per_launch": nb_blocks * 6 * n * 8 + 6 * n * 8,
                "peak_source": "measured live: bia_measure_fp64_peak DFMA loop on this GPU",
                "flops_per_launch": per_launch_flops, "kernel_ms_per_launch": per_launch_s * 1e3,
                "kernel": kernel_name}
    if method == 3:
        roofline["bf16_tensor_flops_per_launch"] = stats["learned"] * LEARNED_TENSOR_FLOPS / max(kern_launches, 1)

    # the plain FP64 form (the reference's ALG algorithm) on the same workload, timed the
    # same way, and the distance of one step of the measured form from one plain step
    plain = None
    if method != 1 and not args.no_plain:
        cfg_p = default_config(eps_th=eps, dt=dt, method=1)
        p_ms, _, p_stats, _ = timer.time(d_init, cfg_p, d_q, steps, args.warmup)
        a_state = d_init.clone()
        b_state = d_init.clone()
        with torch.cuda.stream(stream):
            solver.step(a_state, cfg_p, q=d_q, stats=False)
            solver.step(b_state, cfg, q=d_q, stats=False)
        timer.barrier()
        aa, bb = a_state.cpu().numpy(), b_state.cpu().numpy()
        solver.counters(reset=True)
        plain = {"method": "alg", "value": world * steps * pairs / (p_ms * 1e-3),
                 "ms_per_step": p_ms / steps, "speedup_of_measured_form": (p_ms / total_ms),
                 "one_step_rel_pos_err_vs_plain": float(np.linalg.norm(bb[:3] - aa[:3]) /
                                                        np.linalg.norm(aa[:3])),
                 "one_step_rel_vel_err_vs_plain": float(np.linalg.norm(bb[3:] - aa[3:]) /
                                                        np.linalg.norm(aa[3:])),
                 "newton_iterations": newton_per_pair(p_stats, 1)}

    # the universal-variable method (every pair on the Stumpff-function solver, this
    # library's fastest plain FP64 form), timed exactly as the measured form
    universal = None
    if method != 2 and not args.no_universal:
        cfg_u = default_config(eps_th=eps, dt=dt, method=2)
        u_ms, _, u_stats, _ = timer.time(d_init, cfg_u, d_q, steps, args.warmup)
        universal = {"method": "universal", "value": world * steps * pairs / (u_ms * 1e-3),
                     "unit": "pair-updates/s", "ms_per_step": u_ms / steps,
                     "nonconverged": u_stats["nonconverged"],
                     "newton_iterations": newton_per_pair(u_stats, 2)}
    # the learned form against the fastest plain FP64 form measured in this run
    learned_vs_best_plain = None
    if method == 3:
        plain_ms = [x["ms_per_step"] for x in (plain, universal) if x is not None]
        if plain_ms:
            learned_vs_best_plain = {"ratio": min(plain_ms) / (total_ms / steps),
                                     "best_plain": "universal" if universal and universal["ms_per_step"] == min(plain_ms)
                                     else "alg", "best_plain_ms_per_step": min(plain_ms),
                                     "learned_ms_per_step": total_ms / steps}

    errors = None
    if rank == 0 and world == 1 and not args.no_oracle_check:
        errors = error_vs_oracle(solver, cfg, d_init, d_q, state, eps, q, dt)

    # the reference's own GPU pair kernel (bia/find_dXYUV_kernel.cu built for sm_100a by
    # oracle/build_ref.sh) on a seeded row sample of a global-coupling workload
    # (plummer_32768: the reference has one eps for all pairs, so no Coulomb charges),
    # through its per-particle entry with its own per-call allocation and copies
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_kernel(solver, dev, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cmethod = {0: 0, 1: 1, 2: 1, 3: 1}[method]
        v, cores, sample = cpu_sample(state, eps, q, dt, cmethod, args.cpu_seconds)
        v1, _, sample1 = cpu_sample(state, eps, q, dt, cmethod, args.cpu_seconds / 2, seed=1, threads=1)
        cpu = {"value": v, "unit": "pair-updates/s", "cores": cores, "kind": "port",
               "sample": sample,
               "single_thread": {"value": v1, "unit": "pair-updates/s", "cores": 1, "sample": sample1,
                                 "note": "the reference's own single-threaded CPU figure is for "
                                         "its Fortran build (README.md:43)"}}

    extras = None
    if rank == 0 and world == 1 and not args.no_extras and args.n is None and args.dt is None:
        extras = run_extras(solver, timer, args)

    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": metric_name(args.method), "value": value,
            "unit": "pair-updates/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_keys(args.workload, n, dt, args.method, world, reduction="deterministic",
                                  precision=("heads: BF16 operands, FP32 accumulation; first correction "
                                             "FP32; final step, composition and sums FP64"
                                             if method == 3 else "FP64"),
                                  l2="256 MB buffer written between timed steps (untimed)",
                                  state="reset to the seeded state before every timed step (untimed "
                                        "device copy; the e2e loop runs consecutive steps from it through host buffers)",
                                  autotuned=tuned, shard=shard),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            # pair kernels (the split learned step: rest, head, finish) and the reduction per
            # step; a shard's reduction is two launches (the shard's sums, then the update
            # after the all-reduce)
            "gpu_launches": ((4 if split else 2) + (1 if shard else 0)) * steps,
            "learned_vs_best_plain": learned_vs_best_plain,
            "error_vs_oracle": errors,
            "plain_fp64": plain, "universal": universal,
            "reference_gpu_kernel": ref_gpu,
            "learned_pair_fraction": stats["learned"] / max(1, steps * pairs) if method == 3 else None,
            "stats": {k: v for k, v in stats.items()},
            # Newton iterations per pair of each solver the measured form ran
            "newton_iterations": newton_per_pair(stats, method),
            "extra_workloads": extras,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


def reference_gpu_kernel(solver, dev, stream):
    """The reference's GPU kernel through its per-row entry against ours (see main)."""
    import torch

    import oracle
    from bia_3d_gpu_b200 import default_config, find_dxyuv_kernel, initial
    if not oracle.ref_gpu_available():
        return None
    ps, peps, _, pdt, _ = initial.make("plummer_32768")
    pn = ps.shape[1]
    rows = np.random.default_rng(5).choice(np.arange(2, pn + 1), 256, replace=False)
    oracle.ref_gpu_rows(ps, peps, pdt, rows[:4])
    t0 = time.perf_counter()
    oracle.ref_gpu_rows(ps, peps, pdt, rows)
    el = time.perf_counter() - t0
    rpairs = int(sum(pn - r for r in rows))
    # ours through the same per-row drop-in entry (host buffers, one row per call)
    acc = [np.zeros(pn) for _ in range(6)]
    rel, out = np.zeros(6 * pn), np.zeros(6 * pn)

    def _our_rows(rr):
        for r_ in rr:
            for k_ in range(6):
                rel[k_::6] = ps[k_, r_ - 1] - ps[k_]
            find_dxyuv_kernel(1, pn, int(r_), peps, pdt, 18, *acc, rel, out)

    _our_rows(rows[:4])
    t0 = time.perf_counter()
    _our_rows(rows)
    el_ours = time.perf_counter() - t0
    pt = torch.tensor(ps, device=dev)
    pcfg = default_config(eps_th=peps, dt=pdt)
    with torch.cuda.stream(stream):
        solver.step(pt, pcfg, stats=False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            solver.step(pt, pcfg, stats=False)
        e1.record(stream)
    torch.cuda.synchronize()
    return {"workload": "plummer_32768", "unit": "pair-updates/s",
            "reference_kernel": rpairs / el,
            "ours_dropin_rows": rpairs / el_ours,
            "ours_alg": 3 * (pn * (pn - 1) // 2) / (e0.elapsed_time(e1) * 1e-3),
            "sample": f"{len(rows)} seeded rows I through find_dxyuv_kernel_ (reference, "
                      f"and ours as reference_kernel / ours_dropin_rows; ours_alg "
                      f"is the whole-step kernel path), "
                      f"{rpairs} pairs, {el:.2f} s wall"}


def run_extras(solver, timer, args):
    """The other configurations, each timed as the main line (steps from the seeded state,
    L2 flushed between them, CUDA events), with fewer steps: {workload: {form: result}}."""
    import torch

    from bia_3d_gpu_b200 import default_config, initial
    out = {}
    dev = timer.dev

    def forms(name, entries, steps, warmup, dt=None):
        s, eps, q, dt_cfg, _ = initial.make(name)
        dt = dt_cfg if dt is None else dt
        n = s.shape[1]
        pairs = n * (n - 1) // 2
        d_init = torch.tensor(s, device=dev)
        d_q = torch.tensor(q, device=dev) if q is not None else None
        res = {"n": n, "dt": dt, "steps": steps, "warmup": warmup}
        for label, m, kw in entries:
            fdt = kw.pop("dt", dt)
            c = default_config(eps_th=eps, dt=fdt, method=m, **kw)
            tuned = None
            if m == 1 and not args.no_autotune:
                # the context keeps one ALG shape per size: tune it on this workload's state
                var, _ = solver.autotune(d_init, c, q=d_q)
                tuned = ("tiles8", "phase32_lane", "phase32")[var]
            ms, _, st, _ = timer.time(d_init, c, d_q, steps, warmup)
            res[label] = {"ms_per_step": ms / steps, "pair_updates_per_s": steps * pairs / (ms * 1e-3),
                          "newton_iterations": newton_per_pair(st, m), "nonfinite": st["nonfinite"]}
            if tuned:
                res[label]["alg_shape"] = tuned
            if fdt != dt:
                res[label]["dt"] = fdt
            if m == 0:
                res[label]["rkf_steps_per_pair"] = st["rkf_steps"] / max(1, st["rkf"] + st["degenerate"])
        return res

    out["coulomb_cube_32768"] = forms("coulomb_cube_32768", [
        ("alg", 1, {}), ("universal", 2, {}), ("learned", 3, {}),
        ("rkf_rel_1e-12", 0, {"rkf_relerr": 1e-12, "rkf_abserr": 1e-16}),
        ("rkf_reference_tol_0_1e-16", 0, {})], steps=3, warmup=3)
    out["coulomb_cube_32768"]["learned_long_step_dt_1e-3"] = forms(
        "coulomb_cube_32768", [("learned", 3, {}), ("universal", 2, {})], steps=3, warmup=3, dt=1e-3)
    out["cold_ball_131072"] = forms("cold_ball_131072", [("alg", 1, {}), ("universal", 2, {}),
                                                         ("learned", 3, {})], steps=3, warmup=3)
    out["gravity_ball_1332"] = forms("gravity_ball_1332", [("alg", 1, {}), ("universal", 2, {}),
                                                           ("learned", 3, {})], steps=20, warmup=3)
    # a trajectory: the learned configuration's 100 consecutive steps in one CUDA graph
    s, eps, q, dt, steps_cfg = initial.make("plummer_32768")
    d_init = torch.tensor(s, device=dev)
    traj = {"steps": steps_cfg, "graph": True}
    for label, m in (("learned", 3), ("universal", 2)):
        ms, st = timer.graph_run(d_init, default_config(eps_th=eps, dt=dt, method=m), None, steps_cfg)
        traj[label] = {"ms_per_step": ms / steps_cfg, "newton_iterations": newton_per_pair(st, m)}
    out["plummer_32768_trajectory"] = traj
    ens, _, sizes, epairs = ensemble_forms(solver, 4096, 20, 3, [("alg", 1), ("universal", 2), ("learned", 3)],
                                           dev=dev)
    out["plummer_ensemble_4096"] = {"systems": 4096, "pairs_per_step": epairs, "steps": 20, "graph": True,
                                    "forms": {k: {kk: vv for kk, vv in v.items() if kk != "stats"}
                                              for k, v in ens.items()}}
    # the DIM direct-sum RKF45 solver as the physics check of the learned step on the same
    # sphere: DIM from 0 to dt (per-particle coupling eps/2) against one BIA step
    t = d_init.clone()
    solver.step(t, default_config(eps_th=eps, dt=dt, method=3), stats=False)
    torch.cuda.synchronize()
    b = t.cpu().numpy()
    t = d_init.clone()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dst = solver.dim_integrate(t, eps / 2, 0.0, dt)
    torch.cuda.synchronize()
    dim_s = time.perf_counter() - t0
    g = t.cpu().numpy()

    def rel(a, c):
        return float(np.linalg.norm(a - c) / np.linalg.norm(c))

    out["dim_plummer_32768"] = {"t_end": dt, "wall_s": dim_s, "accepted_steps": dst["accepted"],
                                "derivative_evaluations": dst["nde"],
                                "learned_bia_vs_dim_pos": rel(b[:3], g[:3]), "learned_bia_vs_dim_vel": rel(b[3:], g[3:]),
                                "note": "one BIA step of dt against the direct N-body integration over dt: the "
                                        "difference is the binary approximation itself"}
    return out


if __name__ == "__main__":
    main()
