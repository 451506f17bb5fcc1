"""Benchmark: Rodas5P ensemble solves/s on the Robertson configuration (one B200).

Workload (the configuration the headline metric is quoted on): Robertson
chemical kinetics, 3 states, 65,536 trajectories per GPU, rates k1 = 0.04,
k2 = 3e7, k3 = 1e4 each scaled by log-uniform[0.5, 2], y0 = (1, 0, 0), 20 save
times on [0, 1e5], rtol 1e-6, atol 1e-10, FP32 LU through the persistent refill
kernel.  One step = one full ensemble solve.

* ``value``  -- solves/s with inputs resident in HBM, device time (CUDA events on
  the launching stream), max over ranks; L2 (126 MB) is flushed between steps by
  writing a 256 MB buffer outside the timed launches.
* ``e2e``    -- the same through the public ``rodas5P.solve`` call with pinned host
  inputs: host->device copies, the solve and the device->host read of the
  history and counters inside the timed region (host wall clock).
* ``vs_plain`` -- the plain FP64 one-launch kernel (the reference's design) on the
  same ensemble, device-timed.
* ``roofline`` -- algorithmic FP64 + LU operations per launch (traced-graph counts
  x the step counts the kernel reports) against the measured CUDA-core FMA peaks.
* ``cpu_baseline`` -- the CPU oracle (C++/OpenMP restatement of the reference
  solver) on a bounded sample, all host cores, rank 0 at N=1 only.

``--impl reference`` times the reference's algorithm on the host instead (the
oracle port: the reference's own implementation needs numba-cuda-mlir, Enzyme and
JAX, none of which exist here) and prints the same line with ``"impl": "reference"``.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ensemble solves/s & gradients/s at fixed error vs FP64 oracle, vs plain kernel"
N_TRAJ = 65536


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_TRAJ)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the compact lines of the other configurations")
    ap.add_argument("--warm-s", type=float, default=None,
                    help="seconds of warm-up launches before each timed headline variant, at least "
                         "(default 0.5; the --warmup launches are always run)")
    ap.add_argument("--profile", action="store_true",
                    help="only the tuned timed launches (for ncu captures); prints no bench line")
    ap.add_argument("--max-steps", type=int, default=100000,
                    help="--config runs: step cap per trajectory (the solvers' default 100000); "
                         "lower caps split a makespan into its device-full and tail parts")
    ap.add_argument("--launch", default="auto", choices=["auto", "plain", "persistent"],
                    help="launch of the timed kernel (auto = autotuned)")
    ap.add_argument("--config", default="robertson",
                    choices=["robertson", "lorenz", "vdp4", "vdp16", "vdp64", "brusselator",
                             "grad_vdp1", "grad_vdp8"],
                    help="robertson: the headline line; the others print a line for that configuration")
    return ap.parse_args()


def config_dict(n_total, world):
    return {
        "workload": "Robertson Rodas5P, 3 states, FP32 LU (fast arithmetic), autotuned launch",
        "trajectories_per_gpu": n_total // world,
        "save_times": 20,
        "rtol": 1e-6,
        "atol": 1e-10,
        "l2": "flushed between timed steps (256 MB write)",
        "parallelism": f"replicas x{world} (independent trajectory ranges)",
    }


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.lines = []
        self.window_start = 0.0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.uuid}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self):
        """Keep only the samples taken from now on (the timed region)."""
        self.window_start = time.monotonic()

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        mhz, max_mhz, reasons = [], None, set()
        for stamp, line in self.lines:
            if stamp < self.window_start:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                mhz.append(float(parts[0]))
                max_mhz = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                  "sw_power_cap"), parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(mhz) if mhz else None,
            "sm_max_mhz": max_mhz,
            "reasons": sorted(reasons),
            "samples": len(mhz),
        }


# --------------------------------------------------------------------------- helpers
def dist_setup(args):
    from menodax_b200 import _dist

    return _dist.init(backend="nccl")


def max_over_ranks(x, world):
    from menodax_b200 import _dist

    return _dist.max_over_ranks(x, world)


def barrier(world):
    from menodax_b200 import _dist

    _dist.barrier(world)


def cpu_sample_solve(cfg, n_sample, lu_precision):
    """The oracle on the first ``n_sample`` trajectories, every host thread."""
    from oracle import oracle

    oracle.build()
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"][:n_sample], cfg["t_span"],
                 cfg["params"][:n_sample], rtol=cfg["rtol"], atol=cfg["atol"],
                 lu_precision=lu_precision, threads=threads)
    dt = time.perf_counter() - t0
    return n_sample / dt, threads, dt


# --------------------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from workloads import systems

    cfg = systems.robertson_config(size=args.n)
    sample = 8192
    for _ in range(args.warmup):
        cpu_sample_solve(cfg, 1024, "fp32")
    rates, threads, total = [], 0, 0.0
    for _ in range(args.steps):
        r, threads, dt = cpu_sample_solve(cfg, sample, "fp32")
        rates.append(r)
        total += dt
    value = sample * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (FP32 LU)", "data": "synthetic (seed 42)",
        "config": config_dict(args.n * world, world),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} of the {args.n} trajectories per step, C++ oracle, OpenMP"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference kernels need numba-cuda-mlir, numba-enzyme and JAX (absent); "
                "this is the CPU restatement of the same algorithm",
    }
    print(json.dumps(line))


def scipy_baseline(cfg, sample):
    """The reference's own CPU ensemble solver, restated (one scipy ``solve_ivp``
    per trajectory over a spawn pool of one process per core, LSODA:
    ``reference/solvers/python/scipy_solve_ivp.py:165-255``), timed on a sample."""
    from oracle import scipy_ensemble
    from workloads import systems

    workers = os.cpu_count() or 1
    rate, _ = scipy_ensemble.timed_rate(systems.robertson, cfg["y0"][:sample], cfg["t_span"],
                                        cfg["params"][:sample], method="LSODA", rtol=cfg["rtol"],
                                        atol=cfg["atol"], workers=workers)
    scipy_ensemble.close()
    return {"value": rate, "unit": "solves/s", "cores": workers, "kind": "port",
            "sample": f"first {sample} trajectories, scipy solve_ivp LSODA per trajectory, spawn pool "
                      "(the reference's scipy_solve_ivp.py approach)"}


# --------------------------------------------------------------------------- oracle checks
def error_summary(err, rtol):
    import numpy as np

    return {"median": float(np.median(err)), "p99": float(np.quantile(err, 0.99)), "max": float(err.max()),
            "within_10_rtol": float((err <= 10.0 * rtol).mean())}


def headline_errors(cfg, outputs, sample):
    """CPU-baseline leg, used as the checker: each sampled GPU output against the FP64
    oracle at rtol 1e-12.  A trajectory's error is the largest over its saves and
    components of |x - x_ref| / (|x_ref| + atol / rtol)."""
    import numpy as np

    from oracle import oracle

    ref, *_ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"][:sample], cfg["t_span"],
                           cfg["params"][:sample], rtol=1e-12, atol=1e-14, lu_precision="fp64",
                           max_steps=10_000_000, threads=oracle.max_threads())
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    out = {name: error_summary((np.abs(h - ref) / scale).reshape(sample, -1).max(axis=1), cfg["rtol"])
           for name, h in outputs.items()}
    out["against"] = (f"FP64 oracle at rtol 1e-12, atol 1e-14, first {sample} trajectories; per-trajectory "
                      "max over saves and components of |x - x_ref| / (|x_ref| + atol/rtol)")
    return out


def gradient_errors(cfg, target, grads, sample):
    """CPU-baseline leg, used as the checker: each sampled gradient of
    sum((y - target)^2) against the oracle's forward sensitivities at rtol 1e-10
    with the sensitivities under error control (the tight gradient).  A
    trajectory's error is max |g - g_ref| / max |g_ref| over its y0 and mu
    components."""
    import numpy as np

    from oracle import oracle

    system = oracle.System.vdp_ring(1, 1.0, 0.1)
    y0, mu = cfg["y0"][:sample], cfg["params"][:sample]
    hist, *_ = oracle.solve("rodas5P", system, y0, cfg["t_span"], mu, rtol=1e-10, atol=1e-12,
                            lu_precision="fp64", sens=(True, [0], True), max_steps=10_000_000,
                            threads=oracle.max_threads())
    n = system.n
    w = 2.0 * (hist[:, :, :n] - target)
    sens = hist[:, :, n:].reshape(sample, len(cfg["t_span"]), n + 1, n)
    g_ref = np.einsum("nsj,nskj->nk", w, sens)
    scale = np.abs(g_ref).max(axis=1)
    out = {}
    for name, g in grads.items():
        rel = np.abs(g - g_ref).max(axis=1) / scale
        out[name] = {"median": float(np.median(rel)), "p90": float(np.quantile(rel, 0.9)),
                     "max": float(rel.max()), "within_1e-5": float((rel <= 1e-5).mean())}
    out["against"] = (f"oracle forward sensitivities at rtol 1e-10 (error control on), first {sample} "
                      "trajectories, same targets")
    return out


# --------------------------------------------------------------------------- gradients
def measure_gradients(n, steps, warmup, rank, world, n_osc=1, oracle_checks=False, ring_forward_sens=False):
    """Stiff Van der Pol gradients: discrete-adjoint value_and_grad of sum((y - target)^2), device-timed.

    VdP (n_osc=1: 2 states), mu ~ log-uniform[10, 500], y0 and mu differentiated,
    20 saves on [0, 1000], rtol 1e-6, atol 1e-8, FP64; targets are the same solve
    with mu * 1.05.  One step = forward checkpointing solve + reverse sweep."""
    import torch

    from menodax_b200 import rodas5P
    from workloads import systems

    cfg = systems.vdp_gradient_config(n_osc, size=n, seed=42 + rank)
    fn = cfg["ode_fn"]
    dev = torch.device("cuda", torch.cuda.current_device())
    y0 = torch.as_tensor(cfg["y0"], device=dev)
    mu = torch.as_tensor(cfg["params"], device=dev)
    t = cfg["t_span"]
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    if n_osc > 1:
        # The ring's Jacobian pattern: a sparse LU in the forward and reverse sweeps.
        kw["sparsity"] = systems.vdp_sparsity(n_osc)
    with torch.no_grad():
        target = rodas5P.solve(fn, y0, t, mu * 1.05, **kw)

    def value_and_grad(lu_precision, **tighter):
        y0_t = y0.clone().requires_grad_(True)
        p_t = mu.clone().requires_grad_(True)
        hist, stats = rodas5P.solve(fn, y0_t, t, p_t, return_stats=True, sens_error_control=False,
                                    **{**kw, "lu_precision": lu_precision, **tighter})
        loss = ((hist - target) ** 2).sum()
        loss.backward()
        return loss, y0_t.grad, p_t.grad, stats

    stream = torch.cuda.current_stream(dev)

    def timed(lu_precision, n_steps, n_warm=None, **tighter):
        for _ in range(warmup if n_warm is None else n_warm):
            value_and_grad(lu_precision, **tighter)
        barrier(world)
        ms = []
        for _ in range(n_steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            # Each step starts on an idle device, so no step's time holds the
            # tail of the one before.
            torch.cuda.synchronize(dev)
            e0.record(stream)
            loss, gy, gp, stats = value_and_grad(lu_precision, **tighter)
            e1.record(stream)
            ms.append((e0, e1))
        barrier(world)
        total = max_over_ranks(sum(a.elapsed_time(b) for a, b in ms), world)
        return total, gy, gp, stats

    total, gy, gp, stats = timed("fp64", steps)
    from menodax_b200 import autograd

    ckpt64 = dict(autograd.last_checkpoint)
    acc = stats["accepted_steps"].to(torch.float64)
    finite = bool(torch.isfinite(gy).all() and torch.isfinite(gp).all())
    # The FP32-LU adjoint (fast arithmetic) on the same ensemble: its own step
    # sequence, so its gradients differ from the FP64 ones at solver-tolerance
    # level; the median relative difference says by how much.
    fs32 = max(1, steps // 2)
    total32, gy32, gp32, _ = timed("fp32", fs32)
    g64 = torch.cat([gy, gp], dim=1)
    g32 = torch.cat([gy32, gp32], dim=1)
    rel32 = (g32 - g64).abs().max(dim=1).values / g64.abs().max(dim=1).values.clamp_min(1e-300)

    result = {
        "metric": "gradients/s", "value": n * world * steps / (total * 1e-3), "unit": "gradients/s",
        "ms_per_step": total / steps,
        "workload": f"VdP ring n_osc={n_osc} ({2 * n_osc} states), Rodas5P FP64"
                    f"{' sparse LU' if n_osc > 1 else ''}, discrete adjoint, "
                    f"{n} trajectories per GPU, 20 saves on [0, 1000], rtol 1e-6, atol 1e-8",
        "accepted_steps_mean": float(acc.mean()), "accepted_steps_max": float(acc.max()),
        "checkpoints": ckpt64,
        "gradients_finite": finite,
        "fp32_lu": {
            "value": n * world * fs32 / (total32 * 1e-3), "unit": "gradients/s",
            "ms_per_step": total32 / fs32,
            "method": "the same discrete adjoint with FP32 LUs and fast arithmetic",
            "median_rel_diff_vs_fp64": float(rel32.median()),
        },
    }
    if n_osc > 1 and not ring_forward_sens:
        return result
    if n_osc > 1:
        # The reference's method on the same GPU for the ring: the joint [y, S]
        # system carries 2 n_osc (2 n_osc + 2) components (288 at 16 states; its
        # kernel takes minutes to compile), so it is timed once on the first
        # FS_SAMPLE trajectories, and only by --config grad_vdp8.
        from menodax_b200 import sensitivity

        fs_n = min(n, FS_SAMPLE)
        sensitivity.solve("rodas5P", fn, y0[:64], t, mu[:64], **kw)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        state, sens = sensitivity.solve("rodas5P", fn, y0[:fs_n], t, mu[:fs_n], **kw)
        g_fs = torch.einsum("nsj,nsjk->nk", 2.0 * (state - target[:fs_n]), sens)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        fs_ms = max_over_ranks(e0.elapsed_time(e1), world)
        g_adj = torch.cat([gy, gp], dim=1)[:fs_n]
        rel = ((g_adj - g_fs).abs().max(dim=1).values / g_fs.abs().max(dim=1).values.clamp_min(1e-300))
        result["forward_sensitivities"] = {
            "value": fs_n * world / (fs_ms * 1e-3), "unit": "gradients/s",
            "method": "joint [y, S] Rodas5P solve, sensitivities under error control (the reference's method), "
                      f"first {fs_n} trajectories, one launch",
            "median_rel_diff_vs_adjoint": float(rel.median()),
        }
        return result

    # The reference's method on the same GPU: forward sensitivities (the joint
    # [y, S] solve with the sensitivities under error control, its default),
    # contracted with the loss's cotangent.
    from menodax_b200 import sensitivity

    def forward_sensitivity_grad():
        state, sens = sensitivity.solve("rodas5P", fn, y0, t, mu, **kw)
        resid = state - target
        g = torch.einsum("nsj,nsjk->nk", 2.0 * resid, sens)
        return (resid ** 2).sum(), g

    fs_steps = max(1, steps // 2)
    forward_sensitivity_grad()
    barrier(world)
    fms = []
    for _ in range(fs_steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, g_fs = forward_sensitivity_grad()
        e1.record(stream)
        fms.append((e0, e1))
    barrier(world)
    fs_total = max_over_ranks(sum(a.elapsed_time(b) for a, b in fms), world)
    # The adjoint at a tighter tolerance (rtol 1e-8, atol 1e-10): its error
    # against the tight oracle gradient next to the forward sensitivities' at
    # rtol 1e-6, so the two methods can be compared at matched error.
    total_t, gy_t, gp_t, _ = timed("fp64", 1, n_warm=1, rtol=1e-8, atol=1e-10)
    g_tight = torch.cat([gy_t, gp_t], dim=1)
    result["adjoint_fp64_rtol_1e-8"] = {
        "value": n * world / (total_t * 1e-3), "unit": "gradients/s", "ms_per_step": total_t,
        "method": "the discrete adjoint, FP64, rtol 1e-8, atol 1e-10 (same loss and targets)",
    }
    if oracle_checks and rank == 0 and world == 1:
        sample = 256
        result["error_vs_tight_oracle_gradient"] = gradient_errors(
            {"y0": cfg["y0"], "params": cfg["params"], "t_span": t}, target[:sample].cpu().numpy(),
            {"adjoint_fp64": g64[:sample].cpu().numpy(), "adjoint_fp32_lu": g32[:sample].cpu().numpy(),
             "forward_sensitivities": g_fs[:sample].cpu().numpy(),
             "adjoint_fp64_rtol_1e-8": g_tight[:sample].cpu().numpy()}, sample)
    g_adj = torch.cat([gy, gp], dim=1)
    rel = ((g_adj - g_fs).abs().max(dim=1).values / g_fs.abs().max(dim=1).values.clamp_min(1e-300))
    result["forward_sensitivities"] = {
        "value": n * world * fs_steps / (fs_total * 1e-3), "unit": "gradients/s",
        "method": "joint [y, S] Rodas5P solve, sensitivities under error control (the reference's method)",
        "median_rel_diff_vs_adjoint": float(rel.median()),
    }
    return result


# --------------------------------------------------------------------------- other configurations
FS_SAMPLE = 4096  # trajectories of the ring's forward-sensitivity timing
WARM_S = 0.5   # seconds of warm-up launches per configuration variant, at least
WARM_MAX = 50  # and at most this many launches for it


def config_roofline(fn, n_vars, n_params, opts, counters, n, n_save, launch_ms, peaks):
    """Algorithmic FP64 + LU-type operations of one launch (attempted steps the
    kernel reported x per-step counts of the traced problem) over its device
    time, against the measured CUDA-core peaks blended by the same mix."""
    import torch

    from menodax_b200._flops import rodas5p_cost, tsit5_cost
    from menodax_b200._problem import wide_solve
    from menodax_b200._sparse_direct import sparse_lu_for

    if opts.solver == "tsit5":
        cost = tsit5_cost(fn, n_vars, n_params)
    else:
        sparse = sparse_lu_for(opts.sparsity, opts.ordering) if opts.sparsity is not None else None
        cost = rodas5p_cost(fn, n_vars, n_params, sparse=sparse, wide_solve=wide_solve(opts, n_vars))
    steps = float(counters[2].to(torch.float64).sum())
    f64 = steps * cost.f64 + n * (n_save - 1) * cost.per_save
    lu = steps * cost.lu
    peak64, peak32 = peaks
    lu_peak = peak32 if opts.lu_precision == "fp32" else peak64
    seconds = launch_ms * 1e-3
    t_roof = f64 / peak64 + lu / lu_peak
    achieved = (f64 + lu) / seconds
    return {"bound": "fp64", "achieved": achieved / 1e12, "peak": (f64 + lu) / t_roof / 1e12,
            "unit": "TFLOP/s", "frac": t_roof / seconds}


def measure_config(name, steps, warmup, rank, world, *, max_steps=100000, n_limit=None, cpu_baseline=True,
                   verbose=True, skip=()):
    """Device-timed solves/s of one non-headline configuration: the autotuned
    FP32-LU kernel (Tsit5: FP64) and the plain FP64 reference-arithmetic kernel
    (the reference's design), each with its roofline, plus the step statistics
    and (rank 0, one GPU) the CPU oracle on a sample.  ``skip`` names variants
    left out."""
    import torch

    from menodax_b200 import _native, autotune
    from menodax_b200._ensemble import launch
    from menodax_b200._frontend import longest_first
    from menodax_b200._problem import KernelOptions, get_problem
    from menodax_b200._sparsity import normalize_sparsity
    from workloads import systems

    dev = torch.device("cuda", torch.cuda.current_device())
    variants = []
    if name == "lorenz":
        cfg = systems.lorenz_config(size=4096, seed=42 + rank)
        n_vars, n_params = 3, 1
        variants = [("tsit5_fp64", KernelOptions(solver="tsit5"))]
        oracle_sys = ("tsit5", "lorenz", ())
    elif name.startswith("vdp"):
        n_osc = int(name[3:])
        cfg = systems.vdp_ring_config(n_osc, size=32768, seed=42 + rank)
        n_vars, n_params = 2 * n_osc, 1
        pat = normalize_sparsity(cfg["sparsity"], n_vars)
        variants = [("sparse_fp32_fast", KernelOptions(lu_precision="fp32", fast=True, sparsity=pat)),
                    ("plain_fp64_sparse_reference_arith", KernelOptions(lu_precision="fp64", sparsity=pat))]
        if n_vars <= 32:
            # Dense LUs last.  At 32 states the FP32 one runs on a team kernel;
            # the plain FP64 one-thread-per-trajectory kernel keeps a 32 x 32 double
            # matrix in local memory and takes minutes, so it runs only up to 16
            # states.  At 128 (what the reference's own benchmark timed out on)
            # neither runs.
            variants.append(("dense_fp32", KernelOptions(lu_precision="fp32", fast=True)))
            if n_vars <= 16:
                variants.append(("plain_fp64_reference_arith", KernelOptions(lu_precision="fp64")))
        oracle_sys = ("rodas5P", "vdp_ring", (n_osc, 1.0, 0.1))
    else:
        cfg = systems.brusselator_config(size=16384, seed=42 + rank)
        n_vars, n_params = 64, 1
        pat = normalize_sparsity(cfg["sparsity"], n_vars)
        variants = [("sparse_fp32_fast", KernelOptions(lu_precision="fp32", fast=True, sparsity=pat)),
                    ("dense_fp32", KernelOptions(lu_precision="fp32", fast=True)),
                    ("plain_fp64_sparse_reference_arith", KernelOptions(lu_precision="fp64", sparsity=pat)),
                    ("plain_fp64_reference_arith", KernelOptions(lu_precision="fp64"))]
        oracle_sys = ("rodas5P", "brusselator", (32,))
    variants = [v for v in variants if v[0] not in skip]
    if n_limit is not None:
        cfg = {**cfg, "y0": cfg["y0"][:n_limit], "params": cfg["params"][:n_limit]}
    fn = cfg["ode_fn"]
    n = cfg["y0"].shape[0]
    y0 = torch.as_tensor(cfg["y0"], device=dev).contiguous()
    params = torch.as_tensor(cfg["params"], device=dev).contiguous()
    times = torch.as_tensor(cfg["t_span"], device=dev).contiguous()
    common = dict(y0=y0, times=times, params=params, weights=None, dt0=0.0, rtol=cfg["rtol"],
                  atol=cfg["atol"], max_steps=max_steps)
    stream = torch.cuda.current_stream(dev)
    results = {}
    stats = None
    peaks = (_native.measure_fma_peak(True), _native.measure_fma_peak(False))
    for vname, opts in variants:
        if vname.startswith("plain"):
            prob, mode, grid = get_problem(fn, n_vars, n_params, opts), _native.MDX_LAUNCH_PLAIN, 0
            label = "plain, 32 threads/block"
        else:
            choice = autotune.tune(fn, n_vars, n_params, opts, tune_team=True,
                                   tune_shared=opts.solver == "tsit5", **common)
            opts = autotune.options_for(opts, choice)
            prob = get_problem(fn, n_vars, n_params, opts)
            mode, grid = choice.mode, autotune.grid_blocks(prob, choice, n)
            label = choice.describe()
        # Warm up for the requested launches and at least WARM_S of device work:
        # the first launches after a pause run below steady clocks (a 20 ms
        # kernel takes 25-36 ms on its first two launches).
        warm_start = time.perf_counter()
        done = 0
        order = None
        while done < warmup or (time.perf_counter() - warm_start < WARM_S and done < WARM_MAX):
            hist, counters = launch(prob, mode=mode, grid_blocks=grid, order=order, **common)
            torch.cuda.synchronize()
            if mode == _native.MDX_LAUNCH_PERSISTENT:
                # As rodas5P.solve does from its second call on: the persistent
                # launch takes the trajectories longest first by the last one's steps.
                order = longest_first(counters[2])
            done += 1
        barrier(world)
        ms = []
        # NVTX range per variant: ncu --nvtx --nvtx-include "timed:<variant>/" takes its launches.
        torch.cuda.nvtx.range_push(f"timed:{vname}")
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            hist, counters = launch(prob, mode=mode, grid_blocks=grid, order=order, **common)
            e1.record(stream)
            ms.append((e0, e1))
        torch.cuda.nvtx.range_pop()
        barrier(world)
        t = max_over_ranks(sum(a.elapsed_time(b) for a, b in ms), world)
        loop = counters[2].to(torch.float64)
        results[vname] = {"solves_per_s": n * world * steps / (t * 1e-3), "ms_per_solve": t / steps,
                          "launch": label,
                          "max_steps_fraction": float((counters[3] & 1).to(torch.float64).mean()),
                          "roofline": config_roofline(fn, n_vars, n_params, opts, counters, n,
                                                      times.numel(), t / steps, peaks)}
        if rank == 0 and verbose:
            print(json.dumps({"config": name, "variant": vname, **results[vname]}), flush=True)
        if stats is None:
            stats = {"steps_mean": float(loop.mean()), "steps_max": float(loop.max()),
                     "max_steps_hit": int((counters[3] & 1).sum())}
    cpu = None
    if rank == 0 and world == 1 and cpu_baseline:
        # CPU-baseline leg: the oracle timed on a sample of the same ensemble.
        from oracle import oracle

        solver, sysname, sysargs = oracle_sys
        system = getattr(oracle.System, sysname)(*sysargs)
        sample = min(n, 256 if n_vars > 8 else 2048)
        t0 = time.perf_counter()
        oracle.solve(solver, system, cfg["y0"][:sample], cfg["t_span"], cfg["params"][:sample],
                     rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp32", threads=oracle.max_threads())
        cpu = {"value": sample / (time.perf_counter() - t0), "unit": "solves/s",
               "cores": oracle.max_threads(), "kind": "port", "sample": f"first {sample} trajectories"}
    return {"config": name, "trajectories": n * world, "n_vars": n_vars, "max_steps": max_steps,
            "variants": results, "step_stats": stats, "cpu_baseline": cpu}


def run_config(args):
    """``--config``: one line per variant of one configuration, then a summary line."""
    rank, world, _ = dist_setup(args)
    if args.config.startswith("grad_"):
        n_osc = int(args.config[len("grad_vdp"):])
        n = 65536 if args.n == N_TRAJ else args.n
        res = measure_gradients(n, args.steps, args.warmup, rank, world, n_osc=n_osc, ring_forward_sens=True)
        if rank == 0:
            print(json.dumps({"config": args.config, **res}))
        return
    res = measure_config(args.config, args.steps, args.warmup, rank, world, max_steps=args.max_steps,
                         n_limit=None if args.n == N_TRAJ else args.n, cpu_baseline=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(res))


# --------------------------------------------------------------------------- our arm
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.config != "robertson":
        run_config(args)
        return
    import torch

    from menodax_b200 import _native, rodas5P
    from workloads import systems
    from menodax_b200._ensemble import launch
    from menodax_b200._flops import rodas5p_cost
    from menodax_b200._problem import KernelOptions, get_problem, wide_solve

    rank, world, local = dist_setup(args)
    dev = torch.device("cuda", torch.cuda.current_device())
    n = args.n
    cfg = systems.robertson_config(size=n, seed=42 + rank)
    fn = cfg["ode_fn"]

    from menodax_b200 import autotune

    fp32 = get_problem(fn, 3, 3, KernelOptions(lu_precision="fp32", fast=True))
    fp32_ref = get_problem(fn, 3, 3, KernelOptions(lu_precision="fp32"))
    fp64 = get_problem(fn, 3, 3, KernelOptions(lu_precision="fp64"))
    y0 = torch.as_tensor(cfg["y0"], device=dev).contiguous()
    params = torch.as_tensor(cfg["params"], device=dev).contiguous()
    times = torch.as_tensor(cfg["t_span"], device=dev).contiguous()
    hist = torch.empty((n, times.numel(), 3), dtype=torch.float64, device=dev)
    counters = torch.empty((4, n), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def solve(problem, mode, grid=0, order=None):
        return launch(problem, y0=y0, times=times, params=params, weights=None, dt0=0.0,
                      rtol=cfg["rtol"], atol=cfg["atol"], max_steps=100000, mode=mode,
                      grid_blocks=grid, out=(hist, counters), order=order)

    def visiting_order(problem, mode, grid=0):
        """A persistent launch visits the trajectories longest first by the step
        counts of the previous solve of the same problem, as ``rodas5P.solve``
        does from its second call on; a plain launch takes them in index order."""
        if mode != _native.MDX_LAUNCH_PERSISTENT:
            return None
        solve(problem, mode, grid)
        return autotune.longest_first(counters[2].clone())

    headline_warm_s = WARM_S if args.warm_s is None else args.warm_s

    def timed(problem, mode, steps, warmup, grid=0, warm_s=None, order=None):
        warm_s = headline_warm_s if warm_s is None else warm_s
        # At least `warmup` launches and warm_s of device work: a 0.5 ms kernel
        # launched after an idle moment runs below steady clocks for a while.
        start = time.perf_counter()
        done = 0
        while done < warmup or time.perf_counter() - start < warm_s:
            solve(problem, mode, grid, order)
            done += 1
            if done % 64 == 0:
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        evs = []
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solve(problem, mode, grid, order)
            e1.record(stream)
            evs.append((e0, e1))
        barrier(world)
        ms = [a.elapsed_time(b) for a, b in evs]
        return ms

    # Autotune the FP32-LU launch on this ensemble (outside any timing), then
    # warm every module that is timed below.
    fast_opts = KernelOptions(lu_precision="fp32", fast=True)
    choice = autotune.tune(fn, 3, 3, fast_opts, y0=y0, times=times, params=params, weights=None,
                           dt0=0.0, rtol=cfg["rtol"], atol=cfg["atol"], max_steps=100000)
    tuned = get_problem(fn, 3, 3, autotune.options_for(fast_opts, choice))
    tuned_grid = autotune.grid_blocks(tuned, choice, n)
    tuned_order = visiting_order(tuned, choice.mode, tuned_grid)
    for prob, mode in ((tuned, choice.mode), (fp32, _native.MDX_LAUNCH_PERSISTENT),
                       (fp64, _native.MDX_LAUNCH_PLAIN), (fp32_ref, _native.MDX_LAUNCH_PLAIN)):
        solve(prob, mode, tuned_grid if prob is tuned else 0)
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid) if uuid else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    if args.profile:
        # The timed launches sit in an NVTX range "timed", so a capture can take
        # exactly them: ncu --nvtx --nvtx-include "timed/" ...
        torch.cuda.nvtx.range_push("timed")
        timed(tuned, choice.mode, args.steps, args.warmup, tuned_grid, warm_s=0.0, order=tuned_order)
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile": "done", "launch": choice.describe()}))
        return
    if sampler:
        sampler.mark()
    ms = timed(tuned, choice.mode, args.steps, args.warmup, tuned_grid, order=tuned_order)
    total_ms = max_over_ranks(sum(ms), world)
    value = n * world * args.steps / (total_ms * 1e-3)
    steps_done = counters[2].to(torch.int64).sum().item()
    n_saves = n * (times.numel() - 1)
    # The timed output's first trajectories, for the error against the oracle.
    err_sample = min(n, 1024)
    outputs = {"timed_fp32_lu_fast": hist[:err_sample].cpu().numpy()}

    # the plain FP64 one-launch kernel and the other two variants, same ensemble
    variants = {}
    for name, prob, mode in (("plain_fp64_reference_arith", fp64, _native.MDX_LAUNCH_PLAIN),
                             ("plain_fp32_reference_arith", fp32_ref, _native.MDX_LAUNCH_PLAIN),
                             ("plain_fp32_fast", fp32, _native.MDX_LAUNCH_PLAIN),
                             ("persistent_fp32_fast", fp32, _native.MDX_LAUNCH_PERSISTENT),
                             ("persistent_fp64_reference_arith", fp64, _native.MDX_LAUNCH_PERSISTENT)):
        v_ms = timed(prob, mode, max(3, args.steps // 2), 2, order=visiting_order(prob, mode))
        t = max_over_ranks(sum(v_ms), world)
        variants[name] = n * world * len(v_ms) / (t * 1e-3)
        if name == "plain_fp64_reference_arith":
            outputs[name] = hist[:err_sample].cpu().numpy()
    # Clock samples cover the timed launches of the headline and its variants.
    clocks = sampler.stop() if sampler else {}

    # roofline of the timed kernel
    cost = rodas5p_cost(fn, 3, 3, wide_solve=wide_solve(fast_opts, 3))
    peak64 = _native.measure_fma_peak(True)
    peak32 = _native.measure_fma_peak(False)
    per_launch_f64 = steps_done * cost.f64 + n_saves * cost.per_save
    per_launch_f32 = steps_done * cost.lu
    launch_s = (sum(ms) / len(ms)) * 1e-3
    t_roof = per_launch_f64 / peak64 + per_launch_f32 / peak32
    achieved = (per_launch_f64 + per_launch_f32) / launch_s
    blended_peak = (per_launch_f64 + per_launch_f32) / t_roof
    # DRAM traffic per launch is an ncu figure: it cannot be read inside a timed
    # run, so it comes from the committed capture of this kernel, labelled as such.
    traffic_path = ROOT / "profiles" / "robertson_traffic.json"
    traffic, traffic_source = None, None
    if traffic_path.exists():
        try:
            capture = json.loads(traffic_path.read_text())
            traffic = capture.get("bytes_per_launch")
            traffic_source = f"ncu capture in {traffic_path.relative_to(ROOT)} ({capture.get('kernel', '')})"
        except (OSError, ValueError):
            traffic = None

    # end to end through the public API, pinned host buffers
    y0_h = torch.as_tensor(cfg["y0"]).pin_memory()
    p_h = torch.as_tensor(cfg["params"]).pin_memory()
    t_h = torch.as_tensor(cfg["t_span"]).pin_memory()
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp32", return_stats=True,
              launch="auto")
    # Warm-up keeps its results alive the way the timed loop does, so torch's
    # pinned host allocator holds the two result buffers a steady state needs.
    out = None
    for _ in range(max(2, args.warmup)):
        out, st = rodas5P.solve(fn, y0_h, t_h, p_h, **kw)
    barrier(world)
    per_call = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        tc = time.perf_counter()
        out, st = rodas5P.solve(fn, y0_h, t_h, p_h, **kw)
        per_call.append(time.perf_counter() - tc)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    print("e2e per call (ms):", [round(1e3 * x, 3) for x in per_call], file=sys.stderr)
    e2e = n * world * args.steps / e2e_s
    h2d = y0_h.numel() * 8 + p_h.numel() * 8 + t_h.numel() * 8
    d2h = out.numel() * 8 + 3 * n * 4

    checks = rank == 0 and world == 1 and not args.no_cpu_baseline
    grads = measure_gradients(n, max(3, args.steps // 2), args.warmup, rank, world, oracle_checks=checks)

    # The other configurations, compactly: every variant device-timed with its
    # roofline and the fraction of trajectories stopped by max_steps.
    configs = {}
    if not args.headline_only:
        for cname, csteps in (("lorenz", max(3, args.steps // 2)), ("vdp4", 1), ("brusselator", 1)):
            configs[cname] = measure_config(cname, csteps, 1, rank, world, cpu_baseline=checks, verbose=False)
        configs["grad_vdp8"] = measure_gradients(n, 1, 1, rank, world, n_osc=8)

    cpu = None
    errors = None
    cpu_scipy = None
    if checks:
        # CPU-baseline leg: the oracle timed on a sample, then used as the checker.
        sample = 8192
        rate, threads, _ = cpu_sample_solve(cfg, sample, "fp32")
        cpu = {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"first {sample} of the {n} trajectories, FP32 LU, C++ oracle with OpenMP"}
        errors = headline_errors(cfg, outputs, err_sample)
        cpu_scipy = scipy_baseline(cfg, 2048)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (FP32 LU)", "data": "synthetic (seed 42 + rank)",
            "config": config_dict(n * world, world),
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "vs_plain": {k: v for k, v in variants.items()},
            "speedup_vs_plain_fp64": value / variants["plain_fp64_reference_arith"],
            "launch": choice.describe(),
            "error_vs_oracle": errors,
            "gradients": grads,
            "configs": configs,
            "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": blended_peak / 1e12,
                         "unit": "TFLOP/s", "frac": achieved / blended_peak, "traffic": traffic,
                         "traffic_source": traffic_source,
                         "peak_source": "FP64 / FP32 FMA peaks measured in this run (mdx_measure_fma_peak); "
                                        "MEASURED_PEAKS.json holds HBM and bf16 tensor figures only",
                         "peak_fp64_measured": peak64 / 1e12, "peak_fp32_measured": peak32 / 1e12,
                         "ops_per_launch_fp64": per_launch_f64, "ops_per_launch_lu_fp32": per_launch_f32,
                         "attempted_steps_per_launch": steps_done},
            "cpu_baseline": cpu,
            "cpu_baseline_scipy": cpu_scipy,
            "clocks": clocks,
            "gpu_launches": args.steps,
        }
        print(json.dumps(line))
    from menodax_b200 import _dist

    _dist.finalize(world)


if __name__ == "__main__":
    main()
