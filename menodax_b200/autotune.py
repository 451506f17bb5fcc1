"""Launch-shape autotuner for the ensemble kernels.

The best launch depends on the ensemble, not only on the problem: the plain
one-launch kernel wins when every trajectory is resident at once and step counts
are even; the persistent refill kernel wins when the ensemble outruns what the
device holds, or when step counts are uneven enough that warps would idle on one
long lane.  Block size moves the occupancy granularity.  So the choice is made by
measurement: each candidate launch is timed (CUDA events, after one warm-up
launch) on the caller's own inputs -- or on a leading sample of them for large
ensembles -- and the fastest is remembered per (problem, ensemble size, device).

Candidates: plain and persistent launches at 32, 64 and 128 threads per block,
the persistent grid at the occupancy limit or half of it.  Tuning is bounded in
time: a probe solve of the leading ``PROBE`` trajectories estimates the cost of
a full launch, and when timing every candidate on the whole ensemble would take
longer than ``BUDGET_S`` the candidates run on a leading sample instead (never
smaller than ``PROBE``).  When even that would blow the budget tenfold, no
candidate is timed: uneven step counts in the probe (max over mean above 2)
choose the persistent refill launch at half fill, even ones the plain launch.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass, replace

import torch

from menodax_b200 import _native
from menodax_b200._ensemble import launch
from menodax_b200._problem import get_problem

BLOCK_SIZES = (32, 64, 128)
PERSISTENT_FILL = (1.0, 0.5)
PROBE = 4096
BUDGET_S = 3.0


@dataclass(frozen=True)
class LaunchChoice:
    threads_per_block: int
    mode: int
    grid_fill: float  # persistent: fraction of the occupancy-limited grid

    def describe(self) -> str:
        kind = "plain" if self.mode == _native.MDX_LAUNCH_PLAIN else f"persistent(fill={self.grid_fill})"
        return f"{kind}, {self.threads_per_block} threads/block"


_cache: dict = {}
_lock = threading.Lock()


def candidates(block_sizes=BLOCK_SIZES):
    out = []
    for tpb in block_sizes:
        out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PLAIN, 0.0))
        for fill in PERSISTENT_FILL:
            out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PERSISTENT, fill))
    return out


def grid_blocks(problem, choice: LaunchChoice, n: int) -> int:
    if choice.mode == _native.MDX_LAUNCH_PLAIN:
        return 0
    per_sm, sms = problem.plan.occupancy(choice.mode)
    full = max(1, per_sm) * sms
    needed = (n + choice.threads_per_block - 1) // choice.threads_per_block
    return max(1, int(min(full, needed) * choice.grid_fill))


def tune(ode_fn, n_vars, n_params, options, *, y0, times, params, weights, dt0, rtol, atol,
         max_steps, n_save_hist=None, tune_block=True):
    """The fastest launch for this problem on these inputs (device tensors).

    With ``tune_block=False`` the block size stays ``options.threads_per_block``
    and only the launch kind and grid are chosen."""
    n = y0.shape[0]
    blocks = BLOCK_SIZES if tune_block else (options.threads_per_block,)
    key = (ode_fn, n_vars, n_params, replace(options, threads_per_block=32), n, blocks,
           torch.cuda.get_device_name(y0.device))
    with _lock:
        found = _cache.get(key)
    if found is not None:
        return found
    stream = torch.cuda.current_stream(y0.device)
    m = n
    if n > PROBE:
        prob = get_problem(ode_fn, n_vars, n_params, options)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, counters = launch(prob, y0=y0[:PROBE], times=times, params=params[:PROBE],
                             weights=weights[:PROBE] if weights is not None else None, dt0=dt0,
                             rtol=rtol, atol=atol, max_steps=max_steps,
                             mode=_native.MDX_LAUNCH_PLAIN, n_save_hist=n_save_hist)
        e1.record(stream)
        e1.synchronize()
        probe_s = e0.elapsed_time(e1) * 1e-3
        # A latency-bound launch costs about the same for the probe and a
        # full-device ensemble, so the probe time bounds one candidate launch.
        launches = 2 * len(candidates(blocks))
        if probe_s * launches > 10 * BUDGET_S:
            steps = counters[2].to(torch.float64)
            uneven = float(steps.max()) > 2.0 * float(steps.mean())
            tpb = options.threads_per_block if not tune_block else 64
            choice = (LaunchChoice(tpb, _native.MDX_LAUNCH_PERSISTENT, 0.5) if uneven
                      else LaunchChoice(options.threads_per_block, _native.MDX_LAUNCH_PLAIN, 0.0))
            with _lock:
                _cache[key] = choice
            return choice
        if probe_s * launches > BUDGET_S:
            m = PROBE
    ys, ps = y0[:m], params[:m]
    ws = weights[:m] if weights is not None else None
    best = None
    for choice in candidates(blocks):
        prob = get_problem(ode_fn, n_vars, n_params, replace(options, threads_per_block=choice.threads_per_block))
        kw = dict(y0=ys, times=times, params=ps, weights=ws, dt0=dt0, rtol=rtol, atol=atol,
                  max_steps=max_steps, mode=choice.mode, n_save_hist=n_save_hist,
                  grid_blocks=grid_blocks(prob, choice, m))
        launch(prob, **kw)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch(prob, **kw)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if best is None or ms < best[0]:
            best = (ms, choice)
    with _lock:
        _cache[key] = best[1]
    return best[1]


