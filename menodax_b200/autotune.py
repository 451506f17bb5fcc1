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
the persistent grid at the occupancy limit or half of it; for fast FP32-LU
thread kernels of 9 to ``WIDE_TUNE_MAX_VARS`` states, each of those with the
stage solves in FP32 and in FP64 against the widened factors (which wins
depends on what the larger vectors do to register spills); for systems of
``TEAM_MIN_VARS`` states or more, also the team kernel (a team of 8 to 32 lanes
per trajectory, its vectors and matrix in shared memory), plain and persistent.
The thread kernel is a candidate up to ``THREAD_MAX_VARS`` states with a sparse
LU, and for dense LUs only while the matrix stays in registers
(``DENSE_UNROLL_MAX``): past that its matrix lives in local memory and a team is
faster by an order of magnitude.  For Tsit5 of up to 16 components the launches
with the stage vectors in shared memory (the reference's "shared" backend) are
candidates beside the register ones.

Tuning is bounded in time.  The first candidate runs on the whole ensemble
with at most ``PROBE_STEPS`` steps per trajectory.  When that finishes every
trajectory, its time is a launch's, and the candidates are timed in full, or on
the leading ``PROBE`` trajectories when that would exceed ``BUDGET_S``; the
persistent ones visit the trajectories longest first by the probe's step
counts, as the front end runs them once it has solved the problem before (a
warp of trajectories of about the same length finishes together).  When it
hits the step cap the integrations are long (tens of thousands of steps): the
plain candidates are ranked by the same capped run, which measures the cost of
a step with the ensemble resident, and the winner runs as a persistent refill
launch, since long stiff ensembles have uneven step counts.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass, replace

import torch

from menodax_b200 import _native
from menodax_b200._ensemble import launch
from menodax_b200._problem import (
    DENSE_UNROLL_MAX,
    STATIC_SHARED_MAX,
    WIDE_SOLVE_MAX_VARS,
    get_problem,
    team_block_threads,
    tsit5_stage_bytes,
    wide_solve_applies,
)
from menodax_b200._team import TEAM_SIZES

BLOCK_SIZES = (32, 64, 128)
PERSISTENT_FILL = (1.0, 0.5)
PROBE = 4096
PROBE_STEPS = 500
BUDGET_S = 3.0
TEAM_MIN_VARS = 16
SHARED_STAGES_MAX_VARS = 16   # the reference's bound for its shared Tsit5 backend
THREAD_MAX_VARS = 128
WIDE_TUNE_MAX_VARS = 64


@dataclass(frozen=True)
class LaunchChoice:
    threads_per_block: int
    mode: int
    grid_fill: float  # persistent: fraction of the occupancy-limited grid
    team: int = 0     # lanes per trajectory; 0 = one thread per trajectory
    shared_stages: bool = False  # Tsit5: stage vectors in shared memory
    wide_solve: bool | None = None  # fast FP32-LU thread kernels: FP64 stage solves; None = by size

    def describe(self) -> str:
        kind = "plain" if self.mode == _native.MDX_LAUNCH_PLAIN else f"persistent(fill={self.grid_fill})"
        lanes = f", team of {self.team}" if self.team else ""
        stages = ", stages in shared memory" if self.shared_stages else ""
        solves = "" if self.wide_solve is None else (", FP64 solves" if self.wide_solve else ", FP32 solves")
        return f"{kind}, {self.threads_per_block} threads/block{lanes}{stages}{solves}"


def options_for(options, choice: LaunchChoice):
    """``options`` with the launch choice's block size, team, stage placement and
    solve type."""
    return replace(options, threads_per_block=choice.threads_per_block, team=choice.team,
                   shared_stages=choice.shared_stages,
                   wide_solve=options.wide_solve if choice.wide_solve is None else choice.wide_solve)




_cache: dict = {}
_lock = threading.Lock()


def candidates(block_sizes=BLOCK_SIZES, teams=(), shared_blocks=(), shared_default=False, solves=(None,)):
    """Thread-kernel launches per block size (and per stage-solve type in
    ``solves``); team launches as ``(team, threads_per_block)`` pairs; Tsit5
    launches with shared-memory stages per block size in ``shared_blocks``."""
    out = []
    for wide in solves:
        for tpb in block_sizes:
            out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PLAIN, 0.0, 0, shared_default, wide))
            for fill in PERSISTENT_FILL:
                out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PERSISTENT, fill, 0, shared_default, wide))
    for tpb in shared_blocks:
        out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PLAIN, 0.0, 0, True))
        for fill in PERSISTENT_FILL:
            out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PERSISTENT, fill, 0, True))
    for team, tpb in teams:
        out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PLAIN, 0.0, team))
        out.append(LaunchChoice(tpb, _native.MDX_LAUNCH_PERSISTENT, 1.0, team))
    return out


def team_sizes_for(n_vars: int):
    """Teams worth timing: no wider than the system's state (rounded up to a power of two)."""
    return tuple(t for t in TEAM_SIZES if t // 2 < n_vars)


def grid_blocks(problem, choice: LaunchChoice, n: int) -> int:
    if choice.mode == _native.MDX_LAUNCH_PLAIN:
        return 0
    per_sm, sms = problem.plan.occupancy(choice.mode)
    full = max(1, per_sm) * sms
    per_block = choice.threads_per_block // max(1, choice.team)
    needed = (n + per_block - 1) // per_block
    return max(1, int(min(full, needed) * choice.grid_fill))


def streams_to_host(choice: LaunchChoice) -> bool:
    """Whether a solve whose results go to host memory should run the one-launch
    kernel of ``choice``'s module instead of ``choice`` itself.  A fully filled
    persistent thread launch is picked only for short integrations (every
    trajectory finished within the probe's step cap), where the history's trip
    across the host link takes longer than the kernel; the one-launch kernel's
    warps copy their rows to the host as they finish, which the persistent
    launch cannot do in whole rows, so it gets the history there sooner."""
    return choice.mode == _native.MDX_LAUNCH_PERSISTENT and choice.team == 0 and choice.grid_fill == 1.0


def longest_first(loop_steps: torch.Tensor) -> torch.Tensor:
    """The int32 visiting order of a persistent launch: trajectories by
    descending attempted steps (stable, so ties keep index order)."""
    return torch.argsort(loop_steps, descending=True, stable=True).to(torch.int32)


def _timed_launch(problem, choice, stream, *, n, y0, times, params, weights, dt0, rtol, atol, max_steps,
                  n_save_hist, order=None):
    kw = dict(y0=y0[:n], times=times, params=params[:n], weights=weights[:n] if weights is not None else None,
              dt0=dt0, rtol=rtol, atol=atol, max_steps=max_steps, mode=choice.mode, n_save_hist=n_save_hist,
              grid_blocks=grid_blocks(problem, choice, n), order=order)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _, counters = launch(problem, **kw)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3, counters


def tune(ode_fn, n_vars, n_params, options, *, y0, times, params, weights, dt0, rtol, atol,
         max_steps, n_save_hist=None, tune_block=True, tune_team=False, tune_shared=False):
    """The fastest launch for this problem on these inputs (device tensors).

    With ``tune_block=False`` the block size stays ``options.threads_per_block``
    and only the launch kind and grid are chosen.  With ``tune_team`` the team
    kernel is a candidate too (for systems of ``TEAM_MIN_VARS`` states or more);
    an ``options.team`` already set is kept and only its launch kind is tuned.
    With ``tune_shared`` (Tsit5) the launches with the stage vectors in shared
    memory are candidates beside the register ones; ``options.shared_stages``
    already set keeps them there.

    The first candidate runs once on the whole ensemble with at most
    ``PROBE_STEPS`` steps per trajectory.  If that finished every trajectory, its
    time is a launch's, and the candidates are timed in full (on the leading
    ``PROBE`` trajectories when that would exceed ``BUDGET_S``).  If it hit the
    step cap, the integrations are long: the plain launches are ranked by the
    same capped run -- the cost of a step with the ensemble resident -- and the
    winner runs as a persistent launch, which refills lanes as the uneven
    trajectories finish."""
    n = y0.shape[0]
    if options.team:
        blocks, teams = (), ((options.team, options.threads_per_block),)
    else:
        sizes = team_sizes_for(n_vars) if tune_team and n_vars >= TEAM_MIN_VARS else ()
        teams = []
        for t in sizes:
            try:
                teams.append((t, team_block_threads(n_vars, n_params, replace(options, team=t))))
            except ValueError:
                continue
        thread_ok = n_vars <= THREAD_MAX_VARS and (options.sparsity is not None or n_vars <= DENSE_UNROLL_MAX)
        if teams and not thread_ok:
            blocks = ()
        else:
            blocks = BLOCK_SIZES if tune_block else (options.threads_per_block,)
    shared_blocks = ()
    if tune_shared and options.solver == "tsit5" and not options.shared_stages and n_vars <= SHARED_STAGES_MAX_VARS:
        shared_blocks = tuple(b for b in blocks if tsit5_stage_bytes(n_vars, b) <= STATIC_SHARED_MAX)
    solves = (None,)
    if (wide_solve_applies(options) and options.wide_solve is None
            and WIDE_SOLVE_MAX_VARS < n_vars <= WIDE_TUNE_MAX_VARS):
        solves = (False, True)
    cands = candidates(blocks, teams, shared_blocks, options.shared_stages, solves)
    key = (ode_fn, n_vars, n_params, replace(options, threads_per_block=32, team=0, shared_stages=False), n,
           tuple(cands), max_steps, torch.cuda.get_device_name(y0.device))
    with _lock:
        found = _cache.get(key)
    if found is not None:
        return found

    def problem_for(choice):
        return get_problem(ode_fn, n_vars, n_params, options_for(options, choice))

    buildable = []
    for choice in cands:
        try:
            problem_for(choice)
        except ValueError:  # a team slice too large for a block's shared memory
            continue
        buildable.append(choice)
    if not buildable:
        raise ValueError("no launch candidate fits this problem")
    stream = torch.cuda.current_stream(y0.device)
    inputs = dict(y0=y0, times=times, params=params, weights=weights, dt0=dt0, rtol=rtol, atol=atol,
                  n_save_hist=n_save_hist)
    m = min(n, PROBE)
    cap = min(int(max_steps), PROBE_STEPS)
    first = replace(buildable[0], mode=_native.MDX_LAUNCH_PLAIN, grid_fill=0.0)
    probe_s, counters = _timed_launch(problem_for(first), first, stream, n=n, max_steps=cap, **inputs)
    capped = cap < int(max_steps) and int(counters[2].max()) >= cap
    if capped:
        best = None
        for choice in buildable:
            if choice.mode != _native.MDX_LAUNCH_PLAIN:
                continue
            prob = problem_for(choice)
            _timed_launch(prob, choice, stream, n=n, max_steps=cap, **inputs)
            secs, _ = _timed_launch(prob, choice, stream, n=n, max_steps=cap, **inputs)
            if best is None or secs < best[0]:
                best = (secs, choice)
        winner = best[1]
        fill = 1.0 if winner.team else 0.5
        persistent = [c for c in buildable if c.mode == _native.MDX_LAUNCH_PERSISTENT and c.team == winner.team
                      and c.threads_per_block == winner.threads_per_block and c.grid_fill == fill
                      and c.shared_stages == winner.shared_stages and c.wide_solve == winner.wide_solve]
        choice = persistent[0] if persistent else winner
        with _lock:
            _cache[key] = choice
        return choice
    # The probe ran to completion; a latency-bound launch costs about the same
    # for the probe set and a full-device ensemble, so it bounds one candidate.
    launches = 2 * len(buildable)
    sample = n if probe_s * launches <= BUDGET_S else m
    # Persistent candidates are timed as the front end runs them once a problem
    # has been solved: longest first by the probe's step counts, so each warp
    # takes trajectories of about the same length.
    order = longest_first(counters[2][:sample])
    best = None
    for choice in buildable:
        prob = problem_for(choice)
        visit = order if choice.mode == _native.MDX_LAUNCH_PERSISTENT else None
        _timed_launch(prob, choice, stream, n=sample, max_steps=max_steps, order=visit, **inputs)
        secs, _ = _timed_launch(prob, choice, stream, n=sample, max_steps=max_steps, order=visit, **inputs)
        if best is None or secs < best[0]:
            best = (secs, choice)
    with _lock:
        _cache[key] = best[1]
    return best[1]
