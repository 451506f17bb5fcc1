"""The common body of ``tsit5.solve`` and ``rodas5P.solve``.

Inputs may be NumPy arrays (results come back as NumPy, like the reference's
host-array calls) or torch tensors (results stay on their CUDA device; CPU
tensors are copied in and the results copied back).  A torch input that
requires grad routes through the discrete adjoint (``menodax_b200.autograd``).
"""

from __future__ import annotations

import numpy as np
import torch

from menodax_b200 import _native
from menodax_b200._ensemble import (
    build_error_weights,
    initial_step,
    launch,
    normalize_y0_params,
    pick_device,
    solver_stats,
    to_device,
)
from menodax_b200._problem import KernelOptions, get_problem
from menodax_b200.autotune import longest_first

LAUNCH_MODES = ("auto", "plain", "persistent")

# Per problem (the compiled options, ensemble size, save times, tolerances and
# step cap): the trajectories of the last persistent launch, most attempted
# steps first.  The next persistent launch of the same problem takes them in that
# order, so the long integrations start in the grid's first wave instead of
# setting the makespan from a late one (the 64-state Brusselator's 16,384
# trajectories 16.9 -> 15.0 ms, the 32-state Van der Pol ring's 32,768 7.5 ->
# 4.1 s); every trajectory's integration, and so the result, is the same in any
# order.  At most ORDER_HINT_PROBLEMS problems are remembered, oldest dropped
# first.
ORDER_HINT_PROBLEMS = 16
_order_hint: dict = {}


def _remember_order(key, order) -> None:
    _order_hint.pop(key, None)
    _order_hint[key] = order
    while len(_order_hint) > ORDER_HINT_PROBLEMS:
        _order_hint.pop(next(iter(_order_hint)))


def _is_torch(*xs):
    return any(isinstance(x, torch.Tensor) for x in xs)


def _times_tensor(t_span):
    if isinstance(t_span, torch.Tensor):
        t = t_span.detach().to(torch.float64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(t_span, dtype=np.float64)))
    if t.ndim != 1 or t.shape[0] < 1:
        raise ValueError(f"t_span must be a 1-D array of save times; got shape {tuple(t.shape)}")
    return t


# Below this many trajectories a launch is one partial wave whatever its shape,
# and the reference's own choice (one warp per block, one launch) is kept.
AUTOTUNE_MIN_TRAJECTORIES = 4096


def resolve_mode(launch_mode: str) -> int:
    if launch_mode not in LAUNCH_MODES:
        raise ValueError(f"launch must be one of {LAUNCH_MODES}; got {launch_mode!r}")
    if launch_mode == "persistent":
        return _native.MDX_LAUNCH_PERSISTENT
    return _native.MDX_LAUNCH_PLAIN


def run(ode_fn, y0, t_span, params, options: KernelOptions, *, rtol, atol, first_step,
        max_steps, return_stats, error_weights, launch_mode="auto", grid_blocks=0, tune_block=True,
        tune_team=False, tune_shared=False):
    torch_io = _is_torch(y0, params)
    y0_t, p_t, n, n_vars = normalize_y0_params(y0, params)
    n_params = p_t.shape[1]
    times = _times_tensor(t_span)
    weights = build_error_weights(error_weights, n, n_vars)
    if weights is not None:
        options = _replace(options, runtime_weights=True)
    if options.tf_index >= 0 and not options.tf_index < n_params:
        raise ValueError(f"tf_index {options.tf_index} is outside the {n_params} parameter columns")
    if int(max_steps) < 0:
        raise ValueError("max_steps must be non-negative")
    device = pick_device(y0_t, p_t)
    mode = resolve_mode(launch_mode)
    y0_d = to_device(y0_t.detach(), device)
    p_d = to_device(p_t.detach(), device)
    t_d = to_device(times, device)
    w_d = to_device(weights.detach(), device) if weights is not None else None
    n_hist = None if options.save_history else 1
    common = dict(y0=y0_d, times=t_d, params=p_d, weights=w_d, dt0=initial_step(first_step),
                  rtol=rtol, atol=atol, max_steps=max_steps, n_save_hist=n_hist)
    hook_out = None
    if options.save_hook is not None:
        hook_out = torch.empty((n, options.hook_size), dtype=torch.float64, device=device)
    input_on_gpu = any(isinstance(x, torch.Tensor) and x.is_cuda for x in (y0, params))
    host_results = not (torch_io and input_on_gpu)
    if launch_mode == "auto" and n >= AUTOTUNE_MIN_TRAJECTORIES and hook_out is None:
        from menodax_b200 import autotune

        choice = autotune.tune(ode_fn, n_vars, n_params, options, tune_block=tune_block,
                               tune_team=tune_team, tune_shared=tune_shared, **common)
        options = autotune.options_for(options, choice)
        problem = get_problem(ode_fn, n_vars, n_params, options)
        mode = choice.mode
        grid_blocks = autotune.grid_blocks(problem, choice, n)
        if host_results and autotune.streams_to_host(choice):
            mode = _native.MDX_LAUNCH_PLAIN
            grid_blocks = 0
    else:
        problem = get_problem(ode_fn, n_vars, n_params, options)
    n_save = int(t_d.shape[0])
    for name, length, lo, hi in problem.hook_tables:
        if lo < 0 or n_save - 1 + hi >= length:
            raise ValueError(
                f"the save hook reads or writes {name} at save_idx + {hi if lo >= 0 else lo}, "
                f"outside its {length} entries for {n_save} save times"
            )
    hist_h = None
    streamed = False
    if host_results:
        hist_h = torch.empty((n, n_save if options.save_history else 1, problem.n_system),
                             dtype=torch.float64, pin_memory=True)
        # Host results of a one-launch solve: each warp (or team) writes its
        # finished rows into the pinned buffer itself, overlapping the rest of the
        # solve.  The persistent launch finishes one lane's row at a time, too
        # small a write for the host link, so its history is copied afterwards.
        streamed = mode == _native.MDX_LAUNCH_PLAIN
    order = None
    order_key = None
    if mode == _native.MDX_LAUNCH_PERSISTENT:
        order_key = (ode_fn, n_vars, n_params, options, n, tuple(times.tolist()), float(rtol), float(atol),
                     int(max_steps), int(grid_blocks))
        order = _order_hint.get(order_key)
        if order is not None and (order.device != device or order.numel() != n):
            order = None
    hist, counters = launch(problem, mode=mode, grid_blocks=grid_blocks, hook_out=hook_out,
                            hist_host=hist_h if streamed else None, order=order, **common)
    if order_key is not None and n > 0:
        _remember_order(order_key, longest_first(counters[2]))
    if hist_h is None:
        result = (hist,) if hook_out is None else (hist, hook_out)
        if return_stats:
            result += (solver_stats(counters[0], counters[1], counters[2], counters[3]),)
        return result[0] if len(result) == 1 else result
    counters_h = _to_host(hist, None if streamed else hist_h, counters if return_stats else None)
    hook_h = None
    if hook_out is not None:
        hook_h = torch.empty(hook_out.shape, dtype=hook_out.dtype, pin_memory=True)
        hook_h.copy_(hook_out)
    if not torch_io:
        hist_h = hist_h.numpy()
        counters_h = counters_h.numpy() if counters_h is not None else None
        hook_h = hook_h.numpy() if hook_h is not None else None
    result = (hist_h,) if hook_h is None else (hist_h, hook_h)
    if return_stats:
        result += (solver_stats(counters_h[0], counters_h[1], counters_h[2], counters_h[3]),)
    return result[0] if len(result) == 1 else result


def _to_host(hist, hist_h, counters):
    """Copies the history (unless the kernel wrote it to ``hist_h`` itself) and
    the step counters to pinned host memory, and waits for the stream."""
    if hist_h is not None:
        hist_h.copy_(hist, non_blocking=True)
    counters_h = None
    if counters is not None:
        counters_h = torch.empty(counters.shape, dtype=counters.dtype, pin_memory=True)
        counters_h.copy_(counters, non_blocking=True)
    torch.cuda.current_stream(hist.device).synchronize()
    return counters_h


def _replace(options, **kw):
    from dataclasses import replace

    return replace(options, **kw)
