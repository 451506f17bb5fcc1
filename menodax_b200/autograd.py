"""torch.autograd front end: the discrete adjoint of an ensemble solve.

``rodas5P.solve`` / ``tsit5.solve`` route here when a torch input requires
grad.  The forward pass runs the checkpointing kernel, which records one
``(t, h, y)`` step state per accepted step; ``backward`` launches the reverse
kernel (``mdx_grad`` in the C ABI), which replays every accepted step from its
state and returns the cotangents of ``y0`` and ``params``.  Step sizes are
constants of the discrete map, so the gradient is the exact derivative of the
solution the forward pass produced -- for that step sequence it equals what the
reference's forward sensitivities give with ``sens_error_control=False``
(``modax/_sensitivity.py:331-413``), computed backwards in one sweep whatever
the number of parameters.
"""

from __future__ import annotations

from dataclasses import replace

import torch

from menodax_b200 import _native
from menodax_b200._ensemble import initial_step, launch, pick_device, solver_stats
from menodax_b200._problem import get_problem

# Checkpoint capacity (accepted steps per trajectory) last seen per problem, so a
# repeated gradient call allocates once and runs the forward pass once.
_capacity_hint: dict = {}


def needs_grad(*xs) -> bool:
    return torch.is_grad_enabled() and any(isinstance(x, torch.Tensor) and x.requires_grad for x in xs)


def _as_double(x, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64)
    return torch.as_tensor(x, dtype=torch.float64, device=device)


class _EnsembleSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y0, params, times, problem, dt0, rtol, atol, max_steps, key):
        n = y0.shape[0]
        n_vars = problem.n_vars
        y0c = y0.detach().contiguous()
        pc = params.detach().contiguous()
        capacity = _capacity_hint.get(key, 256)
        while True:
            ckpt = torch.empty((capacity, n, n_vars + 2), dtype=torch.float64, device=y0.device)
            ckpt_count = torch.empty(n, dtype=torch.int32, device=y0.device)
            hist, counters = launch(
                problem, y0=y0c, times=times, params=pc, weights=None, dt0=dt0, rtol=rtol, atol=atol,
                max_steps=max_steps, mode=_native.MDX_LAUNCH_PLAIN, ckpt=ckpt,
                ckpt_count=ckpt_count, ckpt_capacity=capacity,
            )
            needed = int(counters[0].max().item()) if n else 0
            if needed <= capacity:
                break
            capacity = int(needed * 1.1) + 8
            del ckpt
        _capacity_hint[key] = max(needed + 8, int(needed * 1.1))
        ctx.problem = problem
        ctx.capacity = capacity
        ctx.save_for_backward(pc, times, ckpt, ckpt_count)
        ctx.mark_non_differentiable(counters)
        return hist, counters

    @staticmethod
    def backward(ctx, grad_hist, _grad_counters):
        params, times, ckpt, ckpt_count = ctx.saved_tensors
        problem = ctx.problem
        n = params.shape[0]
        g = grad_hist.contiguous() if grad_hist is not None else torch.zeros(
            (n, times.numel(), problem.n_vars), dtype=torch.float64, device=params.device)
        grad_y0 = torch.empty((n, problem.n_vars), dtype=torch.float64, device=params.device)
        grad_p = torch.empty((n, problem.n_params), dtype=torch.float64, device=params.device)
        status = torch.empty(n, dtype=torch.int32, device=params.device)
        d = _native.GradDesc()
        d.n_traj = n
        d.n_save = times.numel()
        d.times = times.data_ptr()
        d.params = params.data_ptr() if params.numel() else None
        d.ckpt = ckpt.data_ptr()
        d.ckpt_count = ckpt_count.data_ptr()
        d.ckpt_capacity = ctx.capacity
        d.grad_hist = g.data_ptr()
        d.grad_y0 = grad_y0.data_ptr()
        d.grad_params = grad_p.data_ptr()
        d.status = status.data_ptr()
        stream = torch.cuda.current_stream(params.device).cuda_stream
        with torch.cuda.device(params.device):
            problem.plan.grad(d, stream)
        return grad_y0, grad_p, None, None, None, None, None, None, None


def solve_with_grad(ode_fn, y0, t_span, params, options, *, rtol, atol, first_step, max_steps,
                    return_stats, error_weights):
    """Differentiable ensemble solve; returns torch tensors on the solve's device."""
    if error_weights is not None:
        raise NotImplementedError("error_weights are not supported together with gradients")
    device = pick_device(y0, params)
    y0_t = _as_double(y0, device)
    p_t = _as_double(params, device)
    if y0_t.ndim not in (1, 2) or p_t.ndim not in (1, 2):
        raise ValueError("y0 must be (n_vars,) or (N, n_vars) and params (n_params,) or (N, n_params)")
    n = y0_t.shape[0] if y0_t.ndim == 2 else (p_t.shape[0] if p_t.ndim == 2 else 1)
    if y0_t.ndim == 2 and p_t.ndim == 2 and p_t.shape[0] != n:
        raise ValueError("params must have as many rows as y0")
    if y0_t.ndim == 1:
        y0_t = y0_t.unsqueeze(0).expand(n, -1)
    if p_t.ndim == 1:
        p_t = p_t.unsqueeze(0).expand(n, -1)
    n_vars, n_params = y0_t.shape[1], p_t.shape[1]
    if isinstance(t_span, torch.Tensor):
        times = t_span.detach().to(device=device, dtype=torch.float64).contiguous()
    else:
        times = torch.as_tensor(t_span, dtype=torch.float64, device=device).contiguous()
    opts = replace(options, checkpoint=True, adjoint=True, runtime_weights=False)
    problem = get_problem(ode_fn, n_vars, n_params, opts)
    key = (ode_fn, n_vars, n_params, opts, n, tuple(times.tolist()), float(rtol), float(atol))
    hist, counters = _EnsembleSolve.apply(y0_t, p_t, times, problem, initial_step(first_step), rtol,
                                          atol, max_steps, key)
    if return_stats:
        return hist, solver_stats(counters[0], counters[1], counters[2])
    return hist
