"""Continuous forward sensitivities: the reference's differentiation method on the GPU.

``modax`` differentiates a solve by integrating the variational equation
``S' = J_y S + J_p`` alongside the state (``modax/_sensitivity.py:1-47``): one
joint system ``[y, S]`` of ``n_vars * (1 + n_sens)`` components, its sensitivity
right-hand side one directional derivative of ``ode_fn`` per direction, and --
in Rodas5P -- a block lower-triangular joint iteration matrix whose diagonal
blocks all equal ``M0 = I/(h gamma) - J``, so one factorisation serves every
block and the coupling ``L_k k_y`` is a second-order directional derivative
(``modax/rodas5P.py:513-565``).  This module runs that joint system through the
same kernels (the generated source carries the augmented writer, the
sensitivity ``df/dt`` rows and the coupling term).

Layout (``modax/_sensitivity.py:25-37``): ``z[j] = y[j]``,
``z[n + k * n + r] = S[r, k]``, the initial-state directions first, then the
parameter columns.  ``sens_error_control=False`` gives the sensitivity rows zero
weight and divides the error norm by ``n_vars``, which reproduces the plain
solve's step sequence exactly.

``jvp`` contracts ``S`` with input tangents the way the reference's custom_jvp
rule does (``modax/_sensitivity.py:388-411``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from menodax_b200 import _native, autotune
from menodax_b200._ensemble import initial_step, launch, normalize_y0_params, pick_device, to_device
from menodax_b200._problem import KernelOptions, get_problem

# Per joint-solve problem: the trajectories of the last call, longest first (by
# accepted steps), at most ORDER_HINT_PROBLEMS problems, oldest dropped first.
ORDER_HINT_PROBLEMS = 16
_order_hint: dict = {}


@dataclass(frozen=True)
class SensitivitySpec:
    """Which sensitivity blocks a joint solve carries (``modax/_sensitivity.py:64-135``)."""

    n_vars: int
    n_params: int
    wrt_y0: bool
    wrt_params: bool
    error_control: bool = True
    param_columns: tuple[int, ...] | None = None

    def __post_init__(self):
        if not (self.wrt_y0 or self.wrt_params):
            raise ValueError("a sensitivity spec must carry at least one direction block")
        if self.param_columns is not None:
            if len(set(self.param_columns)) != len(self.param_columns):
                raise ValueError("param_columns must not repeat a column")
            bad = [c for c in self.param_columns if not 0 <= c < self.n_params]
            if bad:
                raise ValueError(f"param_columns {bad} lie outside the {self.n_params} parameter columns")

    @property
    def n_y0_dirs(self) -> int:
        return self.n_vars if self.wrt_y0 else 0

    @property
    def param_seed_columns(self) -> tuple[int, ...]:
        if not self.wrt_params:
            return ()
        return tuple(range(self.n_params)) if self.param_columns is None else tuple(self.param_columns)

    @property
    def n_param_dirs(self) -> int:
        return len(self.param_seed_columns)

    @property
    def n_sens(self) -> int:
        return self.n_y0_dirs + self.n_param_dirs

    @property
    def n_aug(self) -> int:
        return self.n_vars * (1 + self.n_sens)

    @property
    def n_error(self) -> int:
        return self.n_aug if self.error_control else self.n_vars

    def kernel_sens(self):
        return (self.n_y0_dirs, self.param_seed_columns, bool(self.error_control))


def augmented_y0(y0: torch.Tensor, spec: SensitivitySpec) -> torch.Tensor:
    """``(n, n_vars)`` -> ``(n, n_aug)``: identity for the y0 block, zeros for parameters."""
    n = y0.shape[0]
    blocks = [y0]
    if spec.wrt_y0:
        eye = torch.eye(spec.n_vars, dtype=y0.dtype, device=y0.device).reshape(1, -1)
        blocks.append(eye.expand(n, -1))
    if spec.n_param_dirs:
        blocks.append(torch.zeros((n, spec.n_vars * spec.n_param_dirs), dtype=y0.dtype, device=y0.device))
    return torch.cat(blocks, dim=1).contiguous()


def split_augmented(hist: torch.Tensor, spec: SensitivitySpec):
    """``(n, S, n_aug)`` -> state ``(n, S, n_vars)`` and ``S`` ``(n, S, n_vars, n_sens)``."""
    n, s, _ = hist.shape
    state = hist[:, :, : spec.n_vars]
    sens = hist[:, :, spec.n_vars:].reshape(n, s, spec.n_sens, spec.n_vars)
    return state, sens.transpose(2, 3)


def solve(solver, ode_fn, y0, t_span, params, *, wrt_y0=True, wrt_params=True,
          sens_error_control=True, sens_param_columns=None, rtol=1e-8, atol=1e-10, first_step=None,
          max_steps=100000, return_stats=False, lu_precision="fp64", sparsity=None, ordering="amd",
          pcoeff=0.0, icoeff=1.0, dcoeff=0.0):
    """Solve the joint ``[y, S]`` system; returns ``(state, S)`` (plus stats) as torch tensors.

    ``solver`` is ``"tsit5"`` or ``"rodas5P"``.  ``S[n, s, r, k]`` is
    ``d y_r(t_s) / d theta_k`` for direction ``k`` (y0 directions first, then the
    parameter columns)."""
    if solver not in ("tsit5", "rodas5P"):
        raise ValueError(f"solver must be 'tsit5' or 'rodas5P'; got {solver!r}")
    y0_t, p_t, n, n_vars = normalize_y0_params(y0, params)
    n_params = p_t.shape[1]
    spec = SensitivitySpec(
        n_vars, n_params, bool(wrt_y0), bool(wrt_params), bool(sens_error_control),
        None if sens_param_columns is None else tuple(int(c) for c in sens_param_columns),
    )
    sparse = None
    if sparsity is not None:
        from menodax_b200._sparsity import normalize_sparsity

        sparse = normalize_sparsity(sparsity, n_vars)
    options = KernelOptions(
        solver=solver, lu_precision=lu_precision, sparsity=sparse, ordering=ordering,
        pcoeff=float(pcoeff), icoeff=float(icoeff), dcoeff=float(dcoeff), sens=spec.kernel_sens(),
    )
    device = pick_device(y0_t, p_t)
    problem = get_problem(ode_fn, n_vars, n_params, options)
    z0 = augmented_y0(to_device(y0_t.detach(), device), spec)
    if isinstance(t_span, torch.Tensor):
        times = t_span.detach().to(device=device, dtype=torch.float64).contiguous()
    else:
        times = torch.as_tensor(np.asarray(t_span, dtype=np.float64), device=device).contiguous()
    # The persistent refill launch, trajectories longest first by the previous
    # call's step counts for the same problem: the joint solves are long and
    # uneven, and the order only moves when each trajectory runs (the 2-state
    # stiff Van der Pol gradients of 65,536 trajectories: 324 ms plain, 207 ms
    # persistent, 163 ms persistent longest first; the same gradients bit for
    # bit).
    key = (ode_fn, n_vars, n_params, options, n, tuple(times.tolist()), float(rtol), float(atol))
    order = _order_hint.get(key)
    if order is not None and (order.device != device or order.numel() != n):
        order = None
    choice = autotune.LaunchChoice(problem.plan.tpb, _native.MDX_LAUNCH_PERSISTENT, 1.0)
    hist, counters = launch(problem, y0=z0, times=times, params=to_device(p_t.detach(), device),
                            weights=None, dt0=initial_step(first_step), rtol=rtol, atol=atol,
                            max_steps=max_steps, mode=_native.MDX_LAUNCH_PERSISTENT,
                            grid_blocks=autotune.grid_blocks(problem, choice, n), order=order)
    _order_hint.pop(key, None)
    _order_hint[key] = torch.argsort(counters[0], descending=True, stable=True).to(torch.int32)
    while len(_order_hint) > ORDER_HINT_PROBLEMS:
        _order_hint.pop(next(iter(_order_hint)))
    state, sens = split_augmented(hist, spec)
    if return_stats:
        from menodax_b200._ensemble import solver_stats

        return state, sens, solver_stats(counters[0], counters[1], counters[2])
    return state, sens


def jvp(solver, ode_fn, y0, t_span, params, dy0=None, dparams=None, **kw):
    """``(hist, tangent)``: the solve and its directional derivative along ``(dy0, dparams)``.

    Only the blocks with a tangent are integrated; ``sens_param_columns`` is not
    used here (every parameter column of ``dparams`` is carried)."""
    state, sens = solve(solver, ode_fn, y0, t_span, params, wrt_y0=dy0 is not None,
                        wrt_params=dparams is not None, **kw)
    n = state.shape[0]
    tangent = torch.zeros_like(state)
    offset = 0
    if dy0 is not None:
        d = torch.as_tensor(dy0, dtype=torch.float64, device=state.device)
        d = d.expand(n, -1) if d.ndim == 1 else d
        tangent = tangent + torch.einsum("nsij,nj->nsi", sens[..., : state.shape[2]], d)
        offset = state.shape[2]
    if dparams is not None:
        d = torch.as_tensor(dparams, dtype=torch.float64, device=state.device)
        d = d.expand(n, -1) if d.ndim == 1 else d
        tangent = tangent + torch.einsum("nsik,nk->nsi", sens[..., offset:], d)
    return state, tangent
