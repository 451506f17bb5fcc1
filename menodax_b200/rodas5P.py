"""Rodas5P ensemble solve: the drop-in for ``modax.rodas5P.solve``.

Same signature and defaults as ``modax/rodas5P.py:1024-1051``, same errors
(``modax/rodas5P.py:1204-1211``), same outputs: ``hist (N, S, n_vars)`` or
``(hist, stats)``.  Extra keyword ``launch`` picks the one-launch kernel
(``"plain"``), the persistent refill kernel (``"persistent"``) or lets the
library choose (``"auto"``); ``team`` picks one thread or a team of lanes per
trajectory.
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import torch

from menodax_b200._frontend import run
from menodax_b200._problem import KernelOptions, team_block_threads
from menodax_b200._sparsity import normalize_sparsity
from menodax_b200._team import TEAM_SIZES

_DEFAULT_TRAJECTORIES_PER_BLOCK = 32
LU_PRECISIONS = ("fp32", "fp64")


def trajectories_per_block_or_default(requested=None) -> int:
    """Trajectories a block carries, one per thread (``modax/rodas5P.py:118-134``)."""
    if requested is None:
        return _DEFAULT_TRAJECTORIES_PER_BLOCK
    requested = int(requested)
    if requested < 1:
        raise ValueError(f"trajectories_per_block must be positive, got {requested}")
    return requested


def _block_size(requested: int) -> int:
    # Warp ballots need whole warps, so a block is rounded up to them.
    return max(32, (requested + 31) // 32 * 32)


def solve(
    ode_fn,
    y0,
    t_span,
    params,
    *,
    rtol=1e-8,
    atol=1e-10,
    first_step=None,
    max_steps=100000,
    return_stats=False,
    error_weights=None,
    pcoeff=0.0,
    icoeff=1.0,
    dcoeff=0.0,
    lu_precision: str = "fp32",
    trajectories_per_block=None,
    sens_error_control=True,
    sens_param_columns=None,
    sparsity=None,
    ordering="amd",
    tf_index=None,
    max_registers=None,
    array_rhs=None,
    save_hook=None,
    hook_size: int = 0,
    save_history: bool = True,
    launch: str = "auto",
    sparse_code: str = "auto",
    arithmetic: str = "auto",
    team="auto",
):
    """Rodas5P ensemble solve of ``y' = ode_fn(y, t, p)`` on one GPU.

    ``lu_precision`` selects the precision of the iteration matrix, its LU and
    the stored stage increments; the state, right-hand side, Jacobian, error and
    controller are always double.  ``arithmetic="reference"`` rounds exactly
    where the reference does (double multipliers in the LU, divisions in the
    substitutions, a double-precision controller power); ``"fast"`` runs the LU
    wholly in the LU type with the reciprocal diagonal multiplied in (in FP32
    the approximate reciprocal), forms 1/h and the error scales' reciprocals
    from a float seed and one double Newton step, and takes the controller
    power of the squared error norm in float (no square root).  ``"auto"`` is
    fast for ``lu_precision="fp32"`` and reference for ``"fp64"``.
    ``sparsity`` (a mask, a scipy sparse matrix or
    ``(nnz, 2)`` pairs) colours the Jacobian sweep and compiles a sparse LU for the
    pattern, ordered by ``ordering`` (``"amd"`` or ``"natural"``).  ``tf_index``
    names a parameter column holding each trajectory's own end time.

    ``team`` picks the kernel layout: ``0`` runs one trajectory per thread with
    its vectors and matrix in registers (the reference's layout); ``4``, ``8``,
    ``16`` or ``32`` give each trajectory a team of that many lanes with its
    vectors and matrix in shared memory; ``"auto"`` leaves the choice to the
    launch autotuner, which considers teams for systems of
    ``autotune.TEAM_MIN_VARS`` or more states.  Teams run no forward
    sensitivities; a save hook runs on a team's first lane; with a sparsity pattern and
    ``sens_error_control=False`` a team also runs the discrete adjoint (its
    checkpointing forward pass and its reverse sweep).

    ``array_rhs(y, t, p, out)`` (optional) is the same right-hand side written as
    an array writer, ``out[i] = ...`` for every component; it is traced like
    ``ode_fn`` and evaluates the stages, while the Jacobian, ``df/dt`` and every
    derivative are still taken from ``ode_fn`` (``modax/rodas5P.py:382-391``).
    The two must compute the same function.

    ``save_hook(save_idx, y, t, p_row, acc)`` runs inside the kernel at every save
    (the initial state, each dense-output save, the frozen saves past a
    trajectory's end) on the state at that time; it is traced like ``ode_fn``:
    ``acc`` is the trajectory's ``hook_size``-wide row, zeroed at the start,
    indexed with literals or with ``save_idx`` (plus a literal offset), and host
    arrays it closes over may be indexed with ``save_idx`` too.  A hooked solve
    returns ``(hist, hook_out)`` (plus the stats when asked); with
    ``save_history=False`` ``hist`` keeps only the final state, shape
    ``(N, 1, n_vars)`` (``modax/rodas5P.py:1161-1171``).

    Torch inputs that require grad are differentiated by the discrete adjoint
    (checkpointed step states, reverse sweep on the device).
    """
    if lu_precision not in LU_PRECISIONS:
        raise ValueError(f"lu_precision must be one of {LU_PRECISIONS}; got {lu_precision!r}")
    if arithmetic not in ("auto", "reference", "fast"):
        raise ValueError(f"arithmetic must be 'auto', 'reference' or 'fast'; got {arithmetic!r}")
    fast = arithmetic == "fast" or (arithmetic == "auto" and lu_precision == "fp32")
    if array_rhs is not None and not callable(array_rhs):
        raise ValueError("array_rhs must be a callable array_rhs(y, t, p, out)")
    if save_hook is not None:
        if hook_size <= 0:
            raise ValueError("a save_hook needs a positive hook_size")
    elif not save_history:
        raise ValueError("save_history=False needs a save_hook to consume the saves")
    n_vars = int(torch.as_tensor(y0).shape[-1]) if not hasattr(y0, "shape") else int(y0.shape[-1])
    team_choice = _team_option(team)
    if sparsity is not None:
        sparsity = normalize_sparsity(sparsity, n_vars)
    tpb = trajectories_per_block_or_default(trajectories_per_block)
    options = KernelOptions(
        solver="rodas5P",
        pcoeff=float(pcoeff),
        icoeff=float(icoeff),
        dcoeff=float(dcoeff),
        lu_precision=lu_precision,
        threads_per_block=_block_size(tpb),
        sparsity=sparsity,
        ordering=ordering,
        sparse_code=sparse_code,
        tf_index=-1 if tf_index is None else int(tf_index),
        max_registers=max_registers,
        save_history=bool(save_history),
        fast=fast,
        save_hook=save_hook,
        hook_size=int(hook_size) if save_hook is not None else 0,
        array_rhs=array_rhs,
    )
    from menodax_b200.autograd import needs_grad, solve_with_grad

    grad = needs_grad(y0, params)
    if team_choice:
        if grad and (sparsity is None or sens_error_control):
            raise ValueError("team gradients run the discrete adjoint over a sparse LU: pass a sparsity "
                             "pattern and sens_error_control=False")
        options = replace(options, team=team_choice)
        if not grad:
            options = replace(options, threads_per_block=team_block_size(
                team_choice, trajectories_per_block, n_vars, _n_params(params), options))
    if grad:
        if save_hook is not None:
            raise NotImplementedError("a solve with a save_hook is not differentiable")
        return solve_with_grad(
            ode_fn, y0, t_span, params, options, rtol=rtol, atol=atol, first_step=first_step,
            max_steps=max_steps, return_stats=return_stats, error_weights=error_weights,
            sens_error_control=bool(sens_error_control), sens_param_columns=sens_param_columns,
        )
    return run(
        ode_fn, y0, t_span, params, options, rtol=rtol, atol=atol, first_step=first_step,
        max_steps=max_steps, return_stats=return_stats, error_weights=error_weights,
        launch_mode=launch, tune_block=trajectories_per_block is None,
        tune_team=team == "auto" and save_hook is None,
    )


def _team_option(team) -> int:
    if team == "auto":
        return 0
    if team in (0, None):
        return 0
    if team not in TEAM_SIZES:
        raise ValueError(f"team must be 'auto', 0 or one of {TEAM_SIZES}; got {team!r}")
    return int(team)


def _n_params(params) -> int:
    shape = params.shape if hasattr(params, "shape") else np.shape(params)
    return int(shape[-1]) if len(shape) else 1


def team_block_size(team: int, trajectories_per_block, n_vars: int, n_params: int, options) -> int:
    """Threads per block of a team launch: ``trajectories_per_block`` teams, by default
    up to 128 threads as the block's shared memory allows."""
    if trajectories_per_block is None:
        return team_block_threads(n_vars, n_params, options)
    threads = int(trajectories_per_block) * team
    if threads % 32 or threads > 1024:
        raise ValueError(
            f"trajectories_per_block={trajectories_per_block} with team={team} gives {threads} threads; "
            "a block must be whole warps, at most 1024 threads")
    return threads
