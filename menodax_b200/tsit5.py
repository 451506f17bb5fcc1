"""Tsit5 ensemble solve: the drop-in for ``modax.tsit5.solve``.

Same signature and defaults as ``modax/tsit5.py:623-641``.  ``backend`` is
validated as the reference does (``modax/tsit5.py:123-139``) and picks where the
stage vectors k1..k6 live: ``"local"`` in registers (every component index is a
literal, so they are register arrays), ``"shared"`` in a shared-memory array of
one column per thread, ``"auto"`` whichever the launch autotuner measures faster
(registers when the ensemble is too small to tune).  The arithmetic is the same
either way, so the choices give the same numbers.
"""

from __future__ import annotations

from dataclasses import replace

from menodax_b200._frontend import run
from menodax_b200._problem import KernelOptions

_SHARED_MAX_NVARS = 16
_SHARED_MAX_ENSEMBLE = 16384


def _use_shared_backend(n: int, n_system: int, backend: str) -> bool:
    if backend == "local":
        return False
    if backend == "shared":
        if n_system > _SHARED_MAX_NVARS:
            raise ValueError(
                "shared backend requires a system size <= "
                f"{_SHARED_MAX_NVARS}; got {n_system}. A solve carrying forward "
                "sensitivities integrates n_vars * (1 + n_sens) components, so "
                "it may need backend='local' where the plain solve does not"
            )
        return True
    if backend != "auto":
        raise ValueError(f"backend must be 'auto', 'shared', or 'local'; got {backend!r}")
    return n_system <= _SHARED_MAX_NVARS and n <= _SHARED_MAX_ENSEMBLE


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
    backend="auto",
    sens_error_control=True,
    sens_param_columns=None,
    launch: str = "auto",
):
    """Tsit5 ensemble solve of ``y' = ode_fn(y, t, p)`` on one GPU."""
    shape = getattr(y0, "shape", None)
    import numpy as np

    y0_shape = shape if shape is not None else np.shape(y0)
    n_vars = int(y0_shape[-1])
    n = int(y0_shape[0]) if len(y0_shape) == 2 else 1
    _use_shared_backend(n, n_vars, backend)
    options = KernelOptions(
        solver="tsit5", pcoeff=float(pcoeff), icoeff=float(icoeff), dcoeff=float(dcoeff),
        threads_per_block=32,
    )
    from menodax_b200.autograd import needs_grad, solve_with_grad

    if needs_grad(y0, params):
        # The discrete adjoint's kernels keep their vectors in registers.
        return solve_with_grad(
            ode_fn, y0, t_span, params, options, rtol=rtol, atol=atol, first_step=first_step,
            max_steps=max_steps, return_stats=return_stats, error_weights=error_weights,
            sens_error_control=bool(sens_error_control), sens_param_columns=sens_param_columns,
        )
    return run(
        ode_fn, y0, t_span, params, replace(options, shared_stages=backend == "shared"), rtol=rtol,
        atol=atol, first_step=first_step, max_steps=max_steps, return_stats=return_stats,
        error_weights=error_weights, launch_mode=launch, tune_block=backend != "shared",
        tune_shared=backend == "auto",
    )
