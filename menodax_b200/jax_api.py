"""JAX front end: the solvers callable under ``jit``, ``vmap`` as one ensemble launch.

The reference's JAX surface (``modax/_jax_common.py:70-111``,
``modax/_jax_numba_custom_call.py:145-231, 262-371``,
``modax/_sensitivity.py:331-413``), over this library's C ABI:

* **Custom calls.**  Two XLA FFI handlers, ``mdx_xla_solve`` and
  ``mdx_xla_grad`` (``csrc/mdx_xla_ffi.cc``), wrap ``mdx_solve`` and
  ``mdx_grad``; ``register_targets`` builds them against
  ``jax.ffi.include_dir()`` (once, in-tree) and registers them for CUDA.  A
  call passes the compiled problem's plan as an attribute; XLA owns every
  buffer, the persistent launch's queue head included (an extra ``uint8``
  output, as the reference returns its scratch arrays).
* **vmap.**  ``custom_vmap`` folds a ``vmap`` over ``y0`` and/or ``params`` into
  the ensemble axis of one launch (``vmap_rule``, the reference's rule); a
  batched ``t_span`` is accepted only as a broadcast constant.
* **Differentiation**, picked by ``sens_error_control`` as in the torch front
  end: ``True`` (the default) attaches the reference's ``custom_jvp`` over the
  joint ``[y, S]`` forward-sensitivity solve (``contract_tangent``; JAX
  transposes its linear contraction for ``grad``); ``False`` attaches a
  ``custom_vjp`` whose forward pass records checkpoints and whose backward pass
  is the discrete adjoint's reverse kernel (``mask_adjoint`` on its output).  The adjoint's
  checkpoint buffer has a static size under ``jit``: ``adjoint_capacity``
  accepted steps per trajectory (default 4096); a trajectory that takes more
  gets NaN gradients (its status carries the overflow bit).

JAX is an optional dependency; importing this module needs none, calling a
solver does.
"""

from __future__ import annotations

import ctypes
import subprocess
from dataclasses import replace
from pathlib import Path

import numpy as np

from menodax_b200 import _native
from menodax_b200._problem import KernelOptions, get_problem

SOLVE_TARGET = "mdx_xla_solve"
GRAD_TARGET = "mdx_xla_grad"
WORKSPACE_BYTES = 256
ADJOINT_STRIDE = 8
HANDLER_SRC = Path(__file__).resolve().parent / "csrc" / "mdx_xla_ffi.cc"
HANDLER_LIB = Path(__file__).resolve().parent / "libmenodax_b200_xla.so"

_registered = False


def _jax():
    try:
        import jax  # noqa: PLC0415
    except ImportError as exc:
        raise ImportError(
            "menodax_b200.jax_api needs JAX with CUDA; the torch front end "
            "(menodax_b200.rodas5P.solve / tsit5.solve) needs only torch") from exc
    return jax


# --------------------------------------------------------------------------- custom calls
def build_handler(include_dir: str, force: bool = False) -> Path:
    """Compile the XLA FFI handlers against JAX's FFI headers into the package."""
    lib = _native.build_library()
    if HANDLER_LIB.exists() and not force and HANDLER_LIB.stat().st_mtime >= HANDLER_SRC.stat().st_mtime:
        return HANDLER_LIB
    cuda = _native.CUDA_HOME
    subprocess.run(
        ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{include_dir}", f"-I{cuda / 'include'}",
         str(HANDLER_SRC), "-o", str(HANDLER_LIB), f"-L{lib.parent}", "-lmenodax_b200",
         f"-Wl,-rpath,{lib.parent}"], check=True)
    return HANDLER_LIB


def register_targets() -> None:
    """Register ``mdx_xla_solve`` and ``mdx_xla_grad`` with XLA for CUDA, once per process."""
    global _registered
    if _registered:
        return
    jax = _jax()
    lib = ctypes.CDLL(str(build_handler(jax.ffi.include_dir())))
    for name in (SOLVE_TARGET, GRAD_TARGET):
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(lib, name)), platform="CUDA")
    _registered = True


def plan_address(problem) -> int:
    """The ``mdx_plan*`` of a compiled problem, as the int64 attribute the handlers take."""
    return int(ctypes.cast(problem.plan.handle, ctypes.c_void_p).value or 0)


def solve_call_args(problem, n: int, n_save: int, *, mode: int, dt0, rtol, atol, max_steps,
                    ckpt_capacity: int = 0):
    """``(output shapes and dtypes, attributes)`` of one ``mdx_xla_solve`` call."""
    n_hist = n_save if problem.options.save_history else 1
    if ckpt_capacity:
        words = problem.plan.checkpoint_size(n, ckpt_capacity) // 8
        ckpt_n = n
    else:
        words, ckpt_n = 1, 1
    outputs = (((n, n_hist, problem.n_system), np.float64), ((4, n), np.int32),
               ((WORKSPACE_BYTES,), np.uint8), ((max(1, words),), np.float64), ((ckpt_n,), np.int32))
    attrs = dict(plan=np.int64(plan_address(problem)), mode=np.int32(mode), dt0=np.float64(dt0),
                 rtol=np.float64(rtol), atol=np.float64(atol), max_steps=np.int32(max_steps),
                 ckpt_capacity=np.int64(ckpt_capacity))
    return outputs, attrs


def _ffi_solve(problem, y0, times, params, *, dt0, rtol, atol, max_steps, ckpt_capacity=0):
    jax = _jax()
    jnp = jax.numpy
    register_targets()
    outputs, attrs = solve_call_args(problem, y0.shape[0], times.shape[0], mode=_native.MDX_LAUNCH_PERSISTENT,
                                     dt0=dt0, rtol=rtol, atol=atol, max_steps=max_steps,
                                     ckpt_capacity=ckpt_capacity)
    specs = tuple(jax.ShapeDtypeStruct(shape, dtype) for shape, dtype in outputs)
    call = jax.ffi.ffi_call(SOLVE_TARGET, specs, has_side_effect=False)
    hist, counters, _workspace, ckpt, ckpt_count = call(
        y0, times, params, jnp.zeros((0,), jnp.float64), **attrs)
    return hist, counters, ckpt, ckpt_count


def _ffi_grad(problem, times, params, ckpt, ckpt_count, grad_hist, ckpt_capacity):
    jax = _jax()
    jnp = jax.numpy
    register_targets()
    n = ckpt_count.shape[0]
    specs = (jax.ShapeDtypeStruct((n, problem.n_vars), jnp.float64),
             jax.ShapeDtypeStruct((n, problem.n_params), jnp.float64),
             jax.ShapeDtypeStruct((n,), jnp.int32))
    # Longest reverse sweeps first, as the torch front end orders them.
    order = jnp.argsort(-ckpt_count).astype(jnp.int32)
    call = jax.ffi.ffi_call(GRAD_TARGET, specs, has_side_effect=False)
    return call(times, params, ckpt, ckpt_count, grad_hist, order, plan=np.int64(plan_address(problem)),
                ckpt_capacity=np.int64(ckpt_capacity))


# --------------------------------------------------------------------------- rules (no JAX needed)
def broadcast_for_vmap(xp, arg, is_batched: bool, axis_size: int, name: str):
    """One vmapped argument as a ``(axis_size, width)`` ensemble array (``modax/_jax_common.py:50-67``)."""
    arr = xp.asarray(arg)
    if is_batched:
        if arr.ndim != 2:
            raise NotImplementedError(
                f"vmap over an already-ensembled {name} is not supported; "
                "call the solver with batched y0/params directly instead.")
        if arr.shape[0] != axis_size:
            raise ValueError(f"batched {name} has leading axis {arr.shape[0]}, expected {axis_size}")
        return arr
    if arr.ndim != 1:
        raise NotImplementedError(
            f"vmap with unbatched ensemble-shaped {name} is not supported; "
            "call the solver with batched y0/params directly instead.")
    return xp.broadcast_to(arr, (axis_size,) + arr.shape)


def vmap_rule(xp, ensemble, axis_size, in_batched, y0, t_span, params):
    """``vmap`` of a single-trajectory solve as one ensemble call (``modax/_jax_common.py:81-111``).

    ``ensemble(y0 (N, n), t_span, params (N, P)) -> (hist (N, S, n), counters (4, N))``.
    Returns the batched outputs -- ``hist`` as ``(axis, 1, S, n)``, the single
    solve's ``(1, S, n)`` per element -- and their batched flags."""
    y0_batched, t_batched, p_batched = in_batched
    if t_batched:
        t = xp.asarray(t_span)
        if t.ndim != 2:
            raise NotImplementedError(
                "vmap over nested t_span values is not supported; use a shared "
                "t_span and vmap over y0 and/or params, or call the solver directly.")
        t_span = t[0]
    y0_arr = broadcast_for_vmap(xp, y0, y0_batched, axis_size, "y0")
    p_arr = broadcast_for_vmap(xp, params, p_batched, axis_size, "params")
    hist, counters = ensemble(y0_arr, t_span, p_arr)
    return (hist[:, None], xp.transpose(counters)[:, :, None]), (True, True)


def sensitivity_blocks(y0_tangent_is_zero: bool, params_tangent_is_zero: bool):
    """``(wrt_y0, wrt_params)``: the blocks a JVP carries (``modax/_sensitivity.py:372-377``)."""
    return not y0_tangent_is_zero, not params_tangent_is_zero


def contract_tangent(xp, sens, n_vars, dy0, dparams, param_columns):
    """``S . (dy0, dparams)`` (``modax/_sensitivity.py:388-408``); ``sens`` is
    ``(N, S, n_vars, n_sens)``, y0 directions first, ``None`` marks a zero tangent."""
    n = sens.shape[0]
    tangent = xp.zeros(sens.shape[:3], dtype=sens.dtype)
    offset = 0
    if dy0 is not None:
        d = xp.broadcast_to(xp.asarray(dy0), (n, n_vars))
        tangent = tangent + xp.einsum("nsij,nj->nsi", sens[..., :n_vars], d)
        offset = n_vars
    if dparams is not None:
        d = xp.asarray(dparams)
        d = xp.broadcast_to(d, (n,) + d.shape[-1:])
        if param_columns is not None:
            d = d[:, xp.asarray(param_columns)]
        tangent = tangent + xp.einsum("nsik,nk->nsi", sens[..., offset:], d)
    return tangent


def mask_adjoint(xp, grad_y0, grad_params, status, param_columns):
    """The reverse kernel's cotangents with overflowed trajectories set to NaN and
    the undifferentiated parameter columns to zero."""
    bad = (status & _native.MDX_STATUS_CKPT_OVERFLOW) != 0
    grad_y0 = xp.where(bad[:, None], xp.nan, grad_y0)
    grad_params = xp.where(bad[:, None], xp.nan, grad_params)
    if param_columns is not None:
        keep = np.zeros(grad_params.shape[1], dtype=bool)
        keep[list(param_columns)] = True
        grad_params = xp.where(xp.asarray(keep)[None, :], grad_params, 0.0)
    return grad_y0, grad_params


# --------------------------------------------------------------------------- public solvers
def _normalize(jnp, y0, params):
    y0 = jnp.asarray(y0, dtype=jnp.float64)
    params = jnp.asarray(params, dtype=jnp.float64)
    if y0.ndim not in (1, 2) or params.ndim not in (1, 2):
        raise ValueError(
            "y0 must have shape (n_vars,) or (N, n_vars) and params shape "
            f"(n_params,) or (N, n_params); got y0.shape={y0.shape} and params.shape={params.shape}")
    if y0.ndim == 2 and params.ndim == 2 and params.shape[0] != y0.shape[0]:
        raise ValueError(
            "params must have shape (n_params,) or (N, n_params) when y0 has "
            f"shape (N, n_vars); got y0.shape={y0.shape} and params.shape={params.shape}")
    n = y0.shape[0] if y0.ndim == 2 else (params.shape[0] if params.ndim == 2 else 1)
    y0 = jnp.broadcast_to(y0, (n, y0.shape[-1]))
    params = jnp.broadcast_to(params, (n, params.shape[-1]))
    return y0, params


class _Solver:
    """One solver configuration: the compiled problems and the JAX-wrapped call."""

    def __init__(self, ode_fn, n_vars, n_params, options, *, rtol, atol, first_step, max_steps,
                 sens_error_control, sens_param_columns, adjoint_capacity):
        self.args = (ode_fn, n_vars, n_params)
        self.options = options
        self.controls = dict(dt0=0.0 if first_step is None else float(first_step), rtol=float(rtol),
                             atol=float(atol), max_steps=int(max_steps))
        self.sens_error_control = bool(sens_error_control)
        self.param_columns = None if sens_param_columns is None else tuple(int(c) for c in sens_param_columns)
        self.adjoint_capacity = int(adjoint_capacity)

    def problem(self, **changes):
        return get_problem(*self.args, replace(self.options, **changes))

    # One launch per call; a vmap over the call folds into its ensemble axis.
    def _impl(self, y0, t_span, params, sens=None):
        jnp = _jax().numpy
        y0, params = _normalize(jnp, y0, params)
        if sens is not None:
            y0 = _augment(jnp, y0, self.args[1], sens)
        problem = self.problem(sens=sens) if sens is not None else self.problem()
        hist, counters, _, _ = _ffi_solve(problem, y0, jnp.asarray(t_span, jnp.float64), params, **self.controls)
        return hist, counters

    def vmapped(self, sens=None):
        jax = _jax()
        jnp = jax.numpy

        def impl(y0, t_span, params):
            return self._impl(y0, t_span, params, sens)

        call = jax.custom_batching.custom_vmap(impl)

        @call.def_vmap
        def _rule(axis_size, in_batched, y0, t_span, params):
            return vmap_rule(jnp, impl, axis_size, in_batched, y0, t_span, params)

        return call

    def build(self):
        jax = _jax()
        jnp = jax.numpy
        n_vars, n_params = self.args[1], self.args[2]
        primal = self.vmapped()

        if self.sens_error_control:
            fn = jax.custom_jvp(primal)

            def _jvp(primals, tangents):
                y0, t_span, params = primals
                dy0, dt, dparams = tangents
                if not _is_zero(jax, dt):
                    raise NotImplementedError(
                        "differentiating a solve with respect to t_span is not supported; wrap the save "
                        "times in jax.lax.stop_gradient, or differentiate with respect to y0 and/or params only")
                wrt_y0, wrt_p = sensitivity_blocks(_is_zero(jax, dy0), _is_zero(jax, dparams))
                if not (wrt_y0 or wrt_p):
                    hist, counters = primal(y0, t_span, params)
                    return (hist, counters), (jnp.zeros_like(hist), _float0_like(jax, counters))
                cols = self.param_columns if self.param_columns is not None else tuple(range(n_params))
                sens = (n_vars if wrt_y0 else 0, cols if wrt_p else (), True)
                hist, counters = self.vmapped(sens)(y0, t_span, params)
                n, s = hist.shape[0], hist.shape[1]
                state = hist[:, :, :n_vars]
                n_sens = sens[0] + len(sens[1])
                sm = jnp.swapaxes(hist[:, :, n_vars:].reshape(n, s, n_sens, n_vars), 2, 3)
                tangent = contract_tangent(jnp, sm, n_vars, dy0 if wrt_y0 else None,
                                           dparams if wrt_p else None,
                                           self.param_columns if wrt_p else None)
                return (state, counters), (tangent, _float0_like(jax, counters))

            fn.defjvp(_jvp, symbolic_zeros=True)
            return fn

        fn = jax.custom_vjp(primal)
        capacity = self.adjoint_capacity
        problem = self.problem(checkpoint=True, adjoint=True, ckpt_stride=ADJOINT_STRIDE)

        def record(y0, t_span, params):
            y0n, pn = _normalize(jnp, y0, params)
            times = jnp.asarray(t_span, jnp.float64)
            hist, counters, ckpt, count = _ffi_solve(problem, y0n, times, params=pn, ckpt_capacity=capacity,
                                                     **self.controls)
            return hist, counters, ckpt, count, pn

        def fwd(y0, t_span, params):
            hist, counters, ckpt, count, pn = record(y0, t_span, params)
            return (hist, counters), (jnp.asarray(t_span, jnp.float64), pn, ckpt, count, jnp.shape(y0),
                                      jnp.shape(params))

        def bwd(res, cotangents):
            times, pn, ckpt, count, y0_shape, p_shape = res
            gy0, gp, status = _ffi_grad(problem, times, pn, ckpt, count, cotangents[0], capacity)
            gy0, gp = mask_adjoint(jnp, gy0, gp, status, self.param_columns)
            # Inputs broadcast over the ensemble get the sum of their rows' cotangents.
            gy0 = gy0 if len(y0_shape) == 2 else gy0.sum(axis=0)
            gp = gp if len(p_shape) == 2 else gp.sum(axis=0)
            return gy0, None, gp

        fn.defvjp(fwd, bwd)
        return fn


def _is_zero(jax, tangent) -> bool:
    zero_types = tuple(t for t in (getattr(getattr(jax, "custom_derivatives", None), "SymbolicZero", None),)
                       if t is not None)
    return tangent is None or (bool(zero_types) and isinstance(tangent, zero_types))


def _float0_like(jax, x):
    return np.zeros(np.shape(x), dtype=jax.dtypes.float0)


def _augment(jnp, y0, n_vars, sens):
    """``[y0, S(t0)]``: identity for the y0 block, zeros for parameter columns (``modax/_sensitivity.py:25-37``)."""
    n = y0.shape[0]
    blocks = [y0]
    if sens[0]:
        blocks.append(jnp.broadcast_to(jnp.eye(n_vars).reshape(1, -1), (n, n_vars * n_vars)))
    if sens[1]:
        blocks.append(jnp.zeros((n, n_vars * len(sens[1]))))
    return jnp.concatenate(blocks, axis=1)


def _solve(solver_name, ode_fn, y0, t_span, params, *, rtol, atol, first_step, max_steps, return_stats,
           error_weights, options, sens_error_control, sens_param_columns, adjoint_capacity):
    jax = _jax()
    jnp = jax.numpy
    if error_weights is not None:
        raise NotImplementedError("error_weights are not supported by the JAX front end; use the torch one")
    n_vars, n_params = int(np.shape(y0)[-1]), int(np.shape(params)[-1])
    solver = _Solver(ode_fn, n_vars, n_params, options, rtol=rtol, atol=atol,
                     first_step=first_step, max_steps=max_steps, sens_error_control=sens_error_control,
                     sens_param_columns=sens_param_columns, adjoint_capacity=adjoint_capacity)
    hist, counters = solver.build()(jnp.asarray(y0, jnp.float64), jnp.asarray(t_span, jnp.float64),
                                    jnp.asarray(params, jnp.float64))
    if not return_stats:
        return hist
    return hist, {"accepted_steps": counters[0], "rejected_steps": counters[1], "loop_steps": counters[2]}


def rodas5P_solve(ode_fn, y0, t_span, params, *, rtol=1e-8, atol=1e-10, first_step=None, max_steps=100000,
                  return_stats=False, error_weights=None, pcoeff=0.0, icoeff=1.0, dcoeff=0.0,
                  lu_precision="fp32", sparsity=None, ordering="amd", sens_error_control=True,
                  sens_param_columns=None, adjoint_capacity=4096):
    """``modax.rodas5P.solve`` under JAX (``modax/rodas5P.py:1024-1051``)."""
    from menodax_b200._sparsity import normalize_sparsity

    n_vars = int(np.shape(y0)[-1])
    options = KernelOptions(solver="rodas5P", pcoeff=float(pcoeff), icoeff=float(icoeff), dcoeff=float(dcoeff),
                            lu_precision=lu_precision, fast=lu_precision == "fp32",
                            sparsity=None if sparsity is None else normalize_sparsity(sparsity, n_vars),
                            ordering=ordering)
    return _solve("rodas5P", ode_fn, y0, t_span, params, rtol=rtol, atol=atol, first_step=first_step,
                  max_steps=max_steps, return_stats=return_stats, error_weights=error_weights, options=options,
                  sens_error_control=sens_error_control, sens_param_columns=sens_param_columns,
                  adjoint_capacity=adjoint_capacity)


def tsit5_solve(ode_fn, y0, t_span, params, *, rtol=1e-8, atol=1e-10, first_step=None, max_steps=100000,
                return_stats=False, error_weights=None, pcoeff=0.0, icoeff=1.0, dcoeff=0.0, backend="auto",
                sens_error_control=True, sens_param_columns=None, adjoint_capacity=4096):
    """``modax.tsit5.solve`` under JAX (``modax/tsit5.py:623-641``)."""
    if backend not in ("auto", "local", "shared"):
        raise ValueError(f"backend must be 'auto', 'shared', or 'local'; got {backend!r}")
    options = KernelOptions(solver="tsit5", pcoeff=float(pcoeff), icoeff=float(icoeff), dcoeff=float(dcoeff),
                            shared_stages=backend == "shared")
    return _solve("tsit5", ode_fn, y0, t_span, params, rtol=rtol, atol=atol, first_step=first_step,
                  max_steps=max_steps, return_stats=return_stats, error_weights=error_weights, options=options,
                  sens_error_control=sens_error_control, sens_param_columns=sens_param_columns,
                  adjoint_capacity=adjoint_capacity)
