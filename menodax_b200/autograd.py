"""torch.autograd front end: gradients of an ensemble solve.

``rodas5P.solve`` / ``tsit5.solve`` route here when a torch input requires
grad.  ``sens_error_control`` picks the method, with the reference's meaning
(``modax/_sensitivity.py:64-135, 331-413``):

* ``True`` (the reference's default): forward sensitivities -- the joint
  ``[y, S]`` solve with the sensitivities under step-size control, the
  reference's own differentiation; ``backward`` contracts ``S`` with the
  incoming cotangent.  The primal output comes from that joint solve, as the
  reference's does under a JAX transform.
* ``False``: the discrete adjoint of the plain solve.  Its step sequence is the
  plain solve's, which is what the reference's forward sensitivities take with
  error control off, and the gradient equals theirs on that step sequence --
  computed backwards in one sweep whatever the number of parameters.

``sens_param_columns`` restricts the parameter columns that are differentiated;
the others receive a zero gradient (the transpose of the reference's gather).

The adjoint's forward pass runs the checkpointing kernel, which records every
accepted step's size and the start state ``(t, y)`` of every K-th step;
``backward`` launches the reverse kernel (``mdx_grad`` in the C ABI), which
replays each K-step segment from its start state, reverses it step by step and
returns the cotangents of ``y0`` and ``params``.  Step sizes are
constants of the discrete map, so the gradient is the exact derivative of the
solution the forward pass produced -- for that step sequence it equals what the
reference's forward sensitivities give with ``sens_error_control=False``
(``modax/_sensitivity.py:331-413``), computed backwards in one sweep whatever
the number of parameters.
"""

from __future__ import annotations

from dataclasses import replace

import torch

from menodax_b200 import _native, autotune
from menodax_b200._ensemble import initial_step, launch, pick_device, solver_stats
from menodax_b200._problem import get_problem

# Checkpoint capacity (accepted steps per trajectory) and stride last used per
# problem, so a repeated gradient call sizes its buffer without a counting pass.
_capacity_hint: dict = {}
# Per problem key: the trajectories of the last call, longest first (by accepted
# steps).  The checkpointing forward launch takes them in that order, so the
# long integrations start in the persistent grid's first wave; results do not
# depend on the order.
_order_hint: dict = {}
# The persistent grid fill of the checkpointing forward launch once it takes
# trajectories longest first.  Measured on the stiff Van der Pol gradient
# ensembles (65,536 trajectories, B200): the 2-state system wants a lightly
# loaded device (FP64 42 ms at half fill against 59-60 ms full,
# FP32 LUs 37-41 against 45-51 ms), the 16-state ring a full one (FP64 0.57 s
# full against 0.76 s at half fill, FP32 LUs 0.47 against 1.36 s): a small
# system's long integrations run fastest with few neighbours on their SM, a
# large one's spilled steps need the full grid's warps to hide their memory
# latency.
FORWARD_FILL_SMALL = 0.5
FORWARD_FILL_LARGE = 1.0
FORWARD_FILL_SMALL_VARS = 8
# Problems remembered by the hints above (oldest dropped first): the order hint
# holds a device tensor per problem.
HINT_PROBLEMS = 16


def _remember(hints: dict, key, value) -> None:
    hints.pop(key, None)
    hints[key] = value
    while len(hints) > HINT_PROBLEMS:
        hints.pop(next(iter(hints)))


# The checkpoint layout of the most recent gradient forward pass (for reports).
last_checkpoint: dict = {}

# Steps per recorded start state.  One record per step costs (n + 2) doubles a
# step; a stride K costs 1 + (n + 1) / K and one forward replay per step in the
# reverse pass.  The smallest stride whose buffer fits the memory budget wins.
CKPT_STRIDES = (1, 8, 32)
MEMORY_FRACTION = 0.6


def checkpoint_bytes(n_traj, n_vars, capacity, stride):
    segments = -(-capacity // stride)
    return 8 * (capacity * n_traj + segments * n_traj * (n_vars + 1))


def choose_stride(n_traj, n_vars, capacity, device):
    free, _ = torch.cuda.mem_get_info(device)
    # Memory torch's caching allocator holds for no live tensor -- the previous
    # call's checkpoint buffer, typically -- is free for this one too; leaving it
    # out would pick a coarser stride on every call after the first, and a
    # stride is a separately compiled kernel.
    free += torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    budget = MEMORY_FRACTION * free
    for stride in CKPT_STRIDES:
        if checkpoint_bytes(n_traj, n_vars, capacity, stride) <= budget:
            return stride
    need = checkpoint_bytes(n_traj, n_vars, capacity, CKPT_STRIDES[-1])
    raise MemoryError(
        f"the checkpoints of {n_traj} trajectories x {capacity} accepted steps need "
        f"{need / 2**30:.1f} GiB even at stride {CKPT_STRIDES[-1]}; solve fewer trajectories per call"
    )


def needs_grad(*xs) -> bool:
    return torch.is_grad_enabled() and any(isinstance(x, torch.Tensor) and x.requires_grad for x in xs)


def _as_double(x, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64)
    return torch.as_tensor(x, dtype=torch.float64, device=device)


def _longest_first(accepted):
    """Trajectory indices by descending step count, as the int32 visiting order
    the persistent launch takes."""
    return torch.argsort(accepted, descending=True, stable=True).to(torch.int32)


def _forward_blocks(problem, n: int, fill: float = 0.5) -> int:
    """Blocks of the forward passes' persistent launch: ``fill`` of the resident limit.

    Gradient ensembles are long stiff integrations with uneven step counts; the
    refill launch keeps lanes busy as trajectories finish, and at half the
    resident warps each runs with less contention (a 16-state ring's
    checkpointing forward in index order: 0.77 s against 1.21 s for the
    one-launch kernel; unchanged for 2 states)."""
    choice = autotune.LaunchChoice(problem.plan.tpb, _native.MDX_LAUNCH_PERSISTENT, fill, int(problem.options.team))
    return autotune.grid_blocks(problem, choice, n)


def _forward_fill(n_vars: int, ordered: bool) -> float:
    """The fill of a checkpointing forward launch: half in index order, else by
    the system's size once the long trajectories go first."""
    if not ordered or n_vars <= FORWARD_FILL_SMALL_VARS:
        return FORWARD_FILL_SMALL
    return FORWARD_FILL_LARGE


# Trajectories per reverse launch (None: the whole ensemble in one launch).  The
# reverse kernel of a larger system keeps its stages and their cotangents in
# local memory; launching the ensemble in slices, longest trajectories first,
# bounds how much of that is resident at once.
REVERSE_CHUNK: int | None = None


def reverse_chunk(problem, n: int) -> int:
    return max(1, min(n, REVERSE_CHUNK or n))


# The reverse sweep of a trajectory with more than REVERSE_SPLIT times the mean
# number of checkpoint segments is cut into chunks of at most that many, reversed
# in parallel and composed (None: never, the default).  A chunk costs n_vars + 1
# sweeps (its transfer matrix's columns and its offset), so splitting pays only
# when a few trajectories are far longer than the rest; on the stiff Van der Pol
# gradient ensembles the long trajectories are a sizeable fraction (at 2.5 x the
# mean, 5,141 of 65,536 2-state trajectories), and splitting them made the
# reverse pass slower.
REVERSE_SPLIT: float | None = None


def split_plan(counts, capacity: int, stride: int, n_vars: int, factor: float | None = None):
    """The split reverse's task table for trajectories with ``counts`` accepted
    steps (a CPU int tensor): ``(tasks, n_slots, combine)`` as int32 tensors
    (``mdx_grad_desc.tasks`` / ``combine``), longest tasks first, or ``None`` when
    no trajectory is long enough to split."""
    import numpy as np

    factor = REVERSE_SPLIT if factor is None else factor
    steps = np.minimum(counts.numpy().astype(np.int64), int(capacity))
    n = steps.shape[0]
    if factor is None or n == 0:
        return None
    n_seg = (steps + stride - 1) // stride
    limit = max(1, int(np.ceil(factor * float(n_seg.mean()))))
    long_traj = np.nonzero(n_seg > limit)[0]
    if long_traj.size == 0:
        return None
    short = np.nonzero(n_seg <= limit)[0]
    rows = [np.stack([n_seg[short], short, np.zeros_like(short), n_seg[short],
                      np.full_like(short, -2), np.full_like(short, -1)], axis=1)]
    combine = []
    slot = 0
    for traj in long_traj:
        total = int(n_seg[traj])
        chunks = -(-total // limit)
        combine.append((int(traj), slot, chunks))
        for c in range(chunks):
            lo, hi = c * total // chunks, (c + 1) * total // chunks
            for kind in range(-1, n_vars):
                rows.append(np.array([[hi - lo, traj, lo, hi, kind, slot]], dtype=np.int64))
                slot += 1
    table = np.concatenate(rows, axis=0)
    table = table[np.argsort(-table[:, 0], kind="stable")]
    tasks = torch.as_tensor(table[:, 1:].astype(np.int32))
    return tasks, slot, torch.as_tensor(np.asarray(combine, dtype=np.int32))


class _EnsembleSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y0, params, times, problems, dt0, rtol, atol, max_steps, key):
        n = y0.shape[0]
        y0c = y0.detach().contiguous()
        pc = params.detach().contiguous()
        kw = dict(y0=y0c, times=times, params=pc, weights=None, dt0=dt0, rtol=rtol, atol=atol,
                  max_steps=max_steps, mode=_native.MDX_LAUNCH_PERSISTENT)
        capacity, stride_hint = _capacity_hint.get(key, (None, None))
        order = _order_hint.get(key)
        if order is not None and (order.device != y0.device or order.numel() != n):
            order = None
        if capacity is None:
            # First call for this problem: count the accepted steps with a plain solve.
            _, counters = launch(problems["plain"], grid_blocks=_forward_blocks(problems["plain"], n), **kw)
            capacity = max(1, int(counters[0].max().item()) if n else 1)
            order = _longest_first(counters[0])
        while True:
            stride = choose_stride(n, problems["plain"].n_vars, capacity, y0.device)
            # Keep the last call's stride when memory still allows it: the same
            # compiled kernel and the same replay cost from call to call.
            if stride_hint is not None and stride < stride_hint:
                stride = stride_hint
            problem = problems[stride]
            nbytes = problem.plan.checkpoint_size(n, capacity)
            ckpt = torch.empty(max(1, nbytes // 8), dtype=torch.float64, device=y0.device)
            ckpt_count = torch.empty(n, dtype=torch.int32, device=y0.device)
            fill = _forward_fill(problems["plain"].n_vars, order is not None)
            hist, counters = launch(problem, ckpt=ckpt, ckpt_count=ckpt_count, ckpt_capacity=capacity,
                                    grid_blocks=_forward_blocks(problem, n, fill), order=order, **kw)
            needed = int(counters[0].max().item()) if n else 0
            if needed <= capacity:
                break
            capacity = int(needed * 1.1) + 8
            del ckpt
        _remember(_capacity_hint, key, (max(needed + 8, int(needed * 1.1)), stride))
        _remember(_order_hint, key, _longest_first(counters[0]))
        last_checkpoint.update(stride=stride, capacity=capacity, bytes=nbytes, forward_fill=fill)
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
        plan = None
        if not problem.options.team and REVERSE_CHUNK is None:
            plan = split_plan(ckpt_count.cpu(), ctx.capacity, int(problem.options.ckpt_stride), problem.n_vars)
        if plan is not None:
            tasks, n_slots, combine = plan
            tasks = tasks.to(params.device)
            combine = combine.to(params.device)
            task_out = torch.empty((max(1, n_slots), problem.n_vars + problem.n_params), dtype=torch.float64,
                                   device=params.device)
            d.tasks, d.n_tasks = tasks.data_ptr(), tasks.shape[0]
            d.task_out, d.n_slots = task_out.data_ptr(), n_slots
            d.combine, d.n_combine = combine.data_ptr(), combine.shape[0]
            last_checkpoint.update(split_tasks=int(tasks.shape[0]), split_trajectories=int(combine.shape[0]))
            with torch.cuda.device(params.device):
                problem.plan.grad(d, stream)
            return grad_y0, grad_p, None, None, None, None, None, None, None
        last_checkpoint.update(split_tasks=0, split_trajectories=0)
        # Longest reverse sweeps first: the reverse kernel's registers leave room
        # for only part of a large ensemble at once, and a long trajectory that
        # started in a later wave would set the makespan.
        order = torch.argsort(ckpt_count, descending=True, stable=True).to(torch.int32)
        chunk = reverse_chunk(problem, n)
        with torch.cuda.device(params.device):
            for first in range(0, n, chunk):
                d.order = order.data_ptr() + 4 * first
                d.count = min(chunk, n - first)
                problem.plan.grad(d, stream)
        return grad_y0, grad_p, None, None, None, None, None, None, None


class _ColumnMask(torch.autograd.Function):
    """Identity forward; backward zeroes the gradient of the undifferentiated columns."""

    @staticmethod
    def forward(ctx, params, keep):
        ctx.save_for_backward(keep)
        return params.clone()

    @staticmethod
    def backward(ctx, grad):
        (keep,) = ctx.saved_tensors
        return grad * keep, None


class _Problems:
    """The plain problem and its checkpointing/adjoint variants, compiled on demand."""

    def __init__(self, ode_fn, n_vars, n_params, options):
        self.args = (ode_fn, n_vars, n_params)
        self.options = options

    def __getitem__(self, which):
        opts = self.options if which == "plain" else replace(
            self.options, checkpoint=True, adjoint=True, ckpt_stride=int(which))
        if opts.team:
            # The reverse sweep's slices take a block's static shared memory.
            from menodax_b200._problem import team_grad_block_threads

            sized = opts if which != "plain" else replace(opts, ckpt_stride=CKPT_STRIDES[-1])
            opts = replace(opts, threads_per_block=team_grad_block_threads(
                self.args[1], self.args[2], replace(sized, checkpoint=True, adjoint=True)))
        return get_problem(*self.args, opts)


class _SensitivitySolve(torch.autograd.Function):
    """Forward sensitivities: the joint solve forward, ``S^T g`` backward."""

    @staticmethod
    def forward(ctx, y0, params, run):
        state, sens, counters = run(y0.detach(), params.detach())
        ctx.save_for_backward(sens)
        ctx.n_params = params.shape[1]
        ctx.wrt_y0 = run.wrt_y0
        ctx.columns = run.columns
        ctx.mark_non_differentiable(counters)
        return state, counters

    @staticmethod
    def backward(ctx, grad_state, _grad_counters):
        (sens,) = ctx.saved_tensors
        n, _, n_vars, _ = sens.shape
        grad_y0 = grad_p = None
        offset = 0
        g = grad_state if grad_state is not None else torch.zeros(sens.shape[:3], dtype=sens.dtype,
                                                                  device=sens.device)
        if ctx.wrt_y0:
            grad_y0 = torch.einsum("nsi,nsij->nj", g, sens[..., :n_vars])
            offset = n_vars
        if ctx.columns is not None:
            grad_p = torch.zeros((n, ctx.n_params), dtype=sens.dtype, device=sens.device)
            if ctx.columns:
                grad_p[:, list(ctx.columns)] = torch.einsum("nsi,nsik->nk", g, sens[..., offset:])
        return grad_y0, grad_p, None


class _JointRun:
    """One joint ``[y, S]`` solve for ``_SensitivitySolve``, fixed but for its inputs."""

    def __init__(self, solver, ode_fn, times, wrt_y0, columns, kw):
        self.solver, self.ode_fn, self.times, self.kw = solver, ode_fn, times, kw
        self.wrt_y0 = wrt_y0
        self.columns = columns  # None: no parameter block; else the differentiated columns

    def __call__(self, y0, params):
        from menodax_b200 import sensitivity

        state, sens, stats = sensitivity.solve(
            self.solver, self.ode_fn, y0, self.times, params, wrt_y0=self.wrt_y0,
            wrt_params=self.columns is not None and len(self.columns) > 0,
            sens_error_control=True, sens_param_columns=self.columns or None,
            return_stats=True, **self.kw)
        counters = torch.stack([stats["accepted_steps"], stats["rejected_steps"], stats["loop_steps"]])
        return state.contiguous(), sens.contiguous(), counters


def _forward_sensitivity_grad(options, ode_fn, y0_t, p_t, times, *, rtol, atol, first_step, max_steps,
                              return_stats, sens_param_columns):
    n_params = p_t.shape[1]
    columns = tuple(range(n_params)) if sens_param_columns is None else tuple(int(c) for c in sens_param_columns)
    if not p_t.requires_grad:
        columns = None
    wrt_y0 = bool(y0_t.requires_grad)
    if not wrt_y0 and columns is not None and not columns:
        columns = None
    if not wrt_y0 and columns is None:
        raise ValueError("sens_param_columns is empty and y0 does not require grad: nothing to differentiate")
    kw = dict(rtol=rtol, atol=atol, first_step=first_step, max_steps=max_steps, pcoeff=options.pcoeff,
              icoeff=options.icoeff, dcoeff=options.dcoeff)
    if options.solver == "rodas5P":
        kw.update(lu_precision=options.lu_precision, sparsity=options.sparsity, ordering=options.ordering)
    run = _JointRun(options.solver, ode_fn, times, wrt_y0, columns, kw)
    hist, counters = _SensitivitySolve.apply(y0_t, p_t, run)
    if return_stats:
        return hist, solver_stats(counters[0], counters[1], counters[2])
    return hist


def solve_with_grad(ode_fn, y0, t_span, params, options, *, rtol, atol, first_step, max_steps,
                    return_stats, error_weights, sens_error_control=False, sens_param_columns=None):
    """Differentiable ensemble solve; returns torch tensors on the solve's device.

    ``sens_error_control`` selects forward sensitivities (``True``) or the discrete
    adjoint (``False``); ``sens_param_columns`` the differentiated parameter columns."""
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
    if sens_param_columns is not None:
        cols = [int(c) for c in sens_param_columns]
        if len(set(cols)) != len(cols):
            raise ValueError("param_columns must not repeat a column")
        bad = [c for c in cols if not 0 <= c < n_params]
        if bad:
            raise ValueError(f"param_columns {bad} lie outside the {n_params} parameter columns")
    if sens_error_control:
        return _forward_sensitivity_grad(options, ode_fn, y0_t, p_t, times, rtol=rtol, atol=atol,
                                         first_step=first_step, max_steps=max_steps,
                                         return_stats=return_stats, sens_param_columns=sens_param_columns)
    if sens_param_columns is not None and p_t.requires_grad:
        keep = torch.zeros(n_params, dtype=torch.float64, device=device)
        keep[list(int(c) for c in sens_param_columns)] = 1.0
        p_t = _ColumnMask.apply(p_t, keep)
    problems = _Problems(ode_fn, n_vars, n_params, replace(options, runtime_weights=False))
    key = (ode_fn, n_vars, n_params, options, n, tuple(times.tolist()), float(rtol), float(atol))
    hist, counters = _EnsembleSolve.apply(y0_t, p_t, times, problems, initial_step(first_step), rtol,
                                          atol, max_steps, key)
    if return_stats:
        return hist, solver_stats(counters[0], counters[1], counters[2])
    return hist
