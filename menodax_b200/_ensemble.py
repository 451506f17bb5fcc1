"""Shared host logic of the ensemble solvers: argument normalisation and the launch.

Mirrors ``modax/_jax_common.py:12-46`` (``normalize_y0_params``) and
``modax/_numba_common.py:55-138`` (error weights, ``dt0`` sentinel, the FFI
call and the stats dict), with torch providing device memory and the stream.
"""

from __future__ import annotations

import numpy as np
import torch

from menodax_b200 import _native

_DEVICE_ERR = (
    "menodax_b200 solves run on a CUDA device and have no CPU implementation; "
    "torch.cuda.is_available() is False"
)


def _as_tensor(x, name):
    if isinstance(x, torch.Tensor):
        return x.to(torch.float64)
    try:
        arr = np.asarray(x, dtype=np.float64)
    except (TypeError, ValueError) as exc:
        raise ValueError(f"{name} must be a numeric array") from exc
    return torch.from_numpy(np.ascontiguousarray(arr))


def normalize_y0_params(y0, params):
    """Broadcast ``y0``/``params`` to ``(N, n_vars)``/``(N, n_params)`` (``modax/_jax_common.py:12-46``)."""
    y0_t = _as_tensor(y0, "y0")
    p_t = _as_tensor(params, "params")
    if y0_t.ndim not in (1, 2) or p_t.ndim not in (1, 2):
        raise ValueError(
            "y0 must have shape (n_vars,) or (N, n_vars) and params shape "
            f"(n_params,) or (N, n_params); got y0.shape={tuple(y0_t.shape)} and "
            f"params.shape={tuple(p_t.shape)}"
        )
    if y0_t.ndim == 2:
        n = y0_t.shape[0]
        if p_t.ndim == 2 and p_t.shape[0] != n:
            raise ValueError(
                "params must have shape (n_params,) or (N, n_params) when y0 has "
                f"shape (N, n_vars); got y0.shape={tuple(y0_t.shape)} and "
                f"params.shape={tuple(p_t.shape)}"
            )
    elif p_t.ndim == 2:
        n = p_t.shape[0]
    else:
        n = 1
    if y0_t.ndim == 1:
        y0_t = y0_t.unsqueeze(0).expand(n, y0_t.shape[0])
    if p_t.ndim == 1:
        p_t = p_t.unsqueeze(0).expand(n, p_t.shape[0])
    return y0_t, p_t, n, y0_t.shape[1]


def build_error_weights(error_weights, n: int, n_vars: int):
    """``None`` -> no weights array (the kernel multiplies by 1.0); else ``(n, n_vars)``."""
    if error_weights is None:
        return None
    w = _as_tensor(error_weights, "error_weights")
    if w.ndim == 1:
        if w.shape[0] != n_vars:
            raise ValueError(f"error_weights has {w.shape[0]} entries for {n_vars} components")
        w = w.unsqueeze(0).expand(n, n_vars)
    if tuple(w.shape) != (n, n_vars):
        raise ValueError(f"error_weights must be ({n_vars},) or ({n}, {n_vars}); got {tuple(w.shape)}")
    return w


def initial_step(first_step) -> float:
    """The kernels' ``dt0``: ``None`` becomes the non-positive sentinel (``modax/_numba_common.py:72-81``)."""
    return 0.0 if first_step is None else float(first_step)


def solver_stats(accepted, rejected, loop_steps, status=None):
    """The reference's stats dict (``modax/_numba_common.py:133-138``), plus the
    per-trajectory status bits when available (1: max_steps reached before the last
    save, 2: non-finite final state, 4: checkpoint capacity exceeded)."""
    stats = {"accepted_steps": accepted, "rejected_steps": rejected, "loop_steps": loop_steps}
    if status is not None:
        stats["status"] = status
    return stats


def pick_device(*tensors):
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return t.device
    if not torch.cuda.is_available():
        raise RuntimeError(_DEVICE_ERR)
    return torch.device("cuda", torch.cuda.current_device())


def to_device(t, device):
    if t is None:
        return None
    if t.device == device and t.is_contiguous():
        return t
    return t.to(device=device, non_blocking=t.is_pinned() if not t.is_cuda else False).contiguous()


class Workspace:
    """Scratch the persistent launch needs (the queue head), one per (device, stream).

    Launches on one stream are ordered, so they may share one; launches on two
    streams may overlap, so each stream gets its own."""

    _by_stream: dict = {}

    @classmethod
    def get(cls, device, stream: int, nbytes: int):
        key = (device, stream)
        buf = cls._by_stream.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
            cls._by_stream[key] = buf
        return buf


def launch(problem, *, y0, times, params, weights, dt0, rtol, atol, max_steps, mode,
           n_save_hist=None, grid_blocks=0, order=None, ckpt=None, ckpt_count=None,
           ckpt_capacity=0, out=None, hook_out=None, hist_host=None):
    """Allocate outputs on ``y0``'s device and launch one ensemble solve.

    All inputs must already be contiguous float64 CUDA tensors on one device.
    Returns ``(hist, counters)``; the rows of ``counters`` (4, N) int32 are the
    accepted, rejected and attempted step counts and the status bits.
    ``hist_host`` (a pinned CPU tensor shaped like ``hist``) receives the
    history from the kernel itself as trajectories finish; it is complete once
    the launching stream is.
    """
    n = y0.shape[0]
    n_save = times.shape[0]
    n_hist = n_save if n_save_hist is None else n_save_hist
    dev = y0.device
    if out is None:
        hist = torch.empty((n, n_hist, problem.n_system), dtype=torch.float64, device=dev)
        counters = torch.empty((4, n), dtype=torch.int32, device=dev)
    else:
        hist, counters = out
    desc = _native.SolveDesc()
    desc.mode = mode
    desc.n_traj = n
    desc.n_save = n_save
    desc.n_save_hist = n_hist
    desc.max_steps = int(max_steps)
    desc.dt0 = float(dt0)
    desc.rtol = float(rtol)
    desc.atol = float(atol)
    desc.y0 = y0.data_ptr()
    desc.times = times.data_ptr()
    desc.params = params.data_ptr() if params.numel() else None
    desc.weights = weights.data_ptr() if weights is not None else None
    desc.hist = hist.data_ptr()
    desc.accepted = counters[0].data_ptr()
    desc.rejected = counters[1].data_ptr()
    desc.loop_steps = counters[2].data_ptr()
    desc.status = counters[3].data_ptr()
    desc.order = order.data_ptr() if order is not None else None
    desc.hook_out = hook_out.data_ptr() if hook_out is not None else None
    if hist_host is not None and n > 0:
        if (hist_host.device.type != "cpu" or not hist_host.is_pinned() or hist_host.dtype != torch.float64
                or tuple(hist_host.shape) != tuple(hist.shape) or not hist_host.is_contiguous()):
            raise ValueError(f"hist_host must be a contiguous pinned float64 CPU tensor of shape {tuple(hist.shape)}")
        desc.hist_host = hist_host.data_ptr()
    stream = torch.cuda.current_stream(dev).cuda_stream
    if mode == _native.MDX_LAUNCH_PERSISTENT:
        nbytes = problem.plan.workspace_size(mode, n)
        ws = Workspace.get(dev, stream, nbytes)
        desc.workspace = ws.data_ptr()
        desc.workspace_bytes = ws.numel()
    desc.grid_blocks = int(grid_blocks)
    if ckpt is not None:
        desc.ckpt = ckpt.data_ptr()
        desc.ckpt_count = ckpt_count.data_ptr()
        desc.ckpt_capacity = int(ckpt_capacity)
    with torch.cuda.device(dev):
        problem.plan.solve(desc, stream)
    return hist, counters
