"""CUDA-graph-captured ensemble solves.

A solve called over and over on same-shaped ensembles (a parameter sweep, an
optimisation loop) pays a host launch path per call: argument packing, the
work-queue memset of the persistent kernel, the launch itself.  ``GraphedSolve``
captures that once -- the memset and the kernel on one stream, into a CUDA graph
over static device buffers -- and each call copies the new inputs into the static
buffers and replays the graph.  The launch shape is the autotuned one.
"""

from __future__ import annotations


import numpy as np
import torch

from menodax_b200 import _native, autotune
from menodax_b200._ensemble import initial_step, launch
from menodax_b200._problem import KernelOptions, get_problem


class GraphedSolve:
    """A captured Rodas5P or Tsit5 ensemble solve of fixed size.

    ``solver`` is ``"rodas5P"`` or ``"tsit5"``; ``n_traj`` trajectories of
    ``n_vars`` states and ``n_params`` parameters, saved at ``t_span``.  Calling
    it with ``(y0, params)`` (device or host arrays of shape ``(n_traj, ...)``)
    returns ``(hist, counters)``, views of the graph's static output buffers that
    the next call overwrites (``counters`` rows: accepted, rejected, attempted,
    status).
    """

    def __init__(self, solver, ode_fn, n_traj, n_vars, n_params, t_span, *, rtol=1e-8, atol=1e-10,
                 first_step=None, max_steps=100000, lu_precision="fp32", arithmetic="auto",
                 sparsity=None, ordering="amd", launch_mode="auto", device=None):
        if solver not in ("tsit5", "rodas5P"):
            raise ValueError(f"solver must be 'tsit5' or 'rodas5P'; got {solver!r}")
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        fast = arithmetic == "fast" or (arithmetic == "auto" and lu_precision == "fp32")
        sparse = None
        if sparsity is not None:
            from menodax_b200._sparsity import normalize_sparsity

            sparse = normalize_sparsity(sparsity, n_vars)
        options = KernelOptions(solver=solver, lu_precision=lu_precision, fast=fast and solver == "rodas5P",
                                sparsity=sparse, ordering=ordering)
        self.y0 = torch.zeros((n_traj, n_vars), dtype=torch.float64, device=dev)
        self.params = torch.zeros((n_traj, n_params), dtype=torch.float64, device=dev)
        self.times = torch.as_tensor(np.asarray(t_span, dtype=np.float64), device=dev).contiguous()
        self.hist = torch.empty((n_traj, self.times.numel(), n_vars), dtype=torch.float64, device=dev)
        self.counters = torch.empty((4, n_traj), dtype=torch.int32, device=dev)
        common = dict(y0=self.y0, times=self.times, params=self.params, weights=None,
                      dt0=initial_step(first_step), rtol=rtol, atol=atol, max_steps=max_steps)
        self._common = common
        self._ode_fn = ode_fn
        self._sizes = (n_vars, n_params)
        self._options = options
        self._launch_mode = launch_mode
        self._graph = None
        self._order = None
        self._stream = torch.cuda.Stream(device=dev)

    def _capture(self):
        n_vars, n_params = self._sizes
        opts = self._options
        n = self.y0.shape[0]
        if self._launch_mode == "auto" and n >= 4096:
            choice = autotune.tune(self._ode_fn, n_vars, n_params, opts, **self._common)
        else:
            mode = _native.MDX_LAUNCH_PERSISTENT if self._launch_mode == "persistent" else _native.MDX_LAUNCH_PLAIN
            choice = autotune.LaunchChoice(opts.threads_per_block, mode, 1.0, opts.team, opts.shared_stages)
        problem = get_problem(self._ode_fn, n_vars, n_params, autotune.options_for(opts, choice))
        grid = autotune.grid_blocks(problem, choice, n)
        kw = dict(mode=choice.mode, grid_blocks=grid, out=(self.hist, self.counters), **self._common)
        self.launch_choice = choice
        with torch.cuda.stream(self._stream):
            launch(problem, **kw)  # loads the module and sizes the workspace before capture
            self._stream.synchronize()
            if choice.mode == _native.MDX_LAUNCH_PERSISTENT:
                # The captured persistent launch visits the trajectories longest
                # first by this first solve's step counts (any order gives the
                # same results; similar lengths in a warp finish together).
                self._order = autotune.longest_first(self.counters[2])
                kw["order"] = self._order
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=self._stream):
                launch(problem, **kw)
        self._graph = graph

    def __call__(self, y0, params):
        self.y0.copy_(torch.as_tensor(y0, dtype=torch.float64))
        self.params.copy_(torch.as_tensor(params, dtype=torch.float64))
        if self._graph is None:
            self._capture()
        self._graph.replay()
        return self.hist, self.counters
