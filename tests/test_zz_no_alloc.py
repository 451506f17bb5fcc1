"""The no-allocation entry point, through the C ABI.

``mdx_solve_persistent_noalloc`` exists for callers that cannot allocate device
memory -- a plugin or custom-call handler that is handed only its input and
output buffers, or a host whose allocator must not be bypassed.  It runs the
persistent refill solve with its work-queue scratch taken from an array inside
the library instead of a caller workspace.  Its results must match the ordinary
persistent launch (``mdx_solve``) exactly, call after call, since both run the
same kernel on the same inputs.

This file is collected last, so a run that stops at the first failure has run
every other test before it; it also passes on its own in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

from menodax_b200 import _native
from workloads import systems
from menodax_b200._problem import KernelOptions, get_problem

pytestmark = pytest.mark.gpu


def _desc(y0, times, params, hist, counters, cfg, workspace=None):
    d = _native.SolveDesc()
    d.struct_size = ctypes.sizeof(_native.SolveDesc)
    d.mode = _native.MDX_LAUNCH_PERSISTENT
    d.n_traj = y0.shape[0]
    d.n_save = times.numel()
    d.n_save_hist = times.numel()
    d.max_steps = 100000
    d.dt0 = 0.0
    d.rtol = cfg["rtol"]
    d.atol = cfg["atol"]
    d.y0 = y0.data_ptr()
    d.times = times.data_ptr()
    d.params = params.data_ptr()
    d.hist = hist.data_ptr()
    d.accepted = counters[0].data_ptr()
    d.rejected = counters[1].data_ptr()
    d.loop_steps = counters[2].data_ptr()
    d.status = counters[3].data_ptr()
    if workspace is not None:
        d.workspace = workspace.data_ptr()
        d.workspace_bytes = workspace.numel()
    return d


def test_noalloc_matches_the_workspace_entry_point_on_repeated_calls():
    _native.build_library()
    lib = _native.lib()
    cfg = systems.robertson_config(size=3000)
    prob = get_problem(cfg["ode_fn"], 3, 3, KernelOptions(lu_precision="fp32"))
    dev = torch.device("cuda", 0)
    y0 = torch.as_tensor(cfg["y0"], device=dev).contiguous()
    params = torch.as_tensor(cfg["params"], device=dev).contiguous()
    times = torch.as_tensor(cfg["t_span"], device=dev).contiguous()
    stream = torch.cuda.current_stream(dev).cuda_stream

    hist_ref = torch.empty((y0.shape[0], times.numel(), 3), dtype=torch.float64, device=dev)
    cnt_ref = torch.empty((4, y0.shape[0]), dtype=torch.int32, device=dev)
    workspace = torch.empty(256, dtype=torch.uint8, device=dev)
    d = _desc(y0, times, params, hist_ref, cnt_ref, cfg, workspace)
    _native.check(lib.mdx_solve(prob.plan.handle, ctypes.byref(d), ctypes.c_void_p(stream)), "mdx_solve")
    torch.cuda.synchronize()

    for _ in range(2):
        hist = torch.full_like(hist_ref, float("nan"))
        cnt = torch.full_like(cnt_ref, -1)
        d = _desc(y0, times, params, hist, cnt, cfg)
        rc = lib.mdx_solve_persistent_noalloc(prob.plan.handle, ctypes.byref(d), ctypes.c_void_p(stream))
        _native.check(rc, "mdx_solve_persistent_noalloc")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(hist.cpu().numpy(), hist_ref.cpu().numpy())
        np.testing.assert_array_equal(cnt.cpu().numpy(), cnt_ref.cpu().numpy())


def test_noalloc_rejects_a_plain_launch_request():
    lib = _native.lib()
    cfg = systems.robertson_config(size=64)
    prob = get_problem(cfg["ode_fn"], 3, 3, KernelOptions(lu_precision="fp32"))
    d = _native.SolveDesc()
    d.struct_size = ctypes.sizeof(_native.SolveDesc)
    d.mode = _native.MDX_LAUNCH_PLAIN
    rc = lib.mdx_solve_persistent_noalloc(prob.plan.handle, ctypes.byref(d), None)
    assert rc == -1
    assert "MDX_LAUNCH_PERSISTENT" in _native.last_error()
