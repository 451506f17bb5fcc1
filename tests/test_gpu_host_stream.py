"""The history written to pinned host memory by the solve kernel itself.

Host results (NumPy or CPU-tensor inputs) of a one-launch solve come back
through ``mdx_solve_desc.hist_host``: each warp, or each team, copies its
finished trajectories' rows across the host link while the rest of the ensemble
still steps (the persistent launch's results are copied after the kernel by the
Python front end, and its in-kernel copy is reached through the C ABI).  The
host copy must equal the device history bit for bit, for both launch shapes,
ragged ensembles (a partial last warp), the final-state-only history and the
team kernel; the runtime must refuse host memory the kernel cannot reach before
it launches anything.
"""

import ctypes

import numpy as np
import pytest
import torch

from menodax_b200 import _native, rodas5P, tsit5
from menodax_b200._ensemble import launch
from menodax_b200._problem import KernelOptions, get_problem
from menodax_b200._sparsity import normalize_sparsity
from workloads import systems

pytestmark = pytest.mark.gpu


def _both(solver, fn, y0, t_span, params, **kw):
    host = solver.solve(fn, y0, t_span, params, **kw)
    dev = torch.device("cuda", 0)
    on_dev = solver.solve(fn, torch.as_tensor(y0, device=dev), torch.as_tensor(t_span, device=dev),
                          torch.as_tensor(params, device=dev), **kw)
    return host, on_dev


def _assert_same(host, on_dev):
    if isinstance(host, tuple):
        for h, d in zip(host, on_dev):
            _assert_same(h, d)
        return
    if isinstance(host, dict):
        return
    np.testing.assert_array_equal(np.asarray(host), on_dev.cpu().numpy())


@pytest.mark.parametrize("launch_mode", ["plain", "persistent"])
@pytest.mark.parametrize("size", [1000, 8192])
def test_robertson_host_history_equals_device_history(launch_mode, size):
    cfg = systems.robertson_config(size=size)
    host, on_dev = _both(rodas5P, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                         atol=cfg["atol"], lu_precision="fp32", launch=launch_mode)
    assert isinstance(host, np.ndarray) and host.shape == (size, len(cfg["t_span"]), 3)
    _assert_same(host, on_dev)


@pytest.mark.parametrize("launch_mode", ["plain", "persistent"])
def test_tsit5_host_copy(launch_mode):
    cfg = systems.lorenz_config(size=777)
    host, on_dev = _both(tsit5, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                         atol=cfg["atol"], launch=launch_mode)
    _assert_same(host, on_dev)


@pytest.mark.parametrize("max_steps", [100000, 40])
def test_chunked_host_copy_many_saves(max_steps):
    """200 save times (a 4,800-byte row per trajectory) and a ragged last warp;
    with a step cap, capped trajectories' later rows hold the frozen state
    written when they stop."""
    cfg = systems.robertson_config(size=1000)
    t_span = np.concatenate([[0.0], np.logspace(-5, 5, 199)])
    host, on_dev = _both(rodas5P, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], rtol=cfg["rtol"],
                         atol=cfg["atol"], lu_precision="fp32", launch="plain", max_steps=max_steps)
    assert host.shape == (1000, 200, 3)
    _assert_same(host, on_dev)


def _sum_first_component(save_idx, y, t, p, acc):
    acc[0] += y[0]


@pytest.mark.parametrize("launch_mode", ["plain", "persistent"])
def test_final_state_only_host_copy(launch_mode):
    cfg = systems.robertson_config(size=777)
    host, on_dev = _both(rodas5P, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                         atol=cfg["atol"], save_history=False, save_hook=_sum_first_component, hook_size=1,
                         launch=launch_mode)
    assert host[0].shape == (777, 1, 3) and host[1].shape == (777, 1)
    _assert_same(host, on_dev)



def test_autotuned_launch_host_copy():
    cfg = systems.robertson_config(size=65536)
    host, on_dev = _both(rodas5P, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                         atol=cfg["atol"], lu_precision="fp32")
    _assert_same(host, on_dev)


@pytest.mark.parametrize("team", [4, 8])
@pytest.mark.parametrize("launch_mode", ["plain", "persistent"])
def test_team_host_copy(team, launch_mode):
    cfg = systems.vdp_ring_config(4, size=300)
    t_span = np.linspace(0.0, 30.0, 20)
    host, on_dev = _both(rodas5P, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], rtol=1e-6, atol=1e-8,
                         sparsity=cfg["sparsity"], team=team, launch=launch_mode)
    _assert_same(host, on_dev)


def test_host_copy_with_stats_and_cpu_tensors():
    cfg = systems.robertson_config(size=512)
    y0 = torch.as_tensor(cfg["y0"])
    p = torch.as_tensor(cfg["params"])
    hist, stats = rodas5P.solve(cfg["ode_fn"], y0, cfg["t_span"], p, rtol=cfg["rtol"], atol=cfg["atol"],
                                return_stats=True)
    assert isinstance(hist, torch.Tensor) and hist.device.type == "cpu"
    ref, ref_stats = rodas5P.solve(cfg["ode_fn"], y0.cuda(), cfg["t_span"], p.cuda(), rtol=cfg["rtol"],
                                   atol=cfg["atol"], return_stats=True)
    assert torch.equal(hist, ref.cpu())
    assert torch.equal(torch.as_tensor(stats["accepted_steps"]), ref_stats["accepted_steps"].cpu())


@pytest.mark.parametrize("team", [0, 4])
def test_persistent_kernels_copy_rows_through_the_abi(team):
    cfg = systems.vdp_ring_config(4, size=777)
    dev = torch.device("cuda", 0)
    t_span = np.linspace(0.0, 30.0, 20)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=normalize_sparsity(cfg["sparsity"], 8),
                         team=team, threads_per_block=64)
    problem = get_problem(cfg["ode_fn"], 8, 1, opts)
    kw = dict(y0=torch.as_tensor(cfg["y0"], device=dev), times=torch.as_tensor(t_span, device=dev),
              params=torch.as_tensor(cfg["params"], device=dev), weights=None, dt0=0.0, rtol=1e-6, atol=1e-8,
              max_steps=100000, mode=_native.MDX_LAUNCH_PERSISTENT)
    host = torch.zeros((777, len(t_span), 8), dtype=torch.float64, pin_memory=True)
    hist, _ = launch(problem, hist_host=host, **kw)
    torch.cuda.synchronize()
    assert torch.equal(host, hist.cpu())


def _robertson_launch_args(n):
    cfg = systems.robertson_config(size=n)
    dev = torch.device("cuda", 0)
    return dict(y0=torch.as_tensor(cfg["y0"], device=dev), times=torch.as_tensor(cfg["t_span"], device=dev),
                params=torch.as_tensor(cfg["params"], device=dev), weights=None, dt0=0.0, rtol=cfg["rtol"],
                atol=cfg["atol"], max_steps=100000, mode=_native.MDX_LAUNCH_PLAIN)


def _desc(args, n, hist, counters, host_ptr):
    s = args["times"].shape[0]
    desc = _native.SolveDesc()
    desc.mode = _native.MDX_LAUNCH_PLAIN
    desc.n_traj, desc.n_save, desc.n_save_hist, desc.max_steps = n, s, s, 100000
    desc.rtol, desc.atol = args["rtol"], args["atol"]
    desc.y0, desc.times, desc.params = args["y0"].data_ptr(), args["times"].data_ptr(), args["params"].data_ptr()
    desc.hist = hist.data_ptr()
    desc.accepted, desc.rejected = counters[0].data_ptr(), counters[1].data_ptr()
    desc.loop_steps, desc.status = counters[2].data_ptr(), counters[3].data_ptr()
    desc.hist_host = ctypes.c_void_p(host_ptr)
    return desc


def test_registered_host_memory_and_refusals():
    """Host memory registered with cudaHostRegister receives the history through
    its device mapping; a pageable buffer, and a registered one too small for
    the history, are refused by the runtime before anything is launched."""
    n = 256
    problem = get_problem(systems.robertson, 3, 3, KernelOptions())
    args = _robertson_launch_args(n)
    s = args["times"].shape[0]
    hist = torch.empty((n, s, 3), dtype=torch.float64, device="cuda")
    counters = torch.empty((4, n), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    cudart = torch.cuda.cudart()
    full = np.zeros((n, s, 3))
    short = np.zeros((n // 2, s, 3))
    assert int(cudart.cudaHostRegister(full.ctypes.data, full.nbytes, 0)) == 0
    assert int(cudart.cudaHostRegister(short.ctypes.data, short.nbytes, 0)) == 0
    try:
        problem.plan.solve(_desc(args, n, hist, counters, full.ctypes.data), stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(full, hist.cpu().numpy())
        pageable = np.zeros((n, s, 3))
        for host_ptr in (pageable.ctypes.data, short.ctypes.data):
            with pytest.raises(_native.NativeError, match="hist_host"):
                problem.plan.solve(_desc(args, n, hist, counters, host_ptr), stream)
        torch.cuda.synchronize()
    finally:
        cudart.cudaHostUnregister(full.ctypes.data)
        cudart.cudaHostUnregister(short.ctypes.data)
    # The Python launcher checks the tensor before the runtime sees it.
    with pytest.raises(ValueError, match="hist_host"):
        launch(problem, hist_host=torch.empty((n, s, 3), dtype=torch.float64), **args)
