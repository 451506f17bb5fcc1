"""The solver kernels' step code, compiled for the host and run against the oracle.

`build_source` emits the whole problem source the GPU compiles: sizes, the
traced right-hand side and Jacobian writers, the LU routines and the solver's
init / running / step / finish.  Here that source, without its launch entry
(`mdx_entry.cuh`), is compiled with g++ under a prelude that maps the CUDA
spellings to host ones, and a loop of the plain kernel's shape (one trajectory
after another: init, step while running, finish) fills the same output buffers.
The result is held to the GPU parity bar against the oracle -- step counts
identical on at least 99% of trajectories, saved states within 1e-9 -- so the
kernel logic of the FP64 path is checked on every CPU run.  Both sides are
compiled with the same FMA contraction setting (measured: identical step counts
on every trajectory, states within 2.5e-10 for Rodas5P and 1.2e-13 for Tsit5;
not bitwise, as the two sources contract different expressions).
"""

import ctypes
import subprocess

import numpy as np
import pytest

from workloads import systems
from menodax_b200._native import KERNEL_DIR
from menodax_b200._problem import KernelOptions, build_source
from menodax_b200._sparse_direct import sparse_lu_for
from menodax_b200._sparsity import normalize_sparsity

PRELUDE = """
#include <cmath>
#include <cstring>
using std::fabs; using std::sqrt; using std::pow; using std::exp; using std::log; using std::sin;
using std::cos; using std::tanh; using std::atan2; using std::log1p; using std::expm1;
using std::isnan; using std::isfinite; using std::fma;
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __noinline__
#define __restrict__
#define __constant__
static inline float host_fdividef(float a, float b) { return a / b; }
static inline float host_powf(float a, float b) { return std::pow(a, b); }
#define __fdividef host_fdividef
#define __powf host_powf
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
template <class T> static inline T __ldcg(const T* p) { return *p; }
template <class T> static inline T __ldg(const T* p) { return *p; }
"""

DRIVER = """
extern "C" int run(MdxSolveArgs a) {
  for (int i = 0; i < a.n_traj; ++i) {
    MDX_HOST_THREAD(i);
    MDX_SOLVER::State st;
    MDX_SOLVER::init(st, a, i);
    while (MDX_SOLVER::running(st, a)) MDX_SOLVER::step(st, a);
    MDX_SOLVER::finish(st, a);
  }
  return 0;
}
"""


class Args(ctypes.Structure):
    """MdxSolveArgs (mdx_args.h), field for field."""

    _fields_ = [("y0", ctypes.c_void_p), ("times", ctypes.c_void_p), ("params", ctypes.c_void_p),
                ("weights", ctypes.c_void_p), ("hist", ctypes.c_void_p), ("accepted", ctypes.c_void_p),
                ("rejected", ctypes.c_void_p), ("loop_steps", ctypes.c_void_p), ("status", ctypes.c_void_p),
                ("hook_out", ctypes.c_void_p), ("work_counter", ctypes.c_void_p), ("order", ctypes.c_void_p),
                ("ckpt", ctypes.c_void_p), ("ckpt_count", ctypes.c_void_p), ("ckpt_capacity", ctypes.c_longlong),
                ("hist_host", ctypes.c_void_p), ("n_traj", ctypes.c_int), ("n_save", ctypes.c_int),
                ("n_save_hist", ctypes.c_int), ("max_steps", ctypes.c_int), ("dt0", ctypes.c_double), ("rtol", ctypes.c_double),
                ("atol", ctypes.c_double)]


# Thread-kernel builds run trajectory i as thread i % MDX_TPB of its block, for
# code that keeps a per-thread column of a block's shared array.
THREAD_DIMS = """
struct HostDim { unsigned x, y, z; };
static HostDim threadIdx, blockIdx, blockDim;
#define __shared__ static
#define MDX_HOST_THREAD(i) (threadIdx.x = (unsigned)((i) % MDX_TPB))
"""


def _host_kernel(tmp_path, name, fn, n_vars, n_params, options):
    from oracle.oracle import FMA

    source, _ = build_source(fn, n_vars, n_params, options)
    source = source.replace('#include "mdx_entry.cuh"', "")
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text(PRELUDE + THREAD_DIMS + source + DRIVER)
    flags = ["-mfma", "-ffp-contract=fast"] if FMA else ["-ffp-contract=off"]
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", *flags, f"-I{KERNEL_DIR}", str(cpp),
                    "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.run.argtypes = [Args]
    lib.run.restype = ctypes.c_int
    return lib


def _solve(lib, y0, times, params, rtol, atol, max_steps=100000, hook_out=None):
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    times = np.ascontiguousarray(times, dtype=np.float64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    n, n_vars = y0.shape
    hist = np.zeros((n, len(times), n_vars))
    counters = np.zeros((4, n), dtype=np.int32)
    a = Args()
    a.y0, a.times, a.params = y0.ctypes.data, times.ctypes.data, params.ctypes.data
    a.hist = hist.ctypes.data
    a.accepted, a.rejected = counters[0].ctypes.data, counters[1].ctypes.data
    a.loop_steps, a.status = counters[2].ctypes.data, counters[3].ctypes.data
    a.n_traj, a.n_save, a.n_save_hist = n, len(times), len(times)
    a.max_steps, a.dt0, a.rtol, a.atol = max_steps, 0.0, rtol, atol
    if hook_out is not None:
        a.hook_out = hook_out.ctypes.data
    assert lib.run(a) == 0
    return hist, counters


def _agree(hist, counters, ref):
    h, acc, rej, _ = ref
    same = (counters[0] == acc) & (counters[1] == rej)
    assert same.mean() >= 0.99
    np.testing.assert_allclose(hist[same], h[same], rtol=1e-9, atol=1e-12)


def test_rodas5p_robertson_fp64(tmp_path, oracle):
    cfg = systems.robertson_config(size=64)
    lib = _host_kernel(tmp_path, "rob", cfg["ode_fn"], 3, 3, KernelOptions(lu_precision="fp64"))
    hist, counters = _solve(lib, cfg["y0"], cfg["t_span"], cfg["params"], cfg["rtol"], cfg["atol"])
    ref = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"], cfg["params"],
                       rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    _agree(hist, counters, ref)


@pytest.mark.parametrize("layout", ["dense", "sparse"])
def test_rodas5p_vdp_ring_fp64(tmp_path, oracle, layout):
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=64)
    t_span = np.linspace(0.0, 30.0, 10)
    pattern = normalize_sparsity(cfg["sparsity"], 2 * n_osc) if layout == "sparse" else None
    lib = _host_kernel(tmp_path, f"vdp_{layout}", cfg["ode_fn"], 2 * n_osc, 1,
                       KernelOptions(lu_precision="fp64", sparsity=pattern))
    hist, counters = _solve(lib, cfg["y0"], t_span, cfg["params"], 1e-6, 1e-8)
    kw = {}
    if pattern is not None:
        solver = sparse_lu_for(pattern, "amd")
        kw = dict(sparsity_mask=cfg["sparsity"], colour=solver.slots.colour, order=solver.structure.order)
    ref = oracle.solve("rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), cfg["y0"], t_span, cfg["params"],
                       rtol=1e-6, atol=1e-8, lu_precision="fp64", **kw)
    _agree(hist, counters, ref)


def test_tsit5_lorenz(tmp_path, oracle):
    """Both stage placements (registers; a per-thread column of a shared array,
    the reference's shared backend): the same arithmetic, so bit for bit."""
    cfg = systems.lorenz_config(size=64)
    out = {}
    for shared in (False, True):
        lib = _host_kernel(tmp_path, f"lorenz_{int(shared)}", cfg["ode_fn"], 3, 1,
                           KernelOptions(solver="tsit5", shared_stages=shared))
        out[shared] = _solve(lib, cfg["y0"], cfg["t_span"], cfg["params"], cfg["rtol"], cfg["atol"])
    assert np.array_equal(out[False][0], out[True][0]) and np.array_equal(out[False][1], out[True][1])
    ref = oracle.solve("tsit5", oracle.System.lorenz(), cfg["y0"], cfg["t_span"], cfg["params"],
                       rtol=cfg["rtol"], atol=cfg["atol"])
    _agree(*out[False], ref)


@pytest.mark.parametrize("layout", ["dense", "sparse"])
def test_rodas5p_fast_fp32_within_10_rtol(tmp_path, oracle, layout):
    """The fast path's logic (squared-norm controller, Newton-refined reciprocals,
    shared dense-output weights, latest-solved-last back substitution) on the
    host: within 10 rtol of an rtol = 1e-12 oracle on Robertson, and as accurate
    as the FP64-LU solve on the VdP ring."""
    if layout == "dense":
        cfg = systems.robertson_config(size=64)
        lib = _host_kernel(tmp_path, "rob32", cfg["ode_fn"], 3, 3, KernelOptions(lu_precision="fp32", fast=True))
        hist, _ = _solve(lib, cfg["y0"], cfg["t_span"], cfg["params"], cfg["rtol"], cfg["atol"])
        ref, *_ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"], cfg["params"],
                               rtol=1e-12, atol=1e-16, lu_precision="fp64")
        err = np.abs(hist - ref) / (np.abs(ref) + cfg["atol"] / cfg["rtol"])
        assert err.max() <= 10 * cfg["rtol"]
        return
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=64)
    t_span = np.linspace(0.0, 30.0, 10)
    pattern = normalize_sparsity(cfg["sparsity"], 2 * n_osc)
    lib = _host_kernel(tmp_path, "vdp32", cfg["ode_fn"], 2 * n_osc, 1,
                       KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern))
    hist, _ = _solve(lib, cfg["y0"], t_span, cfg["params"], 1e-6, 1e-8)
    system = oracle.System.vdp_ring(n_osc, 1.0, 0.1)
    ref, *_ = oracle.solve("rodas5P", system, cfg["y0"], t_span, cfg["params"], rtol=1e-12, atol=1e-14,
                           lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, cfg["y0"], t_span, cfg["params"], rtol=1e-6, atol=1e-8,
                           lu_precision="fp64")
    scale = np.abs(ref) + 1e-8 / 1e-6
    err32 = (np.abs(hist - ref) / scale).reshape(len(ref), -1).max(axis=1)
    err64 = (np.abs(o64 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    assert np.median(err32) <= 1.5 * np.median(err64) + 1e-5
    assert err32.max() <= 3.0 * err64.max()


# --- the discrete adjoint -------------------------------------------------------------
GRAD_PRELUDE = """
#define __launch_bounds__(...)
"""

GRAD_DRIVER = """
extern "C" void run_grad(MdxGradArgs g) {
  blockIdx.x = 0; blockDim.x = 1;
  for (int i = 0; i < g.n_traj; ++i) { threadIdx.x = (unsigned)i; mdx_grad_reverse(g); }
}
extern "C" void run_grad_tasks(MdxGradArgs g) {
  blockIdx.x = 0; blockDim.x = 1;
  for (int i = 0; i < g.n_run; ++i) { threadIdx.x = (unsigned)i; mdx_grad_reverse(g); }
  for (int k = 0; k < g.n_combine; ++k) { threadIdx.x = (unsigned)k; mdx_grad_combine(g); }
}
"""


class GradArgs(ctypes.Structure):
    """MdxGradArgs (mdx_args.h), field for field."""

    _fields_ = [("times", ctypes.c_void_p), ("params", ctypes.c_void_p), ("ckpt", ctypes.c_void_p),
                ("ckpt_count", ctypes.c_void_p), ("grad_hist", ctypes.c_void_p), ("grad_y0", ctypes.c_void_p),
                ("grad_params", ctypes.c_void_p), ("status", ctypes.c_void_p), ("order", ctypes.c_void_p),
                ("ckpt_capacity", ctypes.c_longlong), ("n_traj", ctypes.c_int), ("n_save", ctypes.c_int),
                ("n_run", ctypes.c_int), ("tasks", ctypes.c_void_p), ("task_out", ctypes.c_void_p),
                ("combine", ctypes.c_void_p), ("n_slots", ctypes.c_int), ("n_combine", ctypes.c_int)]


def _host_adjoint(tmp_path, name, fn, n_vars, n_params, options):
    from oracle.oracle import FMA

    source, _ = build_source(fn, n_vars, n_params, options)
    source = source.replace('#include "mdx_entry.cuh"', "")
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text(PRELUDE + THREAD_DIMS + GRAD_PRELUDE + source + DRIVER + GRAD_DRIVER)
    flags = ["-mfma", "-ffp-contract=fast"] if FMA else ["-ffp-contract=off"]
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", *flags, f"-I{KERNEL_DIR}", str(cpp),
                    "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.run.argtypes = [Args]
    lib.run.restype = ctypes.c_int
    lib.run_grad.argtypes = [GradArgs]
    lib.run_grad_tasks.argtypes = [GradArgs]
    return lib


def _value_and_grad(lib, y0, times, params, w, rtol, atol, stride, capacity, split=None):
    """Checkpointing forward pass, then the reverse sweep of sum(w * hist)."""
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    times = np.ascontiguousarray(times, dtype=np.float64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    n, n_vars = y0.shape
    segments = -(-capacity // stride)
    ckpt = np.zeros(capacity * n + segments * n * (n_vars + 1))
    ckpt_count = np.zeros(n, dtype=np.int32)
    hist = np.zeros((n, len(times), n_vars))
    counters = np.zeros((4, n), dtype=np.int32)
    a = Args()
    a.y0, a.times, a.params = y0.ctypes.data, times.ctypes.data, params.ctypes.data
    a.hist = hist.ctypes.data
    a.accepted, a.rejected = counters[0].ctypes.data, counters[1].ctypes.data
    a.loop_steps, a.status = counters[2].ctypes.data, counters[3].ctypes.data
    a.ckpt, a.ckpt_count, a.ckpt_capacity = ckpt.ctypes.data, ckpt_count.ctypes.data, capacity
    a.n_traj, a.n_save, a.n_save_hist = n, len(times), len(times)
    a.max_steps, a.dt0, a.rtol, a.atol = 100000, 0.0, rtol, atol
    assert lib.run(a) == 0
    assert (counters[3] == 0).all()
    w = np.ascontiguousarray(w, dtype=np.float64)
    grad_y0 = np.zeros((n, n_vars))
    grad_p = np.zeros((n, params.shape[1]))
    status = np.zeros(n, dtype=np.int32)
    g = GradArgs()
    g.times, g.params, g.ckpt, g.ckpt_count = times.ctypes.data, params.ctypes.data, ckpt.ctypes.data, \
        ckpt_count.ctypes.data
    g.grad_hist, g.grad_y0, g.grad_params, g.status = w.ctypes.data, grad_y0.ctypes.data, grad_p.ctypes.data, \
        status.ctypes.data
    g.ckpt_capacity, g.n_traj, g.n_save, g.n_run = capacity, n, len(times), n
    if split is None:
        lib.run_grad(g)
    else:
        # The split reverse's task table from autograd.split_plan at factor `split`.
        import torch

        from menodax_b200.autograd import split_plan

        plan = split_plan(torch.as_tensor(ckpt_count), capacity, stride, n_vars, factor=split)
        assert plan is not None
        tasks, n_slots, combine = (x.numpy() if hasattr(x, "numpy") else x for x in plan)
        tasks = np.ascontiguousarray(tasks, dtype=np.int32)
        combine = np.ascontiguousarray(combine, dtype=np.int32)
        task_out = np.full((n_slots, n_vars + params.shape[1]), np.nan)
        g.tasks, g.task_out, g.combine = tasks.ctypes.data, task_out.ctypes.data, combine.ctypes.data
        g.n_run, g.n_slots, g.n_combine = tasks.shape[0], n_slots, combine.shape[0]
        lib.run_grad_tasks(g)
        assert not np.isnan(task_out).any()
    assert (status == 0).all()
    return hist, grad_y0, grad_p


def _oracle_sens_grads(oracle, solver, system, y0, times, params, w, **kw):
    """The oracle's forward sensitivities (no error control on them) contracted with w."""
    n_vars = system.n
    hist, *_ = oracle.solve(solver, system, y0, times, params, sens=(True, list(range(system.np)), False), **kw)
    sens = hist[:, :, n_vars:].reshape(hist.shape[0], hist.shape[1], n_vars + system.np, n_vars)
    g = np.einsum("nsj,nskj->nk", w, sens)
    return hist[:, :, :n_vars], g[:, :n_vars], g[:, n_vars:]


@pytest.mark.parametrize("stride", [1, 8])
@pytest.mark.parametrize("solver", ["rodas5P", "tsit5"])
def test_adjoint_matches_oracle_forward_sensitivities(tmp_path, oracle, solver, stride):
    """The reverse sweep (segment replay, stage recompute, transposed solves,
    VJPs and Hessian-vector products) on the host, against the oracle's forward
    sensitivities on the same step sequence: the two are transposes of one linear
    map, so they agree to rounding (the GPU tests' bar, 1e-7 of the largest)."""
    if solver == "rodas5P":
        cfg = systems.robertson_config(size=32)
        system, n_vars, n_params, kw = oracle.System.robertson(), 3, 3, dict(lu_precision="fp64")
        options = KernelOptions(lu_precision="fp64", checkpoint=True, adjoint=True, ckpt_stride=stride)
    else:
        cfg = systems.lorenz_config(size=32)
        system, n_vars, n_params, kw = oracle.System.lorenz(), 3, 1, {}
        options = KernelOptions(solver="tsit5", checkpoint=True, adjoint=True, ckpt_stride=stride)
    lib = _host_adjoint(tmp_path, f"adj_{solver}_{stride}", cfg["ode_fn"], n_vars, n_params, options)
    w = np.random.default_rng(4).normal(size=(32, len(cfg["t_span"]), n_vars))
    hist, gy, gp = _value_and_grad(lib, cfg["y0"], cfg["t_span"], cfg["params"], w, cfg["rtol"], cfg["atol"],
                                   stride, capacity=4096)
    oh, oy, op = _oracle_sens_grads(oracle, solver, system, cfg["y0"], cfg["t_span"], cfg["params"], w,
                                    rtol=cfg["rtol"], atol=cfg["atol"], **kw)
    np.testing.assert_allclose(hist, oh, rtol=1e-9, atol=1e-14)
    for got, ref in ((gy, oy), (gp, op)):
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(got - ref) / scale).max() < 1e-7


@pytest.mark.parametrize("layout", ["dense", "sparse"])
def test_wide_solve_adjoint_replays_the_forward_steps_exactly(tmp_path, layout):
    """Fast arithmetic with FP32 LUs on a small system solves in double against
    the widened factors.  The reverse sweep's recompute must do the same: with a
    checkpoint every 8 steps it replays 7 of each 8 steps from the segment's
    start, with a checkpoint every step it replays none.  The two gradients agree
    to the last few ulps (contraction of the two code paths differs) when a
    replayed step is the forward step; a replay that solved in FP32 would put
    them ~1e-7 apart."""
    from menodax_b200._problem import wide_solve

    n_osc = 3
    cfg = systems.vdp_gradient_config(n_osc, size=16)
    t_span = np.linspace(0.0, 5.0, 6)
    pattern = normalize_sparsity(systems.vdp_sparsity(n_osc), 2 * n_osc) if layout == "sparse" else None
    w = np.random.default_rng(12).normal(size=(16, len(t_span), 2 * n_osc))
    out = {}
    for stride in (1, 8):
        options = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern, checkpoint=True, adjoint=True,
                                ckpt_stride=stride)
        assert wide_solve(options, 2 * n_osc)
        lib = _host_adjoint(tmp_path, f"wide_{layout}_{stride}", cfg["ode_fn"], 2 * n_osc, 1, options)
        out[stride] = _value_and_grad(lib, cfg["y0"], t_span, cfg["params"], w, 1e-6, 1e-8, stride,
                                      capacity=4096)
    assert np.array_equal(out[1][0], out[8][0])
    for a, b in zip(out[1][1:], out[8][1:]):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    assert np.abs(out[1][1]).max() > 0.0


@pytest.mark.parametrize("solver,stride", [("rodas5P", 1), ("rodas5P", 8), ("tsit5", 8)])
def test_split_reverse_composes_to_the_whole_reverse(tmp_path, solver, stride):
    """Long trajectories' reverse sweeps cut into chunks (each chunk's transfer
    matrix from unit cotangents, its offset from the injected save cotangents),
    reversed independently and composed, give the gradient of the whole sweep to
    rounding; cut at half the mean segment count, nearly every trajectory is split
    into several chunks."""
    if solver == "rodas5P":
        n_osc = 3
        cfg = systems.vdp_gradient_config(n_osc, size=16)
        fn, n_vars, n_params = cfg["ode_fn"], 2 * n_osc, 1
        options = KernelOptions(lu_precision="fp64", checkpoint=True, adjoint=True, ckpt_stride=stride,
                                sparsity=normalize_sparsity(systems.vdp_sparsity(n_osc), 2 * n_osc))
        t_span, rtol, atol = np.linspace(0.0, 5.0, 6), 1e-8, 1e-10
    else:
        cfg = systems.lorenz_config(size=16)
        fn, n_vars, n_params = cfg["ode_fn"], 3, 1
        options = KernelOptions(solver="tsit5", checkpoint=True, adjoint=True, ckpt_stride=stride)
        t_span, rtol, atol = cfg["t_span"], cfg["rtol"], cfg["atol"]
    lib = _host_adjoint(tmp_path, f"split_{solver}_{stride}", fn, n_vars, n_params, options)
    w = np.random.default_rng(21).normal(size=(16, len(t_span), n_vars))
    whole = _value_and_grad(lib, cfg["y0"], t_span, cfg["params"], w, rtol, atol, stride, capacity=4096)
    split = _value_and_grad(lib, cfg["y0"], t_span, cfg["params"], w, rtol, atol, stride, capacity=4096,
                            split=0.5)
    assert np.array_equal(whole[0], split[0])
    for a, b in zip(whole[1:], split[1:]):
        scale = np.abs(a).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(a - b) / scale).max() < 1e-9


def test_rodas5p_time_derivative_and_tf_index(tmp_path):
    """The reference's tests/test_solver_options.py:40-93 on the host: df/dt reaches
    the stages of a non-autonomous system (y' = -a y + b t, exact
    b (a t - 1 + exp(-a t)) / a^2), and tf_index ends each trajectory at its own
    time with the later saves frozen."""
    t_span = np.linspace(0.0, 1.0, 11)
    params = np.array([[10.0, 5.0, 1.0], [10.0, 5.0, 0.5]])
    lib = _host_kernel(tmp_path, "forced", systems.forced_decay, 1, 3,
                       KernelOptions(lu_precision="fp64", tf_index=2))
    a = Args()
    y0 = np.zeros((2, 1))
    hist = np.zeros((2, len(t_span), 1))
    counters = np.zeros((4, 2), dtype=np.int32)
    a.y0, a.times, a.params, a.hist = y0.ctypes.data, t_span.ctypes.data, params.ctypes.data, hist.ctypes.data
    a.accepted, a.rejected = counters[0].ctypes.data, counters[1].ctypes.data
    a.loop_steps, a.status = counters[2].ctypes.data, counters[3].ctypes.data
    a.n_traj, a.n_save, a.n_save_hist = 2, len(t_span), len(t_span)
    a.max_steps, a.dt0, a.rtol, a.atol = 100000, 1e-4, 1e-10, 1e-12
    assert lib.run(a) == 0
    exact = 5.0 * (10.0 * t_span - 1.0 + np.exp(-10.0 * t_span)) / 100.0
    np.testing.assert_allclose(hist[0, :, 0], exact, rtol=1e-8, atol=1e-10)
    stops = int(np.searchsorted(t_span, 0.5, side="right"))
    np.testing.assert_allclose(hist[1, :stops, 0], exact[:stops], rtol=1e-8, atol=1e-10)
    assert (hist[1, stops:, 0] == hist[1, stops - 1, 0]).all()
