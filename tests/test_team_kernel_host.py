"""The team kernel, compiled for the host with its lanes as threads.

The team kernel (one trajectory per team of 4-32 lanes, its vectors and matrix
in a shared-memory slice) keeps every lane of a team on the same path, so its
warp intrinsics can be emulated lane by lane: `__syncwarp` is a barrier over
the team's lanes, a shuffle writes the lane's value to an
exchange slot, meets the team at the barrier, reads the source lane's slot and
meets it again, and `__any_sync` is the same with an OR.  Lanes are
user-level contexts on one host thread, switched at every barrier; the block's
dynamic shared memory is one host buffer; blocks run one after another.  The kernel
source is exactly what the GPU compiles (`build_source`), so this checks the
team code -- class loops, panel LU, blocked solves, the first lane's sparse
solves, the error norm and the controller -- on every CPU run, against the
oracle and the thread kernel compiled the same way.
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

from test_kernel_host import PRELUDE, Args, _host_kernel, _solve

LANES = """
#include <ucontext.h>
#include <cstdio>
#include <cstdlib>
struct HostDim { unsigned x, y, z; };
static HostDim threadIdx, blockIdx, blockDim;
static unsigned host_lane;
static int host_team_size = 32;

// Lanes are user-level contexts on one OS thread: a lane runs until it reaches
// a barrier or ends, then the scheduler runs the next; a team's lanes leave the
// barrier together once every lane of the team that has not ended waits there.
struct HostLane { ucontext_t ctx; bool done, waiting; };
static HostLane host_lanes[32];
static ucontext_t host_scheduler;
static unsigned long long host_slot[32];

static inline void __syncwarp(unsigned = 0xffffffffu) {
  host_lanes[host_lane].waiting = true;
  swapcontext(&host_lanes[host_lane].ctx, &host_scheduler);
}
template <class T> static inline T host_exchange(T v, unsigned src) {
  std::memcpy(&host_slot[host_lane], &v, sizeof(T));
  __syncwarp();
  T r;
  std::memcpy(&r, &host_slot[src], sizeof(T));
  __syncwarp();
  return r;
}
template <class T> static inline T __shfl_xor_sync(unsigned, T v, int off, int width = 32) {
  const unsigned base = host_lane & ~(unsigned)(width - 1);
  return host_exchange(v, base | ((host_lane - base) ^ (unsigned)off));
}
template <class T> static inline T __shfl_sync(unsigned, T v, int src, int width = 32) {
  const unsigned base = host_lane & ~(unsigned)(width - 1);
  return host_exchange(v, base + ((unsigned)src & (unsigned)(width - 1)));
}
static inline bool __any_sync(unsigned mask, bool p) {
  host_slot[host_lane] = p ? 1ull : 0ull;
  __syncwarp();
  bool r = false;
  for (unsigned l = 0; l < 32; ++l) if ((mask >> l) & 1u) r = r || host_slot[l] != 0ull;
  __syncwarp();
  return r;
}
static inline int atomicAdd(int* p, int v) { const int o = *p; *p += v; return o; }
#define __shared__
#define __align__(n)
#define __launch_bounds__(...)
namespace mdx { namespace team { alignas(16) unsigned char mdx_team_smem[1 << 20]; } }
"""

DRIVER = """
static MdxSolveArgs host_args;
static void host_lane_main() {
  mdx_solve_plain(host_args);
  host_lanes[host_lane].done = true;
}

extern "C" int run(MdxSolveArgs a) {
  static char stacks[MDX_TPB][1 << 18];
  host_args = a;
  host_team_size = MDX_TEAM;
  blockDim.x = MDX_TPB;
  const int per_block = MDX_TPB / MDX_TEAM;
  const int blocks = (a.n_traj + per_block - 1) / per_block;
  for (int b = 0; b < blocks; ++b) {
    blockIdx.x = (unsigned)b;
    for (int l = 0; l < MDX_TPB; ++l) {
      HostLane& h = host_lanes[l];
      h.done = h.waiting = false;
      getcontext(&h.ctx);
      h.ctx.uc_stack.ss_sp = stacks[l];
      h.ctx.uc_stack.ss_size = sizeof(stacks[l]);
      h.ctx.uc_link = &host_scheduler;
      makecontext(&h.ctx, host_lane_main, 0);
    }
    for (;;) {
      bool live = false;
      for (int l = 0; l < MDX_TPB; ++l) {
        if (host_lanes[l].done || host_lanes[l].waiting) continue;
        host_lane = (unsigned)l;
        threadIdx.x = (unsigned)l;
        swapcontext(&host_scheduler, &host_lanes[l].ctx);
      }
      for (int t = 0; t < MDX_TPB / MDX_TEAM; ++t) {
        int waiting = 0, done = 0;
        for (int l = t * MDX_TEAM; l < (t + 1) * MDX_TEAM; ++l) {
          waiting += host_lanes[l].waiting;
          done += host_lanes[l].done;
        }
        if (waiting && done) return 1;  // a lane ended while its team waits: divergent code
        if (waiting == MDX_TEAM)
          for (int l = t * MDX_TEAM; l < (t + 1) * MDX_TEAM; ++l) host_lanes[l].waiting = false;
        live = live || done < MDX_TEAM;
      }
      if (!live) break;
    }
  }
  return 0;
}
"""


def _team_kernel(tmp_path, name, fn, n_vars, n_params, options):
    from oracle.oracle import FMA

    source, meta = build_source(fn, n_vars, n_params, options)
    assert meta["shared_bytes"] <= 1 << 20
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text(PRELUDE + LANES + source + DRIVER)
    flags = ["-mfma", "-ffp-contract=fast"] if FMA else ["-ffp-contract=off"]
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", *flags, f"-I{KERNEL_DIR}",
                    str(cpp), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.run.argtypes = [Args]
    lib.run.restype = ctypes.c_int
    return lib


def _same_steps_and_states(hist, counters, h, acc, rej, rtol=1e-9, atol=1e-12):
    same = (counters[0] == acc) & (counters[1] == rej)
    assert same.mean() >= 0.99
    np.testing.assert_allclose(hist[same], h[same], rtol=rtol, atol=atol)


@pytest.mark.parametrize("team", [4, 8])
@pytest.mark.parametrize("layout", ["sparse", "dense"])
def test_team_vdp_ring_fp64_matches_oracle(tmp_path, oracle, team, layout):
    """The GPU test of the same name on the host: FP64, both layouts."""
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=16)
    t_span = np.linspace(0.0, 30.0, 10)
    pattern = normalize_sparsity(cfg["sparsity"], 2 * n_osc) if layout == "sparse" else None
    lib = _team_kernel(tmp_path, f"team_{layout}_{team}", cfg["ode_fn"], 2 * n_osc, 1,
                       KernelOptions(lu_precision="fp64", sparsity=pattern, team=team, threads_per_block=32))
    hist, counters = _solve(lib, cfg["y0"], t_span, cfg["params"], 1e-6, 1e-8)
    kw = {}
    if pattern is not None:
        solver = sparse_lu_for(pattern, "amd")
        kw = dict(sparsity_mask=cfg["sparsity"], colour=solver.slots.colour, order=solver.structure.order)
    h, acc, rej, _ = oracle.solve("rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), cfg["y0"], t_span,
                                  cfg["params"], rtol=1e-6, atol=1e-8, lu_precision="fp64", **kw)
    _same_steps_and_states(hist, counters, h, acc, rej)


@pytest.mark.parametrize("n_osc", [5, 6])
def test_team_dense_panels_factor_like_the_thread_kernel(tmp_path, n_osc):
    """The GPU panel test on the host: fast FP64 arithmetic, four-column panels on
    4 lanes (10 states end on a two-column panel), against the thread kernel's
    register LU compiled the same way."""
    cfg = systems.vdp_ring_config(n_osc, size=16)
    t_span = np.linspace(0.0, 30.0, 10)
    n = 2 * n_osc
    team = _team_kernel(tmp_path, f"panel_{n}", cfg["ode_fn"], n, 1,
                        KernelOptions(lu_precision="fp64", fast=True, team=4, threads_per_block=32))
    thread = _host_kernel(tmp_path, f"thread_{n}", cfg["ode_fn"], n, 1, KernelOptions(lu_precision="fp64", fast=True))
    h4, c4 = _solve(team, cfg["y0"], t_span, cfg["params"], 1e-6, 1e-8)
    h0, c0 = _solve(thread, cfg["y0"], t_span, cfg["params"], 1e-6, 1e-8)
    _same_steps_and_states(h4, c4, h0, c0[0], c0[1], atol=1e-9)


@pytest.mark.parametrize("team", [8, 16])
def test_team_brusselator_dense_fp32_as_accurate_as_fp64(tmp_path, oracle, team):
    """Fast FP32 dense LU with four-column panels (16 states: 8 lanes hold two
    pivot-row entries each, 16 lanes one) on a smooth system."""
    n_grid = 8
    cfg = systems.brusselator_config(n_grid=n_grid, size=16)
    lib = _team_kernel(tmp_path, f"bruss_{team}", cfg["ode_fn"], 2 * n_grid, 1,
                       KernelOptions(lu_precision="fp32", fast=True, team=team, threads_per_block=32))
    h32, _ = _solve(lib, cfg["y0"], cfg["t_span"], cfg["params"], cfg["rtol"], cfg["atol"])
    system = oracle.System.brusselator(n_grid)
    ref, *_ = oracle.solve("rodas5P", system, cfg["y0"], cfg["t_span"], cfg["params"], rtol=1e-12, atol=1e-14,
                           lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                           atol=cfg["atol"], lu_precision="fp64")
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    err64 = (np.abs(o64 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    assert np.median(err32) <= 1.5 * np.median(err64) + 10 * cfg["rtol"]
    assert err32.max() <= 3.0 * err64.max()


# --- the team reverse sweep ----------------------------------------------------------
GRAD_DRIVER = """
static MdxGradArgs host_gargs;
static void host_grad_lane_main() {
  mdx_grad_reverse(host_gargs);
  host_lanes[host_lane].done = true;
}

extern "C" int run_grad(MdxGradArgs g) {
  static char stacks[MDX_TPB][1 << 18];
  host_gargs = g;
  host_team_size = MDX_TEAM;
  blockDim.x = MDX_TPB;
  const int per_block = MDX_TPB / MDX_TEAM;
  const int blocks = (g.n_run + per_block - 1) / per_block;
  for (int b = 0; b < blocks; ++b) {
    blockIdx.x = (unsigned)b;
    for (int l = 0; l < MDX_TPB; ++l) {
      HostLane& h = host_lanes[l];
      h.done = h.waiting = false;
      getcontext(&h.ctx);
      h.ctx.uc_stack.ss_sp = stacks[l];
      h.ctx.uc_stack.ss_size = sizeof(stacks[l]);
      h.ctx.uc_link = &host_scheduler;
      makecontext(&h.ctx, host_grad_lane_main, 0);
    }
    for (;;) {
      bool live = false;
      for (int l = 0; l < MDX_TPB; ++l) {
        if (host_lanes[l].done || host_lanes[l].waiting) continue;
        host_lane = (unsigned)l;
        threadIdx.x = (unsigned)l;
        swapcontext(&host_scheduler, &host_lanes[l].ctx);
      }
      for (int t = 0; t < MDX_TPB / MDX_TEAM; ++t) {
        int waiting = 0, done = 0;
        for (int l = t * MDX_TEAM; l < (t + 1) * MDX_TEAM; ++l) {
          waiting += host_lanes[l].waiting;
          done += host_lanes[l].done;
        }
        if (waiting && done) return 1;
        if (waiting == MDX_TEAM)
          for (int l = t * MDX_TEAM; l < (t + 1) * MDX_TEAM; ++l) host_lanes[l].waiting = false;
        live = live || done < MDX_TEAM;
      }
      if (!live) break;
    }
  }
  return 0;
}
"""


@pytest.mark.parametrize("stride,lu_precision", [(1, "fp64"), (8, "fp64"), (8, "fp32")])
def test_team_adjoint_matches_oracle_forward_sensitivities(tmp_path, oracle, stride, lu_precision):
    """The team kernel's checkpointing forward pass and its reverse sweep (class-loop
    VJPs and Hessian-vector products, the first lane's transposed sparse solves,
    segment replay) on the VdP ring, against the oracle's forward sensitivities on
    the same step sequence (1e-7 of the largest component); with FP32 LUs the
    reverse sweep differentiates the FP32 solve, so it is held against the FP64
    team gradient at the FP32 LU's accuracy."""
    from dataclasses import replace

    from oracle.oracle import FMA
    from menodax_b200._problem import team_grad_block_threads
    from test_kernel_host import GradArgs, _oracle_sens_grads, _value_and_grad

    n_osc = 3
    cfg = systems.vdp_gradient_config(n_osc, size=16)
    t_span = np.linspace(0.0, 5.0, 6)
    pattern = normalize_sparsity(cfg["sparsity"] if "sparsity" in cfg else systems.vdp_sparsity(n_osc), 2 * n_osc)

    def build(prec):
        opts = KernelOptions(lu_precision=prec, fast=prec == "fp32", sparsity=pattern, team=8, checkpoint=True,
                             adjoint=True, ckpt_stride=stride)
        # One warp per block: the host harness emulates 32 lanes.
        opts = replace(opts, threads_per_block=min(32, team_grad_block_threads(2 * n_osc, 1, opts)))
        source, _ = build_source(cfg["ode_fn"], 2 * n_osc, 1, opts)
        name = f"team_adj_{stride}_{prec}"
        cpp = tmp_path / f"{name}.cpp"
        so = tmp_path / f"{name}.so"
        cpp.write_text(PRELUDE + LANES + "#define MDX_BLOCK_SHARED static\n" + source + DRIVER + GRAD_DRIVER)
        flags = ["-mfma", "-ffp-contract=fast"] if FMA else ["-ffp-contract=off"]
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", *flags, f"-I{KERNEL_DIR}",
                        str(cpp), "-o", str(so)], check=True)
        lib = ctypes.CDLL(str(so))
        lib.run.argtypes = [Args]
        lib.run.restype = ctypes.c_int
        lib.run_grad.argtypes = [GradArgs]
        lib.run_grad.restype = ctypes.c_int
        return lib

    w = np.random.default_rng(9).normal(size=(16, len(t_span), 2 * n_osc))
    kw = dict(rtol=1e-8, atol=1e-10)
    h64, gy64, gp64 = _value_and_grad(build("fp64"), cfg["y0"], t_span, cfg["params"], w, stride=stride,
                                      capacity=4096, **kw)
    if lu_precision == "fp64":
        oh, oy, op = _oracle_sens_grads(oracle, "rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), cfg["y0"],
                                        t_span, cfg["params"], w, lu_precision="fp64",
                                        sparsity_mask=np.asarray(systems.vdp_sparsity(n_osc), dtype=bool),
                                        colour=sparse_lu_for(pattern, "amd").slots.colour,
                                        order=sparse_lu_for(pattern, "amd").structure.order, **kw)
        np.testing.assert_allclose(h64, oh, rtol=1e-9, atol=1e-12)
        for got, ref in ((gy64, oy), (gp64, op)):
            scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
            assert (np.abs(got - ref) / scale).max() < 1e-7
    else:
        h32, gy32, gp32 = _value_and_grad(build("fp32"), cfg["y0"], t_span, cfg["params"], w, stride=stride,
                                          capacity=4096, **kw)
        g64 = np.concatenate([gy64, gp64], axis=1)
        g32 = np.concatenate([gy32, gp32], axis=1)
        rel = np.abs(g32 - g64).max(axis=1) / np.abs(g64).max(axis=1)
        assert np.median(rel) < 1e-4


def test_team_save_hook_matches_the_thread_kernel(tmp_path):
    """A save hook in the team kernel (the generated hook code on the team's first
    lane, at the initial state, every dense-output save and the frozen saves)
    accumulates what the thread kernel's hook does (8-state VdP ring, teams of 4)."""
    from test_kernel_host import _host_kernel

    cfg = systems.vdp_ring_config(4, size=4)
    t_span = np.linspace(0.0, 5.0, 9)
    weights = np.linspace(0.5, 1.5, 9)

    def hook(save_idx, y, t, p, acc):
        acc[0] += weights[save_idx] * y[0]
        acc[1] += y[3] * y[3]
        acc[2] += 1.0

    out = []
    for team in (0, 4):
        opts = KernelOptions(lu_precision="fp64", save_hook=hook, hook_size=3, team=team, threads_per_block=32)
        lib = _team_kernel(tmp_path, "hook_team", cfg["ode_fn"], 8, 1, opts) if team else \
            _host_kernel(tmp_path, "hook_thread", cfg["ode_fn"], 8, 1, opts)
        hook_out = np.zeros((4, 3))
        hist, counters = _solve(lib, cfg["y0"], t_span, cfg["params"], 1e-8, 1e-10, hook_out=hook_out)
        out.append((hist, counters, hook_out))
    (h0, c0, a0), (h4, c4, a4) = out
    assert (c0[0] == c4[0]).all() and (a0[:, 2] == 9).all()
    np.testing.assert_allclose(h4, h0, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(a4, a0, rtol=1e-9, atol=1e-12)
