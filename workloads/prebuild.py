"""Ahead-of-time NVRTC compilation of the benchmark problems' kernels.

The cubins land in the in-tree cache (``menodax_b200/_cubin_cache``), keyed on
the generated source, so a solve of the same problem on a GPU box loads them
instead of compiling.  Needs no GPU.
"""

from __future__ import annotations

from menodax_b200 import _native
from workloads import systems
from menodax_b200._problem import KernelOptions, build_source, compile_options


def benchmark_problems():
    """``(ode_fn, n_vars, n_params, options)`` for every kernel the benchmark launches."""
    out = [(systems.lorenz, 3, 1, KernelOptions(solver="tsit5"))]
    for prec in ("fp32", "fp64"):
        out.append((systems.robertson, 3, 3, KernelOptions(lu_precision=prec)))
    for tpb in (32, 64, 128):
        out.append((systems.robertson, 3, 3, KernelOptions(lu_precision="fp32", fast=True, threads_per_block=tpb)))
    vdp = systems.vdp_gradient_config(1, size=1)["ode_fn"]
    for prec, fast in (("fp64", False), ("fp32", True)):
        out.append((vdp, 2, 1, KernelOptions(lu_precision=prec, fast=fast)))
        for stride in (1, 8, 32):
            out.append((vdp, 2, 1, KernelOptions(lu_precision=prec, fast=fast, checkpoint=True, adjoint=True,
                                                  ckpt_stride=stride)))
    return out


def _compile_one(i):
    fn, n_vars, n_params, opts = benchmark_problems()[i]
    src, _ = build_source(fn, n_vars, n_params, opts)
    _native.compile_cubin(src, compile_options(opts))
    return i


def compile_benchmark_kernels(workers: int = 8) -> int:
    """Compile (or find in the cache) every benchmark kernel, in parallel processes."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    count = len(benchmark_problems())
    with ProcessPoolExecutor(min(workers, count), mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_compile_one, range(count)))
    return count
