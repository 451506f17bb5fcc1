"""Ahead-of-time NVRTC compilation of the benchmark problems' kernels.

The cubins land in the in-tree cache (``menodax_b200/_cubin_cache``), keyed on
the generated source, so a solve of the same problem on a GPU box loads them
instead of compiling.  Needs no GPU.
"""

from __future__ import annotations

from menodax_b200 import _native, systems
from menodax_b200._problem import KernelOptions, build_source, compile_options


def benchmark_problems():
    """``(ode_fn, n_vars, n_params, options)`` for every kernel the benchmarks launch."""
    out = [(systems.lorenz, 3, 1, KernelOptions(solver="tsit5"))]
    for prec in ("fp32", "fp64"):
        out.append((systems.robertson, 3, 3, KernelOptions(lu_precision=prec)))
    return out


def compile_benchmark_kernels(verbose: bool = False) -> int:
    n = 0
    for fn, n_vars, n_params, opts in benchmark_problems():
        src, _ = build_source(fn, n_vars, n_params, opts)
        _native.compile_cubin(src, compile_options(opts))
        n += 1
        if verbose:
            print(f"compiled {opts.solver} n_vars={n_vars} {opts}")
    return n
