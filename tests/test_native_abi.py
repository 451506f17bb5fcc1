"""The C ABI: the library loads without a GPU, exports every declared symbol,
compiles kernels with NVRTC for sm_100a, and rejects bad arguments with a
status code instead of crashing."""

import re
from pathlib import Path

import pytest

from workloads import systems
from menodax_b200._problem import KernelOptions, build_source, compile_options

HEADER = Path(__file__).resolve().parents[1] / "include" / "menodax.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(mdx_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported(native):
    lib = native.lib()
    names = declared_functions()
    assert "mdx_solve" in names and "mdx_compile" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(native.EXPORTED)


def test_version_string(native):
    assert native.lib().mdx_version().startswith(b"menodax_b200")


@pytest.mark.parametrize("solver,fn,n,np_", [
    ("tsit5", systems.lorenz, 3, 1),
    ("rodas5P", systems.robertson, 3, 3),
])
def test_nvrtc_compiles_for_sm100a(native, solver, fn, n, np_):
    opts = KernelOptions(solver=solver)
    src, _ = build_source(fn, n, np_, opts)
    cubin = native.compile_cubin(src, compile_options(opts))
    assert cubin[:4] == b"\x7fELF"


def test_compile_error_is_reported(native):
    with pytest.raises(native.NativeError, match="NVRTC"):
        native.compile_cubin("this is not C++", [])


def test_null_arguments_are_rejected(native):
    lib = native.lib()
    assert lib.mdx_solve(None, None, None) == -1
    assert lib.mdx_plan_create(None, None) == -1
    assert "null" in native.last_error()


def test_plan_validation(native):
    opts = KernelOptions(solver="tsit5")
    src, _ = build_source(systems.lorenz, 3, 1, opts)
    cubin = native.compile_cubin(src, compile_options(opts))
    with pytest.raises(native.NativeError, match="threads_per_block"):
        native.Plan(native.MDX_SOLVER_TSIT5, 3, 3, 1, 48, 0, cubin)
    with pytest.raises(native.NativeError, match="unknown solver"):
        native.Plan(7, 3, 3, 1, 32, 0, cubin)
    plan = native.Plan(native.MDX_SOLVER_TSIT5, 3, 3, 1, 32, 0, cubin)
    d = native.SolveDesc()
    d.mode = 5
    d.n_traj = 4
    d.n_save = 2
    d.n_save_hist = 2
    with pytest.raises(native.NativeError, match="launch mode"):
        plan.solve(d, 0)
    assert plan.workspace_size(native.MDX_LAUNCH_PERSISTENT, 100) >= 4
    assert plan.workspace_size(native.MDX_LAUNCH_PLAIN, 100) == 0


def test_grad_count_is_validated(native):
    """mdx_grad's count (trajectories one reverse launch takes) lies in [0, n_traj]."""
    from menodax_b200._problem import get_problem

    prob = get_problem(systems.cascade, 2, 2, KernelOptions(lu_precision="fp64", checkpoint=True, adjoint=True))
    d = native.GradDesc()
    d.n_traj = 4
    d.n_save = 2
    d.count = 5
    with pytest.raises(native.NativeError, match="count 5 outside"):
        prob.plan.grad(d, 0)
    d.count = -1
    with pytest.raises(native.NativeError, match="count -1 outside"):
        prob.plan.grad(d, 0)
