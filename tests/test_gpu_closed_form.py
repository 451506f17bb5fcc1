"""Closed-form systems on the GPU: a stiff decay chain (Bateman), the heat
equation's first eigenmode and Kaps' singular perturbation, whose exact
solutions need no second solver.

The first group is the reference's own check of these systems
(tests/benchmark_helpers.py:37-127: rtol 1e-5, atol 1e-7, its first steps and
its bars, the chain's conservation of mass) for Tsit5 and for Rodas5P with FP64
and FP32 LUs.  The second holds larger, stiffer copies to tight tolerances:
the FP64 path at rtol 1e-10 within 1e-9 of the exact solution, dense and with
the sparse LU of each system's pattern; the FP32-LU path (fast arithmetic) at
rtol 1e-6 within 10 rtol, scaled by |y| + atol/rtol.
"""

import numpy as np
import pytest

from menodax_b200 import rodas5P, tsit5
from workloads import systems

pytestmark = pytest.mark.gpu

N_TRAJ = 256


def _case(name):
    """(ode_fn, y0, times, exact(params), sparsity pairs, first_step)."""
    if name.startswith("bateman"):
        n = int(name[len("bateman"):])
        fn, y0, m = systems.make_bateman_system(n, 1e2 if n <= 4 else 1e4)
        pattern = np.argwhere((m != 0.0) | np.eye(n, dtype=bool))
        return fn, y0, systems.BATEMAN_TIMES, lambda p: systems.linear_exact(m, y0, systems.BATEMAN_TIMES, p), \
            pattern, 1e-4
    if name.startswith("heat"):
        n = int(name[len("heat"):])
        fn, y0 = systems.make_heat_system(n)
        pattern = [(i, j) for i in range(n) for j in (i - 1, i, i + 1) if 0 <= j < n]
        return fn, y0, systems.HEAT_TIMES, lambda p: systems.heat_exact(n, systems.HEAT_TIMES, p), pattern, 1e-4
    pairs = int(name[len("kaps"):])
    fn, y0 = systems.make_kaps_system(pairs, 1e-2 if pairs <= 2 else 1e-6)
    pattern = [(2 * k + a, 2 * k + b) for k in range(pairs) for a in (0, 1) for b in (0, 1)]
    return fn, y0, systems.KAPS_TIMES, lambda p: systems.kaps_exact(systems.KAPS_TIMES, p, pairs), pattern, 1e-3


def _inputs(y0):
    params = systems.rate_scale_params(N_TRAJ)
    return np.broadcast_to(y0, (N_TRAJ, len(y0))).copy(), params


SOLVES = {
    "tsit5": lambda fn, y, t, p, **kw: tsit5.solve(fn, y, t, p, **kw),
    "rodas5P_fp64": lambda fn, y, t, p, **kw: rodas5P.solve(fn, y, t, p, lu_precision="fp64", **kw),
    "rodas5P_fp32": lambda fn, y, t, p, **kw: rodas5P.solve(fn, y, t, p, lu_precision="fp32", **kw),
}


@pytest.mark.parametrize("solve", list(SOLVES))
@pytest.mark.parametrize("name,bar", [("bateman4", 2e-2), ("heat4", 3e-2), ("kaps2", 3e-2)])
def test_reference_closed_form_cases(solve, name, bar):
    fn, y0, times, exact, _, first_step = _case(name)
    y, params = _inputs(y0)
    t_span = times[:3]
    out = SOLVES[solve](fn, y, t_span, params, rtol=1e-5, atol=1e-7, first_step=first_step)
    np.testing.assert_allclose(out, exact(params)[:, :3], rtol=bar, atol=3e-5)
    if name.startswith("bateman"):
        np.testing.assert_allclose(out.sum(axis=-1), 1.0, atol=3e-5)


@pytest.mark.parametrize("layout", ["dense", "sparse"])
@pytest.mark.parametrize("name", ["bateman16", "heat32", "kaps8"])
def test_fp64_reaches_the_exact_solution(name, layout):
    fn, y0, times, exact, pattern, _ = _case(name)
    y, params = _inputs(y0)
    out = rodas5P.solve(fn, y, times, params, rtol=1e-10, atol=1e-14, lu_precision="fp64",
                        sparsity=pattern if layout == "sparse" else None)
    np.testing.assert_allclose(out, exact(params), rtol=1e-8, atol=1e-9)


@pytest.mark.parametrize("name", ["bateman16", "heat32", "kaps8"])
def test_fp32_lu_within_10_rtol_of_the_exact_solution(name):
    fn, y0, times, exact, pattern, _ = _case(name)
    y, params = _inputs(y0)
    rtol, atol = 1e-6, 1e-10
    out = rodas5P.solve(fn, y, times, params, rtol=rtol, atol=atol, lu_precision="fp32", sparsity=pattern)
    ref = exact(params)
    err = np.abs(out - ref) / (np.abs(ref) + atol / rtol)
    assert err.max() <= 10 * rtol
