"""API validation that needs no GPU: the reference's error messages and argument
normalisation (modax/_jax_common.py:23-36, modax/rodas5P.py:1204-1211)."""

import numpy as np
import pytest

from menodax_b200 import _ensemble, rodas5P, tsit5
from workloads import systems


def test_shape_errors():
    with pytest.raises(ValueError, match="y0 must have shape"):
        rodas5P.solve(systems.robertson, np.zeros((2, 3, 1)), systems.ROBERTSON_TIMES, np.zeros(3))
    with pytest.raises(ValueError, match="params must have shape"):
        rodas5P.solve(systems.robertson, np.zeros((2, 3)), systems.ROBERTSON_TIMES, np.zeros((3, 3)))


def test_option_errors():
    with pytest.raises(ValueError, match="lu_precision"):
        rodas5P.solve(systems.robertson, np.zeros(3), systems.ROBERTSON_TIMES, np.zeros(3), lu_precision="fp16")
    with pytest.raises(ValueError, match="save_history=False"):
        rodas5P.solve(systems.robertson, np.zeros(3), systems.ROBERTSON_TIMES, np.zeros(3), save_history=False)
    with pytest.raises(ValueError, match="positive hook_size"):
        rodas5P.solve(systems.robertson, np.zeros(3), systems.ROBERTSON_TIMES, np.zeros(3),
                      save_hook=lambda *a: None)
    with pytest.raises(ValueError, match="trajectories_per_block must be positive"):
        rodas5P.trajectories_per_block_or_default(0)
    with pytest.raises(ValueError, match="backend must be"):
        tsit5.solve(systems.lorenz, np.zeros(3), (0.0, 1.0), np.zeros(1), backend="gpu")
    with pytest.raises(ValueError, match="shared backend requires"):
        tsit5.solve(systems.make_vdp_system(16)[0], np.zeros(32), (0.0, 1.0), np.zeros(1), backend="shared")


def test_normalisation_broadcasts():
    y0, p, n, nv = _ensemble.normalize_y0_params(np.ones(3), np.ones((5, 2)))
    assert (n, nv) == (5, 3) and tuple(y0.shape) == (5, 3) and tuple(p.shape) == (5, 2)
    y0, p, n, nv = _ensemble.normalize_y0_params(np.ones((4, 2)), np.ones(1))
    assert n == 4 and tuple(p.shape) == (4, 1)
    assert _ensemble.initial_step(None) == 0.0 and _ensemble.initial_step(1e-3) == 1e-3
    assert _ensemble.build_error_weights(None, 4, 2) is None
    w = _ensemble.build_error_weights([1.0, 0.0], 4, 2)
    assert tuple(w.shape) == (4, 2)


def test_trajectories_per_block_default():
    assert rodas5P.trajectories_per_block_or_default() == 32
    assert rodas5P.trajectories_per_block_or_default(8) == 8


def test_team_option_errors():
    cfg = systems.vdp_ring_config(4, size=4)
    args = (cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"])
    with pytest.raises(ValueError, match="team must be"):
        rodas5P.solve(*args, team=3)

    import torch

    p_grad = torch.tensor(cfg["params"], requires_grad=True)
    with pytest.raises(ValueError, match="sparsity pattern and sens_error_control=False"):
        rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], p_grad, team=8)
    with pytest.raises(ValueError, match="whole warps"):
        rodas5P.solve(*args, team=8, trajectories_per_block=3)


def _robertson_array(y, t, p, out):
    """The Robertson right-hand side written as an array writer."""
    out[0] = -p[0] * y[0] + p[1] * y[1] * y[2]
    out[1] = p[0] * y[0] - p[1] * y[1] * y[2] - p[2] * y[1] ** 2
    out[2] = p[2] * y[1] ** 2


def test_array_rhs_traces_into_the_primal_graph():
    """An array writer of the same expressions lands on the same graph nodes as the
    tuple form, so the kernels' stage code is the same; derivatives stay with ode_fn."""
    from menodax_b200._problem import KernelOptions, build_source
    from menodax_b200._trace import TraceError, trace, trace_array_rhs

    tr = trace(systems.robertson, 3, 3)
    arr = trace_array_rhs(_robertson_array, tr)
    assert arr.graph is tr.graph and arr.outputs == tr.outputs
    plain, _ = build_source(systems.robertson, 3, 3, KernelOptions())
    with_array, _ = build_source(systems.robertson, 3, 3, KernelOptions(array_rhs=_robertson_array))
    assert plain == with_array

    def partial(y, t, p, out):
        out[0] = y[0]

    with pytest.raises(TraceError, match="unwritten"):
        trace_array_rhs(partial, tr)

    def scaled(y, t, p, out):
        for i in range(3):
            out[i] = 2.0 * y[i]

    src, _ = build_source(systems.robertson, 3, 3, KernelOptions(array_rhs=scaled))
    assert src != plain and "mdx_rhs" in src
    with pytest.raises(ValueError, match="array_rhs must be a callable"):
        rodas5P.solve(systems.robertson, np.zeros(3), systems.ROBERTSON_TIMES, np.zeros(3), array_rhs=3)


def test_gradient_hints_keep_a_bounded_number_of_problems():
    from menodax_b200 import autograd

    hints = {}
    for k in range(autograd.HINT_PROBLEMS + 10):
        autograd._remember(hints, ("problem", k), k)
    assert len(hints) == autograd.HINT_PROBLEMS
    assert ("problem", 0) not in hints and ("problem", autograd.HINT_PROBLEMS + 9) in hints
    autograd._remember(hints, ("problem", 10), "again")   # refreshed: now the newest
    autograd._remember(hints, ("problem", 999), 0)
    assert ("problem", 10) in hints and ("problem", 11) not in hints
