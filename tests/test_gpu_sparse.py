"""The structure-compiled sparse LU on the GPU.

Mirrors the reference's end-to-end checks (tests/test_sparse_direct.py:345-416):
a sparse solve agrees with the dense-LU solve of the same system, with the
oracle run on the same colouring and elimination order, and the table-driven
and straight-line forms of the sparse code agree bit for bit.
"""

import numpy as np
import pytest

from menodax_b200 import rodas5P
from workloads import systems
from menodax_b200._sparse_direct import sparse_lu_for
from menodax_b200._sparsity import normalize_sparsity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("horizon", [30.0, 300.0])
def test_vdp_ring_sparse_matches_oracle(oracle, horizon):
    """Within 1e-9 over a few relaxation cycles; over many, rounding-level phase
    drift is amplified at the fast jumps (|y'| ~ mu), so there a bounded fraction
    of saved values may drift past 1e-9 and none past 1e-6."""
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=512)
    t_span = np.linspace(0.0, horizon, 20)
    mask = cfg["sparsity"]
    hist, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], rtol=1e-6,
                                atol=1e-8, lu_precision="fp64", sparsity=mask, return_stats=True)
    solver = sparse_lu_for(normalize_sparsity(mask, 2 * n_osc), "amd")
    h, a, r, _ = oracle.solve("rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), cfg["y0"], t_span,
                              cfg["params"], rtol=1e-6, atol=1e-8, lu_precision="fp64",
                              sparsity_mask=mask, colour=solver.slots.colour,
                              order=solver.structure.order)
    same = (np.asarray(stats["accepted_steps"]) == a) & (np.asarray(stats["rejected_steps"]) == r)
    assert same.mean() >= 0.999
    if horizon <= 30.0:
        np.testing.assert_allclose(hist[same], h[same], rtol=1e-9, atol=1e-12)
    else:
        rel = np.abs(hist[same] - h[same]) / (np.abs(h[same]) + 1e-12)
        assert (rel <= 1e-9).mean() >= 0.999
        assert rel.max() <= 1e-6


@pytest.mark.parametrize("ordering", ["amd", "natural"])
def test_brusselator_sparse_agrees_with_dense(ordering):
    cfg = systems.brusselator_config(n_grid=8, size=64)
    kw = dict(rtol=1e-10, atol=1e-12, lu_precision="fp64")
    dense = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], **kw)
    sparse = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"],
                           sparsity=cfg["sparsity"], ordering=ordering, **kw)
    np.testing.assert_allclose(sparse, dense, rtol=1e-7, atol=1e-9)


def test_table_driven_and_unrolled_sparse_code_agree_bitwise():
    cfg = systems.brusselator_config(n_grid=8, size=128)
    kw = dict(rtol=1e-6, atol=1e-8, lu_precision="fp32", sparsity=cfg["sparsity"], return_stats=True)
    h1, s1 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], sparse_code="unrolled", **kw)
    h2, s2 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], sparse_code="tables", **kw)
    assert np.array_equal(h1, h2)
    assert np.array_equal(s1["loop_steps"], s2["loop_steps"])


def test_brusselator_64_fp32_sparse_as_accurate_as_fp64(oracle):
    """Against a tight FP64 oracle (rtol 1e-12), the FP32-LU sparse solve is as
    accurate as the FP64-LU dense solve at the same tolerance.  On this oscillatory
    system the global error of any rtol=1e-6 solve is about 1e-4 (the oracle's own
    FP64 solve included), so the 10*rtol bar of the Robertson test does not apply."""
    cfg = systems.brusselator_config(n_grid=32, size=128)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"])
    h32 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], lu_precision="fp32",
                        sparsity=cfg["sparsity"], **kw)
    ref, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), cfg["y0"], cfg["t_span"],
                           cfg["params"], rtol=1e-12, atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), cfg["y0"], cfg["t_span"],
                           cfg["params"], lu_precision="fp64", **kw)
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).max()
    err64 = (np.abs(o64 - ref) / scale).max()
    assert err32 <= 1.5 * err64 + 10 * cfg["rtol"]


def test_vdp_ring_fp32_sparse_as_accurate_as_fp64(oracle):
    """The Van der Pol ring's product path (FP32 LU, fast arithmetic, AMD-ordered sparse LU)
    against a tight FP64 oracle, by the distribution of each trajectory's worst
    relative error: median and 90th percentile as small as the FP64-LU solve's at
    the same tolerance (to 1.5x + 10 rtol), the worst trajectory within 3x.  The
    worst trajectory alone is a noisy measure on this stiff ring: a few
    trajectories near a relaxation jump carry it, and on 1,024 trajectories the
    oracle's own FP32 solve with the reference's arithmetic lands at 5x the FP64
    worst case while its median is within 1.3x."""
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=256)
    t_span = np.linspace(0.0, 30.0, 10)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"])
    h32 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], lu_precision="fp32",
                        sparsity=cfg["sparsity"], **kw)
    system = oracle.System.vdp_ring(n_osc, 1.0, 0.1)
    ref, *_ = oracle.solve("rodas5P", system, cfg["y0"], t_span, cfg["params"], rtol=1e-12, atol=1e-14,
                           lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, cfg["y0"], t_span, cfg["params"], lu_precision="fp64", **kw)
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    err64 = (np.abs(o64 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    for q in (0.5, 0.9):
        assert np.quantile(err32, q) <= 1.5 * np.quantile(err64, q) + 10 * cfg["rtol"]
    assert err32.max() <= 3.0 * err64.max()


def test_decay_chain_sparse_solves_what_dense_solves():
    """tests/test_sparsity.py:110-127: a pattern changes the sweeps and the
    factorisation, not the answer; the chain's state at t = 2 is its closed form."""
    y0 = np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (64, 1))
    p = np.tile(np.array([0.7, 0.4, 0.2]), (64, 1))
    t = np.array([0.0, 0.5, 2.0])
    kw = dict(rtol=1e-11, atol=1e-13, first_step=1e-4, lu_precision="fp64")
    dense = rodas5P.solve(systems.decay_chain, y0, t, p, **kw)
    sparse = rodas5P.solve(systems.decay_chain, y0, t, p, sparsity=systems.DECAY_CHAIN_PATTERN, **kw)
    np.testing.assert_allclose(sparse, dense, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(sparse[0, -1], systems.decay_chain_exact(2.0, 0.7, 0.4, 0.2), rtol=1e-9,
                               atol=1e-11)


def test_decay_chain_gradients_survive_the_sparse_lu():
    """tests/test_sparsity.py:130-144: the gradient of sum(y(2)^2) in the rates is
    the same with and without the pattern (here by the discrete adjoint)."""
    import torch

    dev = torch.device("cuda", 0)
    y0 = torch.tensor([[1.0, 0.0, 0.0, 0.0]], dtype=torch.float64, device=dev)
    t = np.array([0.0, 2.0])
    kw = dict(rtol=1e-11, atol=1e-13, first_step=1e-4, lu_precision="fp64")

    def grad(**extra):
        p = torch.tensor([[0.7, 0.4, 0.2]], dtype=torch.float64, device=dev, requires_grad=True)
        out = rodas5P.solve(systems.decay_chain, y0, t, p, sens_error_control=False, **kw, **extra)
        (out[0, -1] ** 2).sum().backward()
        return p.grad.cpu().numpy()

    np.testing.assert_allclose(grad(sparsity=systems.DECAY_CHAIN_PATTERN), grad(), rtol=1e-9)
