"""Forward sensitivities on the GPU (the reference's gradient method) against the
oracle's joint solve and against closed forms; the error-control switch."""

import numpy as np
import pytest
import torch

from menodax_b200 import rodas5P, sensitivity
from workloads import systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["tsit5", "rodas5P"])
def test_cascade_sensitivities_match_closed_form(solver):
    a, b = 0.7, 1.3
    y0 = np.array([[2.0, 0.5]] * 3)
    t = np.linspace(0.0, 2.0, 5)
    state, sens = sensitivity.solve(solver, systems.cascade, y0, t, np.array([[a, b]] * 3),
                                    rtol=1e-10, atol=1e-12)
    sens = sens.cpu().numpy()
    k = a / (b - a)
    ea, eb = np.exp(-a * t), np.exp(-b * t)
    np.testing.assert_allclose(sens[0, :, 0, 0], ea, rtol=1e-6)
    np.testing.assert_allclose(sens[0, :, 1, 0], k * (ea - eb), rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(sens[0, :, 1, 1], eb, rtol=1e-6)
    np.testing.assert_allclose(sens[0, :, 0, 2], -t * 2.0 * ea, rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("error_control", [True, False])
def test_robertson_joint_solve_matches_oracle(oracle, error_control):
    cfg = systems.robertson_config(size=128)
    state, sens, stats = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], cfg["t_span"],
                                           cfg["params"], rtol=cfg["rtol"], atol=cfg["atol"],
                                           sens_error_control=error_control, return_stats=True)
    h, a, r, _ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"], cfg["params"],
                              rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64",
                              sens=(True, [0, 1, 2], error_control))
    same = (stats["accepted_steps"].cpu().numpy() == a) & (stats["rejected_steps"].cpu().numpy() == r)
    assert same.mean() >= 0.99
    n = 3
    osens = h[:, :, n:].reshape(h.shape[0], h.shape[1], 6, n).transpose(0, 1, 3, 2)
    gs = sens.cpu().numpy()[same]
    os_ = osens[same]
    scale = np.abs(os_).max(axis=(1, 2), keepdims=True) + 1e-300
    assert (np.abs(gs - os_) / scale).max() < 1e-7
    np.testing.assert_allclose(state.cpu().numpy()[same], h[same, :, :n], rtol=1e-9, atol=1e-15)


def test_without_error_control_the_state_matches_the_plain_solve():
    """modax/_sensitivity.py:274-292: zero weights reproduce the plain step sequence."""
    cfg = systems.robertson_config(size=256)
    plain, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                                 atol=cfg["atol"], lu_precision="fp64", return_stats=True, launch="plain")
    state, _, jstats = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"],
                                         rtol=cfg["rtol"], atol=cfg["atol"], sens_error_control=False,
                                         return_stats=True)
    assert np.array_equal(jstats["loop_steps"].cpu().numpy(), stats["loop_steps"])
    # Same step sequence; the joint kernel's state rows are compiled in a larger
    # function, so multiply-adds may contract differently: held to the parity bar.
    np.testing.assert_allclose(state.cpu().numpy(), plain, rtol=1e-9, atol=1e-18)


def test_forward_sensitivities_agree_with_the_adjoint():
    """Two ways to the same gradient: S contracted with a cotangent, and the
    discrete adjoint, on the same step sequence."""
    cfg = systems.vdp_gradient_config(1, size=16)
    t = np.linspace(0.0, 20.0, 6)
    w = np.random.default_rng(5).normal(size=(16, len(t), 2))
    _, sens = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], t, cfg["params"], rtol=1e-8,
                                atol=1e-10, sens_error_control=False)
    g_fwd = np.einsum("nsj,nsjk->nk", w, sens.cpu().numpy())
    y0 = torch.tensor(cfg["y0"], device="cuda", requires_grad=True)
    p = torch.tensor(cfg["params"], device="cuda", requires_grad=True)
    hist = rodas5P.solve(cfg["ode_fn"], y0, t, p, rtol=1e-8, atol=1e-10, lu_precision="fp64",
                         sens_error_control=False)
    (hist * torch.as_tensor(w, device="cuda")).sum().backward()
    g_adj = np.concatenate([y0.grad.cpu().numpy(), p.grad.cpu().numpy()], axis=1)
    scale = np.abs(g_fwd).max(axis=1, keepdims=True)
    assert (np.abs(g_adj - g_fwd) / scale).max() < 1e-7


def test_jvp_contracts_the_sensitivities():
    cfg = systems.robertson_config(size=8)
    dp = np.random.default_rng(6).normal(size=3)
    hist, tangent = sensitivity.jvp("rodas5P", cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"],
                                    dparams=dp, rtol=1e-8, atol=1e-12)
    _, sens = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"],
                                wrt_y0=False, rtol=1e-8, atol=1e-12)
    expect = np.einsum("nsik,k->nsi", sens.cpu().numpy(), dp)
    np.testing.assert_allclose(tangent.cpu().numpy(), expect, rtol=1e-12, atol=1e-20)


def test_joint_solve_visiting_order_changes_nothing():
    """The joint solve's persistent launch takes trajectories longest first by the
    previous call's step counts; the sensitivities are the same bit for bit as
    in index order."""
    cfg = systems.vdp_gradient_config(1, size=3000)
    t_span = np.linspace(0.0, 100.0, 11)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    sensitivity._order_hint.clear()
    first = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], **kw)
    assert len(sensitivity._order_hint) == 1
    ordered = sensitivity.solve("rodas5P", cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], **kw)
    for a, b in zip(first, ordered):
        assert torch.equal(a, b)
