"""The discrete adjoint (torch autograd over ``mdx_grad``, ``sens_error_control=False``)
against independent gradients, and the forward-sensitivity gradient the solvers take
by default (the reference's method).

* closed-form sensitivities of the linear cascade (tests/test_sensitivity.py:41-83
  in the reference),
* the oracle's forward sensitivities on the same step sequence
  (``sens_error_control=False`` semantics, modax/_sensitivity.py:274-292): the
  discrete adjoint and the discrete forward sensitivities are transposes of one
  linear map, so they agree to rounding,
* central differences of the GPU solve itself (step sizes move with the
  perturbation, so the agreement is to the solver tolerance).
"""

import numpy as np
import pytest
import torch

from menodax_b200 import rodas5P, tsit5
from workloads import systems

pytestmark = pytest.mark.gpu

A, B = 0.7, 1.3
Y0 = np.array([2.0, 0.5])
T_SPAN = np.linspace(0.0, 2.0, 5)


def cascade_exact_sens(t, y0, p):
    a, b = p
    c0, c1 = y0
    k = a / (b - a)
    dk_da = b / (b - a) ** 2
    dk_db = -a / (b - a) ** 2
    ea, eb = np.exp(-a * t), np.exp(-b * t)
    d_da = np.stack([-t * c0 * ea, c0 * (dk_da * (ea - eb) - k * t * ea)], axis=-1)
    d_db = np.stack([np.zeros_like(t), c0 * dk_db * (ea - eb) - t * (c1 - k * c0) * eb], axis=-1)
    d_dc0 = np.stack([ea, k * (ea - eb)], axis=-1)
    d_dc1 = np.stack([np.zeros_like(t), eb], axis=-1)
    return np.stack([d_dc0, d_dc1], axis=-1), np.stack([d_da, d_db], axis=-1)


def _grads(solve, fn, y0, t_span, params, w, **kw):
    y0_t = torch.tensor(y0, dtype=torch.float64, device="cuda", requires_grad=True)
    p_t = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    hist = solve(fn, y0_t, t_span, p_t, **{"sens_error_control": False, **kw})
    loss = (hist * torch.as_tensor(w, device="cuda")).sum()
    loss.backward()
    return hist.detach().cpu().numpy(), y0_t.grad.cpu().numpy(), p_t.grad.cpu().numpy()


@pytest.mark.parametrize("solve,kw", [
    (rodas5P.solve, dict(lu_precision="fp64")),
    (tsit5.solve, {}),
])
def test_cascade_gradient_matches_closed_form(solve, kw):
    n = 4
    y0 = np.broadcast_to(Y0, (n, 2)).copy()
    p = np.broadcast_to([A, B], (n, 2)).copy()
    rng = np.random.default_rng(0)
    w = rng.normal(size=(n, len(T_SPAN), 2))
    _, gy, gp = _grads(solve, systems.cascade, y0, T_SPAN, p, w, rtol=1e-10, atol=1e-12, **kw)
    sy, sp = cascade_exact_sens(T_SPAN, Y0, (A, B))
    ey = np.einsum("nsj,sjk->nk", w, sy)
    ep = np.einsum("nsj,sjk->nk", w, sp)
    np.testing.assert_allclose(gy, ey, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(gp, ep, rtol=1e-6, atol=1e-9)


def _sens_grads(oracle, solver, system, y0, t_span, params, w, **kw):
    n_vars = system.n
    hist, *_ = oracle.solve(solver, system, y0, t_span, params,
                            sens=(True, list(range(system.np)), False), **kw)
    n_sens = n_vars + system.np
    sens = hist[:, :, n_vars:].reshape(hist.shape[0], hist.shape[1], n_sens, n_vars)
    g = np.einsum("nsj,nskj->nk", w, sens)
    return hist[:, :, :n_vars], g[:, :n_vars], g[:, n_vars:]


def test_robertson_adjoint_matches_oracle_forward_sensitivities(oracle):
    cfg = systems.robertson_config(size=64)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(64, len(cfg["t_span"]), 3))
    h, gy, gp = _grads(rodas5P.solve, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], w,
                       rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    oh, oy, op = _sens_grads(oracle, "rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"],
                             cfg["params"], w, rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    np.testing.assert_allclose(h, oh, rtol=1e-9, atol=1e-15)
    scale_y = np.abs(oy).max(axis=1, keepdims=True) + 1e-300
    scale_p = np.abs(op).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(gy - oy) / scale_y).max() < 1e-7
    assert (np.abs(gp - op) / scale_p).max() < 1e-7


def test_lorenz_tsit5_adjoint_matches_oracle_forward_sensitivities(oracle):
    cfg = systems.lorenz_config(size=64)
    rng = np.random.default_rng(2)
    w = rng.normal(size=(64, len(cfg["t_span"]), 3))
    h, gy, gp = _grads(tsit5.solve, cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], w,
                       rtol=cfg["rtol"], atol=cfg["atol"])
    oh, oy, op = _sens_grads(oracle, "tsit5", oracle.System.lorenz(), cfg["y0"], cfg["t_span"],
                             cfg["params"], w, rtol=cfg["rtol"], atol=cfg["atol"])
    np.testing.assert_allclose(h, oh, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(gy, oy, rtol=1e-7, atol=1e-9 * np.abs(oy).max())
    np.testing.assert_allclose(gp, op, rtol=1e-7, atol=1e-9 * np.abs(op).max())


def test_forced_decay_gradient_uses_df_dt(oracle):
    """Non-autonomous: the df/dt term's own derivative reaches the gradient."""
    t_span = np.linspace(0.0, 1.0, 11)
    y0 = np.zeros((3, 1))
    p = np.array([[10.0, 5.0], [8.0, 3.0], [12.0, 1.0]])
    w = np.ones((3, 11, 1))
    _, gy, gp = _grads(rodas5P.solve, systems.forced_decay, y0, t_span, p, w, rtol=1e-10,
                       atol=1e-12, first_step=1e-4, lu_precision="fp64")
    _, oy, op = _sens_grads(oracle, "rodas5P", oracle.System.forced(), y0, t_span, p, w,
                            rtol=1e-10, atol=1e-12, first_step=1e-4, lu_precision="fp64")
    np.testing.assert_allclose(gp, op, rtol=1e-7)
    np.testing.assert_allclose(gy, oy, rtol=1e-7, atol=1e-12)


def test_vdp_adjoint_against_central_differences():
    cfg = systems.vdp_gradient_config(1, size=8)
    fn = cfg["ode_fn"]
    t_span = np.linspace(0.0, 10.0, 6)
    y0, p = cfg["y0"], cfg["params"] * 0 + 5.0
    rng = np.random.default_rng(3)
    w = rng.normal(size=(8, len(t_span), 2))
    kw = dict(rtol=1e-10, atol=1e-12, lu_precision="fp64")
    _, gy, gp = _grads(rodas5P.solve, fn, y0, t_span, p, w, **kw)

    def loss(y0_, p_):
        return (rodas5P.solve(fn, y0_, t_span, p_, **kw) * w).sum(axis=(1, 2))

    eps = 1e-6
    fd = (loss(y0, p * (1 + eps)) - loss(y0, p * (1 - eps))) / (2 * eps * p[:, 0])
    np.testing.assert_allclose(gp[:, 0], fd, rtol=1e-4)
    for j in range(2):
        dy = np.zeros_like(y0)
        dy[:, j] = eps
        fd = (loss(y0 + dy, p) - loss(y0 - dy, p)) / (2 * eps)
        np.testing.assert_allclose(gy[:, j], fd, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("solve,kw,which", [
    (rodas5P.solve, dict(lu_precision="fp64"), "vdp"),
    (tsit5.solve, {}, "lorenz"),
])
def test_segmented_checkpoints_give_the_same_gradient(monkeypatch, solve, kw, which):
    """Recording a start state every 8 steps and replaying the segments gives the
    gradient of recording every step."""
    from menodax_b200 import autograd

    if which == "vdp":
        cfg = systems.vdp_gradient_config(1, size=32)
        t_span = np.linspace(0.0, 50.0, 7)
    else:
        cfg = systems.lorenz_config(size=32)
        t_span = cfg["t_span"]
    n_vars = cfg["y0"].shape[1]
    w = np.random.default_rng(4).normal(size=(32, len(t_span), n_vars))
    out = []
    for strides in ((1,), (8,)):
        monkeypatch.setattr(autograd, "CKPT_STRIDES", strides)
        autograd._capacity_hint.clear()
        out.append(_grads(solve, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], w, rtol=1e-6,
                          atol=1e-8, **kw))
    (h1, gy1, gp1), (h8, gy8, gp8) = out
    assert np.array_equal(h1, h8)
    np.testing.assert_allclose(gy8, gy1, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(gp8, gp1, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("lu_precision", ["fp64", "fp32"])
def test_sparse_lu_adjoint_matches_dense(lu_precision):
    """The reverse sweep's transposed solves run on the structure-compiled sparse LU
    when the solve has a sparsity pattern; on the VdP ring the gradient matches the
    dense-LU gradient (FP64: to rounding of the different elimination order; FP32:
    to the FP32 LU's accuracy)."""
    cfg = systems.vdp_gradient_config(3, size=32)
    t_span = np.linspace(0.0, 5.0, 6)
    y0, p = cfg["y0"], cfg["params"]
    w = np.random.default_rng(5).normal(size=(32, len(t_span), 6))
    kw = dict(rtol=1e-8, atol=1e-10, lu_precision=lu_precision)
    hd, gyd, gpd = _grads(rodas5P.solve, cfg["ode_fn"], y0, t_span, p, w, **kw)
    hs, gys, gps = _grads(rodas5P.solve, cfg["ode_fn"], y0, t_span, p, w, sparsity=systems.vdp_sparsity(3), **kw)
    tol = 1e-7 if lu_precision == "fp64" else 1e-3
    np.testing.assert_allclose(hs, hd, rtol=tol, atol=1e-9)
    np.testing.assert_allclose(gys, gyd, rtol=tol, atol=tol * np.abs(gyd).max())
    np.testing.assert_allclose(gps, gpd, rtol=tol, atol=tol * np.abs(gpd).max())


@pytest.mark.parametrize("n_osc", [1, 3])
def test_vdp_gradient_config_matches_oracle_forward_sensitivities(oracle, n_osc):
    """The stiff Van der Pol gradient workload's system and loss: sum((y - target)^2) over the saves, targets
    from mu * 1.05, y0 and mu differentiated.  The discrete adjoint of the solve
    equals the oracle's forward sensitivities on the same step sequence (the
    reference's sens_error_control=False), within 1e-5 relative."""
    cfg = systems.vdp_gradient_config(n_osc, size=64)
    t_span = np.linspace(0.0, 20.0, 6)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    fn, y0, mu = cfg["ode_fn"], cfg["y0"], cfg["params"]
    target = rodas5P.solve(fn, y0, t_span, mu * 1.05, **kw)
    y = rodas5P.solve(fn, y0, t_span, mu, **kw)
    w = 2.0 * (y - target)  # d loss / d hist
    h, gy, gp = _grads(rodas5P.solve, fn, y0, t_span, mu, w, **kw)
    oh, oy, op = _sens_grads(oracle, "rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), y0, t_span, mu, w,
                             **kw)
    np.testing.assert_allclose(h, oh, rtol=1e-9, atol=1e-12)
    scale_y = np.abs(oy).max(axis=1, keepdims=True) + 1e-300
    scale_p = np.abs(op).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(gy - oy) / scale_y).max() < 1e-5
    assert (np.abs(gp - op) / scale_p).max() < 1e-5


def test_fp32_lu_adjoint_agrees_with_fp64_on_a_short_horizon():
    """The FP32-LU adjoint (fast arithmetic) differentiates its own, slightly
    different solution; over a few relaxation cycles of the 2-state stiff Van der Pol system the two
    gradients agree to 1e-4 (median) -- over t in [0, 1000] the loss amplifies the
    rtol-level solution differences into gradient differences of several percent,
    for any two solves that take different steps."""
    import torch

    cfg = systems.vdp_gradient_config(1, size=1024)
    t_span = np.linspace(0.0, 20.0, 20)
    y0 = torch.as_tensor(cfg["y0"], device="cuda")
    mu = torch.as_tensor(cfg["params"], device="cuda")
    with torch.no_grad():
        target = rodas5P.solve(cfg["ode_fn"], y0, t_span, mu * 1.05, rtol=1e-6, atol=1e-8, lu_precision="fp64")
    grads = {}
    for prec in ("fp64", "fp32"):
        y0_t = y0.clone().requires_grad_(True)
        p_t = mu.clone().requires_grad_(True)
        h = rodas5P.solve(cfg["ode_fn"], y0_t, t_span, p_t, rtol=1e-6, atol=1e-8, lu_precision=prec,
                          sens_error_control=False)
        ((h - target) ** 2).sum().backward()
        grads[prec] = torch.cat([y0_t.grad, p_t.grad], dim=1)
    g64, g32 = grads["fp64"], grads["fp32"]
    rel = (g32 - g64).abs().max(dim=1).values / g64.abs().max(dim=1).values
    assert float(rel.median()) < 1e-4
    assert float(rel.quantile(0.9)) < 1e-3


@pytest.mark.parametrize("solve,system,kw", [
    (rodas5P.solve, "robertson", dict(lu_precision="fp64")),
    (tsit5.solve, "lorenz", {}),
])
def test_default_gradient_is_the_references_forward_sensitivities(oracle, solve, system, kw):
    """With sens_error_control left at True (the reference's default) the gradient is
    the forward-sensitivity one with the sensitivities under error control: the
    oracle's joint solve under error control, contracted with the cotangent."""
    cfg = getattr(systems, f"{system}_config")(size=32)
    w = np.random.default_rng(7).normal(size=(32, len(cfg["t_span"]), 3))
    y0_t = torch.tensor(cfg["y0"], dtype=torch.float64, device="cuda", requires_grad=True)
    p_t = torch.tensor(cfg["params"], dtype=torch.float64, device="cuda", requires_grad=True)
    hist = solve(cfg["ode_fn"], y0_t, cfg["t_span"], p_t, rtol=cfg["rtol"], atol=cfg["atol"], **kw)
    (hist * torch.as_tensor(w, device="cuda")).sum().backward()
    sys_ = getattr(oracle.System, system)()
    oh, *_ = oracle.solve("rodas5P" if solve is rodas5P.solve else "tsit5", sys_, cfg["y0"], cfg["t_span"],
                          cfg["params"], rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64",
                          sens=(True, list(range(sys_.np)), True))
    n = sys_.n
    sens = oh[:, :, n:].reshape(32, len(cfg["t_span"]), n + sys_.np, n)
    g = np.einsum("nsj,nskj->nk", w, sens)
    np.testing.assert_allclose(hist.detach().cpu().numpy(), oh[:, :, :n], rtol=1e-9, atol=1e-14)
    scale = np.abs(g).max(axis=1, keepdims=True)
    got = np.concatenate([y0_t.grad.cpu().numpy(), p_t.grad.cpu().numpy()], axis=1)
    assert (np.abs(got - g) / scale).max() < 1e-7


@pytest.mark.parametrize("error_control", [True, False])
def test_sens_param_columns_zero_the_other_columns(error_control):
    """Only the listed parameter columns are differentiated; the rest get zeros, and
    the listed ones match the full gradient's: exactly for the adjoint (the same
    step sequence), to the solver tolerance under error control, where carrying
    fewer sensitivity columns changes the error norm and so the steps."""
    cfg = systems.robertson_config(size=16)
    w = np.random.default_rng(8).normal(size=(16, len(cfg["t_span"]), 3))
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64", sens_error_control=error_control)

    def grad(columns):
        p_t = torch.tensor(cfg["params"], dtype=torch.float64, device="cuda", requires_grad=True)
        hist = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], p_t, sens_param_columns=columns, **kw)
        (hist * torch.as_tensor(w, device="cuda")).sum().backward()
        return p_t.grad.cpu().numpy()

    full, some = grad(None), grad([2, 0])
    assert (some[:, 1] == 0.0).all()
    tol = 1e-5 if error_control else 1e-9
    np.testing.assert_allclose(some[:, [0, 2]], full[:, [0, 2]], rtol=tol, atol=tol * 1e-3 * np.abs(full).max())


@pytest.mark.parametrize("n_osc", [3, 8])
def test_team_adjoint_matches_the_thread_adjoint(n_osc):
    """The team kernels' checkpointing forward pass and reverse sweep (a team of 8
    lanes per trajectory, its vectors in shared memory) give the thread kernels'
    gradient on the VdP ring with its sparse LU: the same step sequence and
    arithmetic, so to rounding."""
    cfg = systems.vdp_gradient_config(n_osc, size=64)
    t_span = np.linspace(0.0, 20.0, 6)
    w = np.random.default_rng(10).normal(size=(64, len(t_span), 2 * n_osc))
    kw = dict(rtol=1e-6, atol=1e-8, lu_precision="fp64", sparsity=systems.vdp_sparsity(n_osc))
    h0, gy0, gp0 = _grads(rodas5P.solve, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], w, team=0, **kw)
    h8, gy8, gp8 = _grads(rodas5P.solve, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], w, team=8, **kw)
    np.testing.assert_allclose(h8, h0, rtol=1e-9, atol=1e-12)
    for got, ref in ((gy8, gy0), (gp8, gp0)):
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(got - ref) / scale).max() < 1e-7


@pytest.mark.parametrize("solve,n_osc,kw", [
    (rodas5P.solve, 1, dict(lu_precision="fp64")),
    (rodas5P.solve, 3, dict(lu_precision="fp32", sparsity=systems.vdp_sparsity(3))),
    (tsit5.solve, None, {}),
], ids=["vdp2_fp64", "ring6_fp32_sparse", "lorenz_tsit5"])
def test_split_reverse_gives_the_whole_reverse(monkeypatch, solve, n_osc, kw):
    """The reverse pass with long trajectories cut into chunks (transfer matrices
    from unit cotangents, offsets from the injected ones, composed afterwards)
    equals the one-sweep-per-trajectory reverse to rounding; cut at half the mean
    length, most trajectories are split."""
    from menodax_b200 import autograd

    if n_osc is None:
        cfg = systems.lorenz_config(size=512)
        t_span, fn, y0, p = cfg["t_span"], cfg["ode_fn"], cfg["y0"], cfg["params"]
        kw = dict(kw, rtol=cfg["rtol"], atol=cfg["atol"])
    else:
        cfg = systems.vdp_gradient_config(n_osc, size=512)
        t_span, fn, y0, p = np.linspace(0.0, 50.0, 11), cfg["ode_fn"], cfg["y0"], cfg["params"]
        kw = dict(kw, rtol=cfg["rtol"], atol=cfg["atol"])
    w = np.random.default_rng(13).normal(size=(512, len(t_span), y0.shape[1]))
    monkeypatch.setattr(autograd, "REVERSE_SPLIT", None)
    h0, gy0, gp0 = _grads(solve, fn, y0, t_span, p, w, **kw)
    assert autograd.last_checkpoint["split_tasks"] == 0
    monkeypatch.setattr(autograd, "REVERSE_SPLIT", 0.5)
    h1, gy1, gp1 = _grads(solve, fn, y0, t_span, p, w, **kw)
    assert autograd.last_checkpoint["split_trajectories"] > 100
    assert np.array_equal(h0, h1)
    for a, b in ((gy0, gy1), (gp0, gp1)):
        scale = np.abs(a).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(a - b) / scale).max() < 1e-9


def test_forward_visiting_order_changes_nothing_but_the_schedule():
    """The checkpointing forward launch takes trajectories longest first (the last
    call's step counts); each trajectory's integration, and so the gradient, is
    the same bit for bit in any order."""
    from menodax_b200 import autograd

    cfg = systems.vdp_gradient_config(1, size=2048)
    t_span = np.linspace(0.0, 100.0, 11)
    w = np.random.default_rng(17).normal(size=(2048, len(t_span), 2))
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    autograd._capacity_hint.clear()
    autograd._order_hint.clear()
    ordered = _grads(rodas5P.solve, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], w, **kw)
    assert len(autograd._order_hint) == 1
    autograd._order_hint.clear()
    plain = _grads(rodas5P.solve, cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], w, **kw)
    for a, b in zip(ordered, plain):
        assert np.array_equal(a, b)
