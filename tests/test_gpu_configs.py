"""GPU parity on the benchmark configurations at their own sizes and horizons.

Each test takes the first trajectories of a configuration's seeded ensemble and
runs them through the layout the launch autotuner picks for that configuration
(32-state ring: one thread per trajectory, persistent launch; 128-state ring:
8-lane teams; 64-state Brusselator: thread and team kernels, dense and sparse
LUs), with FP64 LUs, against the oracle on the same colouring and elimination
order.

Two bars:

* **Strict** (FP64 parity): identical accepted/rejected counts on >= 99.9% of
  trajectories and saved states within 1e-9 relative.  Used on the Brusselator
  horizon, and on the VdP rings over the longest horizon where FP64 itself
  allows it (below).
* **Rounding noise**, for the full VdP-ring horizon (t in [0, 3000]) and the
  gradient configuration's horizon (t in [0, 1000]).  Over those horizons the
  stiff relaxation oscillators amplify a one-ulp difference into different
  accept/reject decisions: the oracle run against itself with ``y0`` changed by
  one ulp already takes different step counts on 10-20% of trajectories and
  differs by O(1) on a few.  The GPU is held to that same statistic: it must
  agree with the oracle on at least as many trajectories as the oracle agrees
  with its one-ulp-perturbed self (less a sampling margin), and its typical
  (median) trajectory difference must be of the size of the oracle's own
  rounding sensitivity.  A wrong kernel fails this by orders of magnitude.

The product path (FP32 LU, fast arithmetic) is held to accuracy instead: its
error against an FP64 oracle at rtol 1e-12 must be of the size of the FP64-LU
solve's at the same tolerance.
"""

import numpy as np
import pytest
import torch

from menodax_b200 import rodas5P
from menodax_b200._sparse_direct import sparse_lu_for
from menodax_b200._sparsity import normalize_sparsity
from workloads import systems

pytestmark = pytest.mark.gpu

ULP = 2.0 ** -52


def _bool_mask(sparsity, n):
    pairs = np.asarray(sparsity)
    if pairs.shape == (n, n):
        return pairs.astype(bool)
    mask = np.zeros((n, n), dtype=bool)
    mask[pairs[:, 0], pairs[:, 1]] = True
    return mask


def _oracle_layout(sparsity, n):
    solver = sparse_lu_for(normalize_sparsity(sparsity, n), "amd")
    return dict(sparsity_mask=_bool_mask(sparsity, n), colour=solver.slots.colour,
                order=solver.structure.order)


def _per_trajectory(a, b):
    """Each trajectory's largest relative difference over its saves and components."""
    rel = np.abs(a - b) / (np.abs(b) + 1e-12)
    return rel.reshape(len(a), -1).max(axis=1)


def _same(stats, acc, rej):
    return (np.asarray(stats["accepted_steps"]) == acc) & (np.asarray(stats["rejected_steps"]) == rej)


def _strict(hist, stats, h, a, r):
    same = _same(stats, a, r)
    assert same.mean() >= 0.999, f"step counts differ on {(~same).sum()} of {len(same)} trajectories"
    np.testing.assert_allclose(hist[same], h[same], rtol=1e-9, atol=1e-12)


def _ring_inputs(n_osc, count):
    cfg = systems.vdp_ring_config(n_osc, size=32768)
    return cfg, cfg["y0"][:count], cfg["params"][:count]


def _ring_gpu(cfg, y0, mu, t_span, team):
    return rodas5P.solve(cfg["ode_fn"], y0, t_span, mu, rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64",
                         arithmetic="reference", sparsity=cfg["sparsity"], team=team, launch="persistent",
                         return_stats=True)


def _ring_oracle(oracle, cfg, n_osc, y0, mu, t_span):
    return oracle.solve("rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), y0, t_span, mu, rtol=cfg["rtol"],
                        atol=cfg["atol"], lu_precision="fp64", **_oracle_layout(cfg["sparsity"], 2 * n_osc))


@pytest.mark.parametrize("n_osc,team,count,horizon", [
    (16, 0, 64, 300.0),   # 32 states: thread kernel
    (64, 8, 32, 100.0),   # 128 states: 8-lane teams
], ids=["ring32_thread", "ring128_team8"])
def test_vdp_ring_strict_parity(oracle, n_osc, team, count, horizon):
    """The strict FP64 bar over the longest horizon at which the oracle agrees with
    its own one-ulp-perturbed run on every trajectory (32 states: t <= 300, 128
    states: t <= 100; measured, 32-64 trajectories)."""
    cfg, y0, mu = _ring_inputs(n_osc, count)
    t_span = np.linspace(0.0, horizon, 50)
    hist, stats = _ring_gpu(cfg, y0, mu, t_span, team)
    h, a, r, _ = _ring_oracle(oracle, cfg, n_osc, y0, mu, t_span)
    same = _same(stats, a, r)
    assert same.mean() >= 0.999
    rel = np.abs(hist[same] - h[same]) / (np.abs(h[same]) + 1e-12)
    # Fast relaxation jumps (|y'| ~ mu) turn rounding-level phase differences into
    # larger value differences at the few saves that land on a jump.
    assert (rel <= 1e-9).mean() >= 0.999
    assert rel.max() <= 1e-6


def _noise_bar(gpu_err, gpu_same, noise_err, noise_same, count):
    margin = max(0.1, 3.0 / count)
    assert gpu_same.mean() >= noise_same.mean() - margin, (gpu_same.mean(), noise_same.mean())
    assert np.median(gpu_err) <= 10.0 * np.median(noise_err) + 1e-12, (np.median(gpu_err), np.median(noise_err))
    close_gpu = (gpu_err <= 1e-6).mean()
    close_noise = (noise_err <= 1e-6).mean()
    assert close_gpu >= close_noise - margin, (close_gpu, close_noise)


@pytest.mark.parametrize("n_osc,team,count", [(16, 0, 64), (64, 8, 32)], ids=["ring32_thread", "ring128_team8"])
def test_vdp_ring_full_horizon_within_rounding_noise(oracle, n_osc, team, count):
    """Configuration 3 over its whole horizon, t in [0, 3000] with 50 saves."""
    cfg, y0, mu = _ring_inputs(n_osc, count)
    t_span = cfg["t_span"]
    hist, stats = _ring_gpu(cfg, y0, mu, t_span, team)
    h, a, r, _ = _ring_oracle(oracle, cfg, n_osc, y0, mu, t_span)
    hp, ap, rp, _ = _ring_oracle(oracle, cfg, n_osc, y0 * (1.0 + ULP), mu, t_span)
    _noise_bar(_per_trajectory(hist, h), _same(stats, a, r), _per_trajectory(hp, h), (ap == a) & (rp == r), count)


@pytest.mark.parametrize("layout,team", [("sparse", 0), ("dense", 0), ("sparse", 8), ("dense", 32)],
                         ids=["thread_sparse", "thread_dense", "team8_sparse", "team32_dense"])
def test_brusselator_64_fp64_strict_parity(oracle, layout, team):
    """Configuration 4 (64 states, t in [0, 10]) with FP64 LUs against the oracle."""
    cfg = systems.brusselator_config(n_grid=32, size=16384)
    y0, b = cfg["y0"][:64], cfg["params"][:64]
    sparsity = cfg["sparsity"] if layout == "sparse" else None
    hist, stats = rodas5P.solve(cfg["ode_fn"], y0, cfg["t_span"], b, rtol=cfg["rtol"], atol=cfg["atol"],
                                lu_precision="fp64", arithmetic="reference", sparsity=sparsity, team=team,
                                launch="plain", return_stats=True)
    kw = _oracle_layout(sparsity, 64) if sparsity is not None else {}
    h, a, r, _ = oracle.solve("rodas5P", oracle.System.brusselator(32), y0, cfg["t_span"], b, rtol=cfg["rtol"],
                              atol=cfg["atol"], lu_precision="fp64", **kw)
    _strict(hist, stats, h, a, r)


def _oracle_gradient(oracle, n_osc, y0, mu, t_span, w, kw):
    system = oracle.System.vdp_ring(n_osc, 1.0, 0.1)
    h, a, r, _ = oracle.solve("rodas5P", system, y0, t_span, mu, sens=(True, [0], False), **kw)
    n = system.n
    sens = h[:, :, n:].reshape(len(y0), len(t_span), n + 1, n)
    return np.einsum("nsj,nskj->nk", w, sens), a, r


@pytest.mark.parametrize("n_osc,count", [(1, 64), (8, 32)], ids=["vdp2", "ring16"])
def test_gradient_config_full_horizon_within_rounding_noise(oracle, n_osc, count):
    """Configuration 5 over its whole horizon (20 saves on [0, 1000]): the discrete
    adjoint's gradient of sum((y - target)^2) in (y0, mu) against the oracle's
    forward sensitivities on the same step sequence, held to the oracle's own
    one-ulp sensitivity of that gradient."""
    cfg = systems.vdp_gradient_config(n_osc, size=65536)
    fn, y0, mu = cfg["ode_fn"], cfg["y0"][:count], cfg["params"][:count]
    t_span = cfg["t_span"]
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64")
    target = rodas5P.solve(fn, y0, t_span, mu * 1.05, **kw)
    y, stats = rodas5P.solve(fn, y0, t_span, mu, return_stats=True, **kw)
    w = 2.0 * (y - target)
    y0_t = torch.tensor(y0, dtype=torch.float64, device="cuda", requires_grad=True)
    p_t = torch.tensor(mu, dtype=torch.float64, device="cuda", requires_grad=True)
    out = rodas5P.solve(fn, y0_t, t_span, p_t, sens_error_control=False, **kw)
    (out * torch.as_tensor(w, device="cuda")).sum().backward()
    g = np.concatenate([y0_t.grad.cpu().numpy(), p_t.grad.cpu().numpy()], axis=1)
    og, a, r = _oracle_gradient(oracle, n_osc, y0, mu, t_span, w, kw)
    pg, ap, rp = _oracle_gradient(oracle, n_osc, y0 * (1.0 + ULP), mu, t_span, w, kw)
    scale = np.abs(og).max(axis=1)
    _noise_bar(np.abs(g - og).max(axis=1) / scale, _same(stats, a, r),
               np.abs(pg - og).max(axis=1) / scale, (ap == a) & (rp == r), count)


def test_vdp_ring_32_fp64_stage_solves_as_accurate_as_fp64(oracle):
    """The 32-state ring's thread kernel with the stage solves in FP64 against
    the widened FP32 factors (an autotuner candidate at this size) held to the
    bar of the FP32-solve test below."""
    from menodax_b200 import _native
    from menodax_b200._ensemble import launch
    from menodax_b200._problem import KernelOptions, get_problem, wide_solve

    n_osc = 16
    cfg, y0, mu = _ring_inputs(n_osc, 64)
    t_span = np.linspace(0.0, 30.0, 10)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=normalize_sparsity(cfg["sparsity"], 2 * n_osc),
                         wide_solve=True)
    assert wide_solve(opts, 2 * n_osc)
    problem = get_problem(cfg["ode_fn"], 2 * n_osc, 1, opts)
    dev = torch.device("cuda", 0)
    hist, counters = launch(problem, y0=torch.as_tensor(y0, device=dev), times=torch.as_tensor(t_span, device=dev),
                            params=torch.as_tensor(mu, device=dev), weights=None, dt0=0.0, rtol=cfg["rtol"],
                            atol=cfg["atol"], max_steps=100000, mode=_native.MDX_LAUNCH_PERSISTENT)
    h32 = hist.cpu().numpy()
    assert int(counters[3].max()) == 0
    system = oracle.System.vdp_ring(n_osc, 1.0, 0.1)
    ref, *_ = oracle.solve("rodas5P", system, y0, t_span, mu, rtol=1e-12, atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, y0, t_span, mu, rtol=cfg["rtol"], atol=cfg["atol"],
                           lu_precision="fp64")
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    err64 = (np.abs(o64 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    for q in (0.5, 0.9):
        assert np.quantile(err32, q) <= 1.5 * np.quantile(err64, q) + 10 * cfg["rtol"]
    assert err32.max() <= 3.0 * err64.max()


@pytest.mark.parametrize("n_osc,team", [(16, 0), (64, 8)], ids=["ring32_thread", "ring128_team8"])
def test_vdp_ring_fp32_lu_as_accurate_as_fp64(oracle, n_osc, team):
    """Configuration 3's product path -- FP32 LU, fast arithmetic, the autotuned
    layout -- against a tight FP64 oracle (rtol 1e-12) over a few relaxation
    cycles: each trajectory's worst error is of the size of the FP64-LU solve's at
    the same tolerance (median and 90th percentile within 1.5x + 10 rtol, the
    worst within 3x), the bar of the 8-state ring's test."""
    cfg, y0, mu = _ring_inputs(n_osc, 64)
    t_span = np.linspace(0.0, 30.0, 10)
    h32 = rodas5P.solve(cfg["ode_fn"], y0, t_span, mu, rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp32",
                        sparsity=cfg["sparsity"], team=team, launch="persistent")
    system = oracle.System.vdp_ring(n_osc, 1.0, 0.1)
    ref, *_ = oracle.solve("rodas5P", system, y0, t_span, mu, rtol=1e-12, atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, y0, t_span, mu, rtol=cfg["rtol"], atol=cfg["atol"],
                           lu_precision="fp64")
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    err64 = (np.abs(o64 - ref) / scale).reshape(len(ref), -1).max(axis=1)
    for q in (0.5, 0.9):
        assert np.quantile(err32, q) <= 1.5 * np.quantile(err64, q) + 10 * cfg["rtol"]
    assert err32.max() <= 3.0 * err64.max()


@pytest.mark.parametrize("layout,team", [("sparse", 8), ("dense", 32)], ids=["team8_sparse", "team32_dense"])
def test_brusselator_64_fp32_lu_config_horizon(oracle, layout, team):
    """Configuration 4's product path (FP32 LU, fast arithmetic, the autotuned team
    layouts) on its own inputs and horizon: within 1.5x the FP64-LU solve's error
    against the rtol 1e-12 oracle, plus 10 rtol."""
    cfg = systems.brusselator_config(n_grid=32, size=16384)
    y0, b = cfg["y0"][:64], cfg["params"][:64]
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"])
    h32 = rodas5P.solve(cfg["ode_fn"], y0, cfg["t_span"], b, lu_precision="fp32",
                        sparsity=cfg["sparsity"] if layout == "sparse" else None, team=team, launch="persistent",
                        **kw)
    ref, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), y0, cfg["t_span"], b, rtol=1e-12,
                           atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), y0, cfg["t_span"], b, lu_precision="fp64",
                           **kw)
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    assert (np.abs(h32 - ref) / scale).max() <= 1.5 * (np.abs(o64 - ref) / scale).max() + 10 * cfg["rtol"]
