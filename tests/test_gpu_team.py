"""The team kernel (several lanes per trajectory, state and matrix in shared memory).

Held to the bars of the thread kernel it stands in for: against the oracle on
the same colouring and elimination order with FP64 LUs (identical step counts on
99.9% of trajectories, saved states within 1e-9), and against a tight FP64
oracle with FP32 LUs.  The persistent team launch must reproduce the plain one
bit for bit (the queue only changes which team runs a trajectory).
"""

import math

import numpy as np
import pytest

from menodax_b200 import rodas5P
from workloads import systems
from menodax_b200._sparse_direct import sparse_lu_for
from menodax_b200._sparsity import normalize_sparsity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("team", [4, 8, 32])
@pytest.mark.parametrize("layout", ["sparse", "dense"])
def test_team_vdp_ring_fp64_matches_oracle(oracle, team, layout):
    n_osc = 4
    cfg = systems.vdp_ring_config(n_osc, size=512)
    t_span = np.linspace(0.0, 30.0, 20)
    mask = cfg["sparsity"] if layout == "sparse" else None
    hist, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], rtol=1e-6, atol=1e-8,
                                lu_precision="fp64", sparsity=mask, team=team, launch="plain",
                                return_stats=True)
    kw = {}
    if mask is not None:
        solver = sparse_lu_for(normalize_sparsity(mask, 2 * n_osc), "amd")
        kw = dict(sparsity_mask=mask, colour=solver.slots.colour, order=solver.structure.order)
    h, a, r, _ = oracle.solve("rodas5P", oracle.System.vdp_ring(n_osc, 1.0, 0.1), cfg["y0"], t_span,
                              cfg["params"], rtol=1e-6, atol=1e-8, lu_precision="fp64", **kw)
    same = (np.asarray(stats["accepted_steps"]) == a) & (np.asarray(stats["rejected_steps"]) == r)
    assert same.mean() >= 0.999
    np.testing.assert_allclose(hist[same], h[same], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("team", [8, 16, 32])
@pytest.mark.parametrize("layout", ["sparse", "dense"])
def test_team_brusselator_64_fp32_as_accurate_as_fp64(oracle, team, layout):
    cfg = systems.brusselator_config(n_grid=32, size=128)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"])
    mask = cfg["sparsity"] if layout == "sparse" else None
    h32 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], lu_precision="fp32",
                        sparsity=mask, team=team, **kw)
    ref, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), cfg["y0"], cfg["t_span"],
                           cfg["params"], rtol=1e-12, atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", oracle.System.brusselator(32), cfg["y0"], cfg["t_span"],
                           cfg["params"], lu_precision="fp64", **kw)
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).max()
    err64 = (np.abs(o64 - ref) / scale).max()
    assert err32 <= 1.5 * err64 + 10 * cfg["rtol"]


@pytest.mark.parametrize("n_grid,team", [(15, 8), (12, 16)])
def test_team_dense_fp32_panels_as_accurate_as_fp64(oracle, n_grid, team):
    """The fast dense LU's four-column panels (each lane's pivot-row entries in
    registers): 30 states on 8 lanes end on a two-column panel, 24 on 16 lanes
    divide evenly."""
    cfg = systems.brusselator_config(n_grid=n_grid, size=128)
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"])
    h32 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], lu_precision="fp32",
                        team=team, launch="plain", **kw)
    system = oracle.System.brusselator(n_grid)
    ref, *_ = oracle.solve("rodas5P", system, cfg["y0"], cfg["t_span"], cfg["params"], rtol=1e-12,
                           atol=1e-14, lu_precision="fp64")
    o64, *_ = oracle.solve("rodas5P", system, cfg["y0"], cfg["t_span"], cfg["params"], lu_precision="fp64",
                           **kw)
    scale = np.abs(ref) + cfg["atol"] / cfg["rtol"]
    err32 = (np.abs(h32 - ref) / scale).max()
    err64 = (np.abs(o64 - ref) / scale).max()
    assert err32 <= 1.5 * err64 + 10 * cfg["rtol"]


@pytest.mark.parametrize("n_osc", [5, 6])
def test_team_dense_panels_factor_like_the_thread_kernel(n_osc):
    """Fast arithmetic in FP64: the thread kernel's register LU and the team's
    four-column panels (4 lanes: 10 states end on a two-column panel, 12 divide
    evenly) apply the same operations to every entry in the same order, so the
    factorisations agree bit for bit and only the substitutions' summation order
    differs (measured: at most 1.6e-10 apart on O(1) states, a handful of entries
    in 1e5 above 1e-9 relative).  A missed or misordered update would put the two
    runs rtol apart."""
    cfg = systems.vdp_ring_config(n_osc, size=512)
    t_span = np.linspace(0.0, 30.0, 20)
    kw = dict(rtol=1e-6, atol=1e-8, lu_precision="fp64", arithmetic="fast", launch="plain",
              return_stats=True)
    h0, s0 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], team=0, **kw)
    h4, s4 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], team=4, **kw)
    same = np.asarray(s0["loop_steps"]) == np.asarray(s4["loop_steps"])
    assert same.mean() >= 0.999
    np.testing.assert_allclose(h4[same], h0[same], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("team", [4, 16])
def test_team_persistent_equals_plain(team):
    cfg = systems.vdp_ring_config(16, size=600)
    t_span = np.linspace(0.0, 20.0, 5)
    kw = dict(rtol=1e-6, atol=1e-8, lu_precision="fp32", sparsity=cfg["sparsity"], team=team,
              return_stats=True)
    h1, s1 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], launch="plain", **kw)
    h2, s2 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], launch="persistent", **kw)
    assert np.array_equal(h1, h2)
    assert np.array_equal(s1["loop_steps"], s2["loop_steps"])


def test_team_robertson_fp64_matches_thread_kernel():
    """A system with no repeated structure (every component its own class)."""
    cfg = systems.robertson_config(size=256)
    kw = dict(rtol=1e-6, atol=1e-10, lu_precision="fp64", return_stats=True)
    h0, s0 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], team=0, **kw)
    h4, s4 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], team=4, **kw)
    same = np.asarray(s0["loop_steps"]) == np.asarray(s4["loop_steps"])
    assert same.mean() >= 0.999
    np.testing.assert_allclose(h4[same], h0[same], rtol=1e-9, atol=1e-14)


def test_team_stats_and_max_steps_status():
    cfg = systems.vdp_ring_config(4, size=64)
    _, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=1e-6, atol=1e-8,
                             sparsity=cfg["sparsity"], team=8, max_steps=50, return_stats=True)
    assert (np.asarray(stats["loop_steps"]) == 50).all()
    assert (np.asarray(stats["status"]) & 1).all()


def test_team_tf_index_and_time_derivative():
    """The reference's tests/test_solver_options.py:40-93 cases on the team kernel:
    df/dt reaches the stages of a non-autonomous system, and tf_index ends each
    trajectory at its own time with the later saves frozen."""
    t_span = np.linspace(0.0, 1.0, 11)
    params = np.array([[10.0, 5.0, 1.0], [10.0, 5.0, 0.5]])
    out = rodas5P.solve(systems.forced_decay, np.zeros((2, 1)), t_span, params, tf_index=2, rtol=1e-10,
                        atol=1e-12, first_step=1e-4, lu_precision="fp64", team=4)
    exact = 5.0 * (10.0 * t_span - 1.0 + np.exp(-10.0 * t_span)) / 100.0
    np.testing.assert_allclose(out[0, :, 0], exact, rtol=1e-8, atol=1e-10)
    stops = int(np.searchsorted(t_span, 0.5, side="right"))
    np.testing.assert_allclose(out[1, :stops, 0], exact[:stops], rtol=1e-8, atol=1e-10)
    assert (out[1, stops:, 0] == out[1, stops - 1, 0]).all()


def _forced_ring(y, t, p):
    n = 12
    return tuple(-p[0] * y[i] + 0.3 * (y[(i + 1) % n] - y[i]) + math.sin(t + 0.5 * i) for i in range(n))


@pytest.mark.parametrize("layout", ["sparse", "dense"])
def test_team_non_autonomous_ring_matches_thread_kernel(layout):
    n = 12
    rng = np.random.default_rng(11)
    y0 = rng.uniform(-1.0, 1.0, size=(300, n))
    p = rng.uniform(0.5, 2.0, size=(300, 1))
    t_span = np.linspace(0.0, 5.0, 9)
    pattern = [(i, i) for i in range(n)] + [(i, (i + 1) % n) for i in range(n)] if layout == "sparse" else None
    kw = dict(rtol=1e-9, atol=1e-11, lu_precision="fp64", sparsity=pattern, return_stats=True)
    h0, s0 = rodas5P.solve(_forced_ring, y0, t_span, p, team=0, **kw)
    h8, s8 = rodas5P.solve(_forced_ring, y0, t_span, p, team=8, **kw)
    same = np.asarray(s0["loop_steps"]) == np.asarray(s8["loop_steps"])
    assert same.mean() >= 0.999
    np.testing.assert_allclose(h8[same], h0[same], rtol=1e-9, atol=1e-12)


def test_team_error_weights_match_thread_kernel():
    cfg = systems.robertson_config(size=256)
    w = np.array([1.0, 0.0, 1.0])
    kw = dict(rtol=cfg["rtol"], atol=cfg["atol"], lu_precision="fp64", error_weights=w, return_stats=True)
    h0, s0 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], team=0, **kw)
    h4, s4 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], team=4, **kw)
    same = np.asarray(s0["loop_steps"]) == np.asarray(s4["loop_steps"])
    assert same.mean() >= 0.98
    # As against the oracle: the zero-weight component's undamped rounding
    # differences reach the controlled ones through the dynamics.
    np.testing.assert_allclose(h4[same][..., [0, 2]], h0[same][..., [0, 2]], rtol=5e-7, atol=1e-15)
