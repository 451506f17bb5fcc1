"""The CPU oracle pinned against the reference's own published results.

Every number here is read from the reference's benchmark CSVs (GPU runs of the
reference kernels) or its closed-form tests; the oracle must reproduce them
before it is trusted as the parity checker.
"""

import numpy as np
import pytest

from workloads import systems


def test_lorenz_tsit5_golden_steps(oracle):
    """722 attempted / 104 rejected: benchmarks/nonstiff_lorenz_divergence CSV row 2."""
    y0, p = systems.lorenz_divergence_scenario(4, divergence=0.0)
    _, acc, rej, loop = oracle.solve("tsit5", oracle.System.lorenz(), y0, (0.0, 5.0), p,
                                     rtol=1e-6, atol=1e-8, first_step=1e-4)
    assert (loop == 722).all() and (rej == 104).all()


def test_lorenz_tsit5_divergence_distribution(oracle):
    """Divergence 0.1, 100,000 trajectories: mean 699.81274, min 664, max 735,
    rejected mean 102.78706 (same CSV, row 3)."""
    y0, p = systems.lorenz_divergence_scenario(100_000, divergence=0.1)
    _, _, rej, loop = oracle.solve("tsit5", oracle.System.lorenz(), y0, (0.0, 5.0), p,
                                   rtol=1e-6, atol=1e-8, first_step=1e-4)
    assert loop.mean() == pytest.approx(699.81274, abs=1e-9)
    assert loop.min() == 664 and loop.max() == 735
    assert rej.mean() == pytest.approx(102.78706, abs=1e-9)


def test_vdp64_tsit5_golden_distribution(oracle):
    """Non-stiff 64-D VdP: 12/0 at divergence 0; divergence 0.25, N=1000: mean 27.109,
    min 24, max 31, rejected 1.161 (benchmarks/nonstiff_vdp_divergence CSV rows 2-3)."""
    system = oracle.System.vdp_ring(32, 1.0, 10.0)
    y0, p = systems.vdp_divergence_scenario(32, 4, divergence=0.0)
    _, _, rej, loop = oracle.solve("tsit5", system, y0, systems.VDP_TIMES, p, rtol=1e-6, atol=1e-8,
                                   first_step=1e-4)
    assert (loop == 12).all() and (rej == 0).all()
    y0, p = systems.vdp_divergence_scenario(32, 1000, divergence=0.25)
    _, _, rej, loop = oracle.solve("tsit5", system, y0, systems.VDP_TIMES, p, rtol=1e-6, atol=1e-8,
                                   first_step=1e-4)
    assert loop.mean() == pytest.approx(27.109, abs=1e-9)
    assert (loop.min(), loop.max()) == (24, 31)
    assert rej.mean() == pytest.approx(1.161, abs=1e-9)


def test_robertson_rodas5p_fp32_golden_steps(oracle):
    """157 attempted / 10 rejected with an FP32 LU (benchmarks/stiff_robertson_divergence
    CSV row 2).  The reference's GPU compiler contracts multiply-adds; the oracle is
    built the same way where the host has FMA, and lands one rejection short without."""
    _, _, rej, loop = oracle.solve("rodas5P", oracle.System.robertson(), systems.ROBERTSON_Y0,
                                   systems.ROBERTSON_TIMES, systems.ROBERTSON_PARAMS, rtol=1e-6,
                                   atol=1e-8, first_step=1e-4, lu_precision="fp32")
    if oracle.FMA:
        assert (int(loop[0]), int(rej[0])) == (157, 10)
    else:
        assert abs(int(loop[0]) - 157) <= 1 and abs(int(rej[0]) - 10) <= 1


def test_vdp96_rodas5p_fp32_golden_steps(oracle):
    """Stiff 96-D VdP (mu=100, d=10), FP32 LU, divergence 0: 21 attempted / 0 rejected
    (benchmarks/stiff_vdp_divergence CSV row 2)."""
    y0, p = systems.vdp_divergence_scenario(48, 2, divergence=0.0)
    _, _, rej, loop = oracle.solve("rodas5P", oracle.System.vdp_ring(48, 100.0, 10.0), y0,
                                   systems.VDP_TIMES, p, rtol=1e-6, atol=1e-8, first_step=1e-4,
                                   lu_precision="fp32")
    assert (loop == 21).all() and (rej == 0).all()


def test_robertson_mass_is_conserved(oracle):
    """tests/benchmark_helpers.py:160-162: the three species sum to one."""
    cfg = systems.robertson_config(size=64)
    hist, *_ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"],
                            cfg["params"], rtol=1e-8, atol=1e-12, lu_precision="fp64")
    np.testing.assert_allclose(hist.sum(axis=-1), 1.0, atol=1e-8)


def test_forced_decay_closed_form(oracle):
    """tests/test_solver_options.py:40-63: df/dt reaches the stages."""
    t = np.linspace(0.0, 1.0, 11)
    hist, *_ = oracle.solve("rodas5P", oracle.System.forced(), np.zeros((1, 1)), t,
                            np.array([[10.0, 5.0]]), rtol=1e-10, atol=1e-12, first_step=1e-4,
                            lu_precision="fp64")
    exact = 5.0 * (10.0 * t - 1.0 + np.exp(-10.0 * t)) / 100.0
    np.testing.assert_allclose(hist[0, :, 0], exact, rtol=1e-8, atol=1e-10)


def test_tf_index_freezes_saves(oracle):
    """tests/test_solver_options.py:66-93: saves past a trajectory's end hold its state."""
    t = np.linspace(0.0, 1.0, 11)
    p = np.array([[10.0, 5.0, 1.0], [10.0, 5.0, 0.5]])
    system = oracle.System.callback(systems.forced_decay, 1, 3)
    hist, *_ = oracle.solve("rodas5P", system, np.zeros((2, 1)), t, p, rtol=1e-10, atol=1e-12,
                            first_step=1e-4, lu_precision="fp64", tf_index=2)
    stops = int(np.searchsorted(t, 0.5, side="right"))
    assert (hist[1, stops:, 0] == hist[1, stops - 1, 0]).all()
    np.testing.assert_allclose(hist[0, :, 0], 5.0 * (10.0 * t - 1.0 + np.exp(-10.0 * t)) / 100.0,
                               rtol=1e-8, atol=1e-10)


def test_callback_system_matches_builtin(oracle):
    """The dual-number callback path and the C++ template path agree."""
    cfg = systems.robertson_config(size=4)
    a, *_ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"],
                         cfg["params"], rtol=1e-6, atol=1e-10, lu_precision="fp64")
    b, *_ = oracle.solve("rodas5P", oracle.System.callback(systems.robertson, 3, 3), cfg["y0"],
                         cfg["t_span"], cfg["params"], rtol=1e-6, atol=1e-10, lu_precision="fp64")
    np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-15)


def test_a_raising_callback_fails_the_oracle_call(oracle):
    """An exception inside a Python callback is recorded and raised after the call,
    never swallowed with the output left undefined."""
    calls = [0]

    def broken(y, t, p):
        calls[0] += 1
        if calls[0] > 20:
            raise ZeroDivisionError("planted")
        return (-p[0] * y[0],)

    with pytest.raises(RuntimeError, match="planted"):
        oracle.solve("rodas5P", oracle.System.callback(broken, 1, 1), np.ones((2, 1)),
                     np.linspace(0.0, 1.0, 3), np.ones((2, 1)), lu_precision="fp64", max_steps=50)


@pytest.mark.parametrize("solver", ["tsit5", "rodas5P"])
def test_forward_sensitivities_match_closed_form_cascade(oracle, solver):
    """tests/test_sensitivity.py:42-83, 165-191: jacfwd of the cascade to rtol 1e-6."""
    a, b = 0.7, 1.3
    y0 = np.array([[2.0, 0.5]])
    t = np.linspace(0.0, 2.0, 5)
    hist, *_ = oracle.solve(solver, oracle.System.cascade(), y0, t, np.array([[a, b]]), rtol=1e-10,
                            atol=1e-12, lu_precision="fp64", sens=(True, [0, 1], True))
    sens = hist[0, :, 2:].reshape(len(t), 4, 2)  # (s, direction, row)
    k = a / (b - a)
    ea, eb = np.exp(-a * t), np.exp(-b * t)
    np.testing.assert_allclose(sens[:, 0, 0], ea, rtol=1e-6)
    np.testing.assert_allclose(sens[:, 0, 1], k * (ea - eb), rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(sens[:, 2, 0], -t * 2.0 * ea, rtol=1e-6, atol=1e-12)


def _scipy_solve(fn, y0, times, params, method):
    from scipy.integrate import solve_ivp

    rows = []
    for y, p in zip(y0, params):
        sol = solve_ivp(lambda t, u: np.array(fn(u, t, p), dtype=float), (times[0], times[-1]), y,
                        method=method, t_eval=times, rtol=1e-12, atol=1e-14)
        assert sol.success, sol.message
        rows.append(sol.y.T)
    return np.array(rows)


def _xcheck_cases(oracle):
    lorenz = systems.lorenz_config(size=4)
    robertson = systems.robertson_config(size=4)
    ring = systems.vdp_ring_config(4, size=4)
    ring["t_span"] = np.linspace(0.0, 30.0, 10)
    bruss = systems.brusselator_config(n_grid=8, size=4)
    return {
        "lorenz": ("tsit5", oracle.System.lorenz(), lorenz, "DOP853"),
        "robertson": ("rodas5P", oracle.System.robertson(), robertson, "Radau"),
        "vdp_ring": ("rodas5P", oracle.System.vdp_ring(4, 1.0, 0.1), ring, "Radau"),
        "brusselator": ("rodas5P", oracle.System.brusselator(8), bruss, "Radau"),
    }


@pytest.mark.parametrize("name", ["lorenz", "robertson", "vdp_ring", "brusselator"])
def test_oracle_agrees_with_scipy(oracle, name):
    """An independent check of the oracle's integrators: its FP64 Tsit5 / Rodas5P
    at rtol 1e-12 against scipy's solve_ivp (DOP853 for the non-stiff Lorenz
    system, Radau for the stiff ones) at the same tolerance, on four trajectories
    of each configuration's inputs.  Measured agreement: 4e-11 absolute on Lorenz,
    8e-12 on Robertson (whose smallest component is ~1e-8), 4e-13 on the VdP ring,
    2e-11 on the Brusselator."""
    solver, system, cfg, method = _xcheck_cases(oracle)[name]
    y0 = np.asarray(cfg["y0"], dtype=float)
    params = np.asarray(cfg["params"], dtype=float)
    times = np.asarray(cfg["t_span"], dtype=float)
    kw = dict(lu_precision="fp64") if solver == "rodas5P" else {}
    hist, *_ = oracle.solve(solver, system, y0, times, params, rtol=1e-12, atol=1e-14, **kw)
    ref = _scipy_solve(cfg["ode_fn"], y0, times, params, method)
    np.testing.assert_allclose(hist, ref, rtol=1e-8, atol=1e-10)


def _closed_form_case(name):
    """(ode_fn, n_vars, y0, times, exact(params)) of the reference's closed-form systems."""
    if name.startswith("bateman"):
        n = int(name[len("bateman"):])
        fn, y0, m = systems.make_bateman_system(n, 1e2 if n <= 4 else 1e4)
        return fn, n, y0, systems.BATEMAN_TIMES, lambda p: systems.linear_exact(m, y0, systems.BATEMAN_TIMES, p)
    if name.startswith("heat"):
        n = int(name[len("heat"):])
        fn, y0 = systems.make_heat_system(n)
        return fn, n, y0, systems.HEAT_TIMES, lambda p: systems.heat_exact(n, systems.HEAT_TIMES, p)
    pairs = int(name[len("kaps"):])
    fn, y0 = systems.make_kaps_system(pairs, 1e-2 if pairs <= 2 else 1e-6)
    return fn, 2 * pairs, y0, systems.KAPS_TIMES, lambda p: systems.kaps_exact(systems.KAPS_TIMES, p, pairs)


@pytest.mark.parametrize("solver,name", [("rodas5P", "bateman16"), ("rodas5P", "heat32"), ("rodas5P", "kaps4"),
                                         ("tsit5", "bateman4"), ("tsit5", "heat4"), ("tsit5", "kaps2")])
def test_oracle_matches_closed_forms(oracle, solver, name):
    """The reference's closed-form systems (reference/systems/python/bateman.py,
    heat.py, kaps.py: a stiff decay chain, the heat equation's first eigenmode,
    Kaps' singular perturbation) at rtol 1e-10: the oracle lands within 1e-10 of
    the exact solution (measured 2e-12 to 1.4e-11)."""
    fn, n, y0, times, exact = _closed_form_case(name)
    params = systems.rate_scale_params(4)
    y = np.broadcast_to(y0, (4, n)).copy()
    kw = dict(lu_precision="fp64") if solver == "rodas5P" else {}
    hist, *_ = oracle.solve(solver, oracle.System.callback(fn, n, 1), y, times, params, rtol=1e-10,
                            atol=1e-14, **kw)
    np.testing.assert_allclose(hist, exact(params), rtol=1e-8, atol=1e-10)


def test_scipy_ensemble_baseline_solves_the_same_problem(oracle):
    """The restated scipy_solve_ivp ensemble (the reference's CPU baseline) on a few
    Robertson trajectories: LSODA at rtol 1e-8 lands near the rtol 1e-12 oracle."""
    from oracle import scipy_ensemble

    cfg = systems.robertson_config(size=8)
    try:
        hist = scipy_ensemble.solve(systems.robertson, cfg["y0"], cfg["t_span"], cfg["params"],
                                    method="LSODA", rtol=1e-8, atol=1e-12, workers=2)
    finally:
        scipy_ensemble.close()
    ref, *_ = oracle.solve("rodas5P", oracle.System.robertson(), cfg["y0"], cfg["t_span"], cfg["params"],
                           rtol=1e-12, atol=1e-14, lu_precision="fp64")
    np.testing.assert_allclose(hist, ref, rtol=1e-5, atol=1e-10)
