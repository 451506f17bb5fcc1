"""The save hook traced into the Rodas5P kernel (reference tests/test_save_hook.py):
an in-kernel accumulation equals the same accumulation over the saved history,
derived per-save values match the history, and save_history=False keeps the
final state."""

import numpy as np
import pytest

from menodax_b200 import rodas5P

pytestmark = pytest.mark.gpu

N_SAVE = 33


def damped_oscillator(y, t, p):
    return (y[1], -p[0] * y[0] - p[1] * y[1])


def _problem():
    t_span = np.linspace(0.0, 4.0, N_SAVE)
    y0 = np.array([[1.0, 0.0], [0.5, 1.0], [-1.0, 0.3]])
    params = np.array([[4.0, 0.2], [9.0, 0.5], [1.0, 0.0]])
    return y0, t_span, params


def _trapezoid_weights(t_span):
    w = np.zeros_like(t_span)
    w[1:] += 0.5 * np.diff(t_span)
    w[:-1] += 0.5 * np.diff(t_span)
    return w


def test_hook_accumulates_what_the_history_integrates():
    y0, t_span, params = _problem()
    weights = _trapezoid_weights(t_span)

    def integrate_state(save_idx, y, t, p_row, acc):
        acc[0] += weights[save_idx] * y[0]
        acc[1] += weights[save_idx] * y[1]
        acc[2] += 1.0

    kw = dict(rtol=1e-8, atol=1e-10, lu_precision="fp64")
    hist = rodas5P.solve(damped_oscillator, y0, t_span, params, **kw)
    final, acc = rodas5P.solve(damped_oscillator, y0, t_span, params, save_hook=integrate_state,
                               hook_size=3, save_history=False, **kw)
    assert final.shape == (3, 1, 2)
    np.testing.assert_allclose(final[:, 0], hist[:, -1], rtol=0, atol=1e-13)
    np.testing.assert_allclose(acc[:, 0], np.trapezoid(hist[..., 0], t_span, axis=1), rtol=1e-12)
    np.testing.assert_allclose(acc[:, 1], np.trapezoid(hist[..., 1], t_span, axis=1), rtol=1e-12)
    assert np.all(acc[:, 2] == N_SAVE)


def test_hook_can_store_derived_saves_beside_the_history():
    y0, t_span, params = _problem()

    def store_energy(save_idx, y, t, p_row, acc):
        acc[save_idx] = 0.5 * (y[1] * y[1] + p_row[0] * y[0] * y[0])

    hist, energy = rodas5P.solve(damped_oscillator, y0, t_span, params, save_hook=store_energy,
                                 hook_size=N_SAVE, rtol=1e-8, atol=1e-10, lu_precision="fp64")
    assert hist.shape == (3, N_SAVE, 2)
    expected = 0.5 * (hist[..., 1] ** 2 + params[:, :1] * hist[..., 0] ** 2)
    np.testing.assert_allclose(energy, expected, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(energy[2], energy[2, 0], rtol=1e-6)


def test_hook_index_outside_its_row_is_refused_before_launch():
    y0, t_span, params = _problem()

    def too_far(save_idx, y, t, p_row, acc):
        acc[save_idx + 1] = y[0]

    with pytest.raises(ValueError, match="outside its"):
        rodas5P.solve(damped_oscillator, y0, t_span, params, save_hook=too_far, hook_size=N_SAVE)


def test_team_kernel_runs_the_save_hook():
    """The save hook in the team kernel (teams of 4 lanes on the 8-state VdP ring):
    the same accumulation as the thread kernel's hook."""
    from workloads import systems

    cfg = systems.vdp_ring_config(4, size=64)
    t_span = np.linspace(0.0, 5.0, 9)
    weights = np.linspace(0.5, 1.5, 9)

    def hook(save_idx, y, t, p_row, acc):
        acc[0] += weights[save_idx] * y[0]
        acc[1] += y[3] * y[3]
        acc[2] += 1.0

    kw = dict(rtol=1e-8, atol=1e-10, lu_precision="fp64", save_hook=hook, hook_size=3, launch="plain")
    h0, a0 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], team=0, **kw)
    h4, a4 = rodas5P.solve(cfg["ode_fn"], cfg["y0"], t_span, cfg["params"], team=4, **kw)
    assert (a0[:, 2] == 9).all() and (a4[:, 2] == 9).all()
    np.testing.assert_allclose(h4, h0, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(a4, a0, rtol=1e-9, atol=1e-12)
