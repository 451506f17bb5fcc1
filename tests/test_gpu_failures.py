"""Failure handling without faulting the GPU: step budgets, non-finite inputs,
empty ensembles.  Every kernel loop is bounded by max_steps, so each of these
ends with a status bit, not a hang or a trap."""

import numpy as np
import pytest

from menodax_b200 import rodas5P, tsit5
from workloads import systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("launch", ["plain", "persistent"])
def test_max_steps_sets_the_status_bit_and_freezes_saves(launch):
    cfg = systems.robertson_config(size=64)
    hist, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=1e-6,
                                atol=1e-10, max_steps=10, return_stats=True, launch=launch)
    assert (stats["loop_steps"] == 10).all()
    assert ((stats["status"] & 1) == 1).all()
    # saves past the point reached hold the last state (modax/rodas5P.py:991-1002)
    assert (hist[:, -1] == hist[:, -2]).all()


def test_tsit5_max_steps_marks_unreached_saves():
    cfg = systems.lorenz_config(size=32)
    hist, stats = tsit5.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], max_steps=3,
                              return_stats=True)
    assert ((stats["status"] & 1) == 1).all()
    assert np.isnan(hist[:, -1]).all()


def test_nan_parameters_end_in_a_status_not_a_hang():
    cfg = systems.robertson_config(size=32)
    p = cfg["params"].copy()
    p[::2, 0] = np.nan
    hist, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], p, rtol=1e-6, atol=1e-10,
                                max_steps=500, return_stats=True)
    bad = stats["status"][::2]
    good = stats["status"][1::2]
    assert ((bad & 1) == 1).all() and (stats["loop_steps"][::2] == 500).all()
    assert (good == 0).all()
    assert np.isfinite(hist[1::2]).all()


def test_empty_ensemble():
    out = rodas5P.solve(systems.robertson, np.zeros((0, 3)), systems.ROBERTSON_TIMES, np.zeros((0, 3)))
    assert out.shape == (0, len(systems.ROBERTSON_TIMES), 3)
