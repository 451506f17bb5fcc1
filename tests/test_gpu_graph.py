"""CUDA-graph-captured solves replay the same kernel on new inputs."""

import numpy as np
import pytest
import torch

from menodax_b200 import rodas5P
from workloads import systems
from menodax_b200.graph import GraphedSolve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("launch_mode", ["plain", "persistent"])
def test_graphed_solve_matches_direct_calls(launch_mode):
    a = systems.robertson_config(size=2048, seed=1)
    b = systems.robertson_config(size=2048, seed=2)
    g = GraphedSolve("rodas5P", a["ode_fn"], 2048, 3, 3, a["t_span"], rtol=a["rtol"], atol=a["atol"],
                     launch_mode=launch_mode)
    for cfg in (a, b, a):
        hist, counters = g(cfg["y0"], cfg["params"])
        torch.cuda.synchronize()
        direct, stats = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"],
                                      rtol=cfg["rtol"], atol=cfg["atol"], launch=launch_mode,
                                      return_stats=True)
        assert np.array_equal(hist.cpu().numpy(), direct)
        assert np.array_equal(counters[2].cpu().numpy(), stats["loop_steps"])
