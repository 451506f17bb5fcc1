"""The front end's launch decisions for host results, with the device stubbed.

No GPU: the launch is a recorder and the autotuner's pick is fixed, so what is
checked is which launch ``rodas5P.solve`` issues for NumPy inputs (results that
go to host memory) after the autotuner has chosen a persistent launch.
"""

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from menodax_b200 import _frontend, _native, autotune, rodas5P
from workloads import systems

PLAIN, PERSISTENT = _native.MDX_LAUNCH_PLAIN, _native.MDX_LAUNCH_PERSISTENT


@pytest.fixture
def stub_device(monkeypatch):
    calls = []

    def fake_launch(problem, **kw):
        calls.append(kw)
        n = kw["y0"].shape[0]
        s = kw.get("n_save_hist") or kw["times"].numel()
        return (torch.zeros((n, s, problem.n_system), dtype=torch.float64),
                torch.zeros((4, n), dtype=torch.int32))

    empty = torch.empty
    monkeypatch.setattr(_frontend, "launch", fake_launch)
    monkeypatch.setattr(_frontend, "pick_device", lambda *a, **k: torch.device("cpu"))
    monkeypatch.setattr(autotune, "grid_blocks", lambda *a, **k: 512)
    monkeypatch.setattr(torch, "empty", lambda *a, pin_memory=False, **k: empty(*a, **k))
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: SimpleNamespace(synchronize=lambda: None))
    _frontend._order_hint.clear()
    yield calls
    _frontend._order_hint.clear()


def _solve(monkeypatch, choice):
    monkeypatch.setattr(autotune, "tune", lambda *a, **k: choice)
    cfg = systems.robertson_config(size=4096)
    out = rodas5P.solve(cfg["ode_fn"], cfg["y0"], cfg["t_span"], cfg["params"], rtol=cfg["rtol"],
                        atol=cfg["atol"], lu_precision="fp32")
    assert isinstance(out, np.ndarray) and out.shape == (4096, len(cfg["t_span"]), 3)


def test_a_short_persistent_thread_launch_gives_way_to_the_streaming_one_launch_kernel(stub_device, monkeypatch):
    _solve(monkeypatch, autotune.LaunchChoice(128, PERSISTENT, 1.0, 0))
    kw = stub_device[-1]
    assert kw["mode"] == PLAIN and kw["grid_blocks"] == 0
    assert kw["hist_host"] is not None and kw["order"] is None


def test_a_half_filled_persistent_launch_is_kept_and_copied_after_the_kernel(stub_device, monkeypatch):
    choice = autotune.LaunchChoice(128, PERSISTENT, 0.5, 0)
    _solve(monkeypatch, choice)
    first = stub_device[-1]
    assert first["mode"] == PERSISTENT and first["grid_blocks"] == 512
    assert first["hist_host"] is None and first["order"] is None
    # The second call of the same problem visits trajectories longest first.
    _solve(monkeypatch, choice)
    second = stub_device[-1]
    assert second["order"] is not None and second["order"].dtype == torch.int32
    assert second["order"].numel() == 4096
