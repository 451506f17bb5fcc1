"""The launch autotuner's decisions, with the timed launches replaced by a cost table.

No GPU: ``autotune._timed_launch`` and ``get_problem`` are stand-ins, so what is
checked is which candidates exist for which systems, which path the step-capped
probe takes, and which launch comes back.
"""

from types import SimpleNamespace

import pytest
import torch

from menodax_b200 import _native, autotune
from workloads import systems
from menodax_b200._problem import KernelOptions
from menodax_b200._sparsity import normalize_sparsity

PLAIN, PERSISTENT = _native.MDX_LAUNCH_PLAIN, _native.MDX_LAUNCH_PERSISTENT


class Recorder:
    """Fake timed launch: seconds from ``cost(choice, n, max_steps)``, steps from ``steps``."""

    def __init__(self, cost, steps):
        self.cost = cost
        self.steps = steps
        self.calls = []

    def __call__(self, problem, choice, stream, *, n, max_steps, **_):
        self.calls.append((choice, n, max_steps))
        counters = torch.zeros((4, n), dtype=torch.int32)
        counters[2] = min(self.steps, max_steps)
        return self.cost(choice, n, max_steps), counters


@pytest.fixture
def fake_device(monkeypatch):
    plan = SimpleNamespace(occupancy=lambda mode: (4, 148))
    monkeypatch.setattr(autotune, "get_problem", lambda *a, **k: SimpleNamespace(plan=plan))
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a, **k: "fake B200")
    autotune._cache.clear()
    yield
    autotune._cache.clear()


def _tune(fn, n_vars, options, recorder, monkeypatch, n=8192, max_steps=100000, **kw):
    monkeypatch.setattr(autotune, "_timed_launch", recorder)
    y0 = torch.zeros((n, n_vars), dtype=torch.float64)
    params = torch.zeros((n, 1), dtype=torch.float64)
    return autotune.tune(fn, n_vars, 1, options, y0=y0, times=torch.zeros(3, dtype=torch.float64),
                         params=params, weights=None, dt0=0.0, rtol=1e-6, atol=1e-8,
                         max_steps=max_steps, **kw)


def _ring(n_osc):
    fn, _ = systems.make_vdp_system(n_osc, mu=1.0, d=0.1)
    return fn, 2 * n_osc, normalize_sparsity(systems.vdp_sparsity(n_osc), 2 * n_osc)


def test_short_integrations_time_every_candidate_and_keep_the_fastest(fake_device, monkeypatch):
    fn, n, pattern = _ring(16)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern)

    def cost(choice, n_traj, steps):
        return 0.010 if (choice.team == 16 and choice.mode == PERSISTENT) else 0.020

    rec = Recorder(cost, steps=120)
    choice = _tune(fn, n, opts, rec, monkeypatch, tune_team=True)
    assert (choice.team, choice.mode) == (16, PERSISTENT)
    timed = {(c.team, c.mode, c.threads_per_block, c.grid_fill) for c, _, s in rec.calls if s == 100000}
    # thread launches at three block sizes (plain + two fills) and two launch kinds per team size
    assert len(timed) == 3 * 3 + 2 * len(autotune.team_sizes_for(n))


def test_long_integrations_rank_plain_launches_by_a_capped_run(fake_device, monkeypatch):
    fn, n, pattern = _ring(64)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern)

    def cost(choice, n_traj, steps):
        return 1.0 if choice.team == 8 else 2.0

    rec = Recorder(cost, steps=100000)
    choice = _tune(fn, n, opts, rec, monkeypatch, tune_team=True)
    assert choice.team == 8 and choice.mode == PERSISTENT and choice.grid_fill == 1.0
    # every launch was capped, ran the whole ensemble, and only plain launches were ranked
    assert all(s == autotune.PROBE_STEPS and m == 8192 for _, m, s in rec.calls)
    assert all(c.mode == PLAIN for c, _, _ in rec.calls)


def test_long_integrations_pick_the_half_filled_persistent_thread_launch(fake_device, monkeypatch):
    fn, n, pattern = _ring(4)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern)

    def cost(choice, n_traj, steps):
        return 1.0 if choice.threads_per_block == 64 else 2.0

    choice = _tune(fn, n, opts, Recorder(cost, steps=100000), monkeypatch, tune_team=True)
    assert (choice.team, choice.threads_per_block, choice.mode, choice.grid_fill) == (0, 64, PERSISTENT, 0.5)


def test_candidate_families_follow_the_system_size(fake_device, monkeypatch):
    seen = {}

    def run(key, fn, n, opts):
        rec = Recorder(lambda c, m, s: 1.0, steps=10)
        _tune(fn, n, opts, rec, monkeypatch, tune_team=True)
        seen[key] = {c.team for c, _, _ in rec.calls}

    fn, n, pattern = _ring(4)
    run("ring8 sparse", fn, n, KernelOptions(sparsity=pattern))
    run("ring8 dense", fn, n, KernelOptions())
    fn, n, pattern = _ring(32)
    run("ring64 sparse", fn, n, KernelOptions(sparsity=pattern, fast=True))
    run("ring64 dense", fn, n, KernelOptions(fast=True))
    assert seen["ring8 sparse"] == {0} and seen["ring8 dense"] == {0}   # below TEAM_MIN_VARS
    assert 0 in seen["ring64 sparse"] and seen["ring64 sparse"] - {0}   # sparse: threads and teams
    assert 0 not in seen["ring64 dense"]                                # dense past registers: teams only


def test_a_fixed_team_is_only_tuned_for_its_launch_kind(fake_device, monkeypatch):
    fn, n, pattern = _ring(16)
    opts = KernelOptions(sparsity=pattern, team=8, threads_per_block=128)
    rec = Recorder(lambda c, m, s: 1.0 if c.mode == PLAIN else 0.5, steps=10)
    choice = _tune(fn, n, opts, rec, monkeypatch)
    assert {c.team for c, _, _ in rec.calls} == {8}
    assert (choice.team, choice.threads_per_block, choice.mode) == (8, 128, PERSISTENT)


def test_tsit5_auto_backend_times_shared_stage_launches(fake_device, monkeypatch):
    fn, _ = systems.make_vdp_system(8, mu=1.0, d=0.1)
    opts = KernelOptions(solver="tsit5")
    rec = Recorder(lambda c, m, s: 0.5 if c.shared_stages else 1.0, steps=10)
    choice = _tune(fn, 16, opts, rec, monkeypatch, tune_shared=True)
    assert choice.shared_stages
    shared = {c.threads_per_block for c, _, _ in rec.calls if c.shared_stages}
    assert shared == {32, 64}   # 128 threads of 16-component stages exceed a block's static shared memory
    rec = Recorder(lambda c, m, s: 1.0, steps=10)
    _tune(fn, 16, opts, rec, monkeypatch, tune_shared=False)
    assert not any(c.shared_stages for c, _, _ in rec.calls)


def test_fp64_stage_solves_are_a_candidate_for_mid_sized_thread_kernels(fake_device, monkeypatch):
    """Fast FP32-LU thread kernels of 9-64 states are timed with the stage solves
    in FP32 and in FP64 against the widened factors; smaller systems take the
    FP64 solves without timing, teams and FP64 LUs never have the choice."""
    fn, n, pattern = _ring(16)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern)
    rec = Recorder(lambda c, m, s: 0.5 if c.wide_solve else 1.0, steps=10)
    choice = _tune(fn, n, opts, rec, monkeypatch)
    assert {c.wide_solve for c, _, _ in rec.calls} == {False, True}
    assert choice.wide_solve is True and choice.team == 0
    assert autotune.options_for(opts, choice).wide_solve is True
    assert "FP64 solves" in choice.describe()

    for fn, n, opts in ((_ring(4)[0], 8, KernelOptions(lu_precision="fp32", fast=True)),
                        (_ring(16)[0], 32, KernelOptions(lu_precision="fp64", sparsity=_ring(16)[2])),
                        (_ring(16)[0], 32, KernelOptions(lu_precision="fp32", fast=True, sparsity=_ring(16)[2],
                                                         wide_solve=False))):
        rec = Recorder(lambda c, m, s: 1.0, steps=10)
        _tune(fn, n, opts, rec, monkeypatch)
        assert {c.wide_solve for c, _, _ in rec.calls} == {None}


def test_persistent_candidates_are_timed_longest_first(fake_device, monkeypatch):
    """Short integrations: every persistent candidate is timed visiting the
    trajectories longest first by the probe's step counts (as the front end runs
    a problem from its second solve on); plain candidates take index order."""
    fn, n, pattern = _ring(4)
    opts = KernelOptions(lu_precision="fp32", fast=True, sparsity=pattern)
    seen = []

    def timed(problem, choice, stream, *, n, max_steps, order=None, **_):
        seen.append((choice, n, max_steps, order))
        counters = torch.zeros((4, n), dtype=torch.int32)
        counters[2] = (torch.arange(n, dtype=torch.int32) * 7) % 13 + 100
        return 0.010 if choice.mode == PERSISTENT and choice.grid_fill == 1.0 else 0.020, counters

    choice = _tune(fn, n, opts, timed, monkeypatch, n=256)
    assert (choice.mode, choice.grid_fill, choice.team) == (PERSISTENT, 1.0, 0)
    steps = (torch.arange(256, dtype=torch.int32) * 7) % 13 + 100
    expected = torch.argsort(steps, descending=True, stable=True).to(torch.int32)
    full = [(c, o) for c, _, s, o in seen if s == 100000]
    assert full and all((o is None) == (c.mode == PLAIN) for c, o in full)
    for c, o in full:
        if o is not None:
            assert o.dtype == torch.int32 and torch.equal(o, expected)
    assert torch.equal(autotune.longest_first(steps), expected)


def test_host_results_of_short_persistent_thread_launches_stream_from_the_one_launch_kernel():
    assert autotune.streams_to_host(autotune.LaunchChoice(128, PERSISTENT, 1.0, 0))
    assert not autotune.streams_to_host(autotune.LaunchChoice(128, PERSISTENT, 0.5, 0))
    assert not autotune.streams_to_host(autotune.LaunchChoice(128, PERSISTENT, 1.0, 8))
    assert not autotune.streams_to_host(autotune.LaunchChoice(128, PLAIN, 0.0, 0))
