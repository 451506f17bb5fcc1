"""The JAX front end's glue, without JAX (not installed here or on the GPU box).

A stand-in ``jax`` module supplies the few pieces the front end touches
(``custom_vmap``, ``custom_jvp``, ``custom_vjp``, ``ffi.ffi_call``,
``ShapeDtypeStruct``), with NumPy as ``jax.numpy``; its "device" runs the two
custom calls on the CPU oracle.  That exercises what this library writes -- the
vmap rule folding a vmap into one ensemble call, the custom-call arguments, the
augmented initial state and the contraction of the forward sensitivities, the
adjoint's masking and reductions -- but not JAX's own transformations.
"""

import sys
import types
from collections import namedtuple

import numpy as np
import pytest

from menodax_b200 import jax_api
from menodax_b200._problem import _cache as problem_cache
from workloads import systems

A, B = 0.7, 1.3
T = np.linspace(0.0, 2.0, 5)


class _Symbolic:
    """A symbolic zero tangent."""


class _Wrapped:
    def __init__(self, fn):
        self.fn = fn
        self.rule = self.jvp = self.fwd = self.bwd = None
        self.symbolic_zeros = None

    def __call__(self, *args):
        return self.fn(*args)

    def def_vmap(self, rule):
        self.rule = rule
        return rule

    def defjvp(self, jvp, symbolic_zeros=False):
        self.jvp, self.symbolic_zeros = jvp, symbolic_zeros
        return jvp

    def defvjp(self, fwd, bwd):
        self.fwd, self.bwd = fwd, bwd


def _problem_for(address):
    for prob in problem_cache.values():
        if jax_api.plan_address(prob) == address:
            return prob
    raise KeyError(address)


def _fake_device(oracle, calls):
    """The two custom calls, run on the oracle (cascade system, Rodas5P, FP64)."""

    def solve(specs, args, attrs):
        y0, times, params, _weights = args
        prob = _problem_for(int(attrs["plan"]))
        n = prob.n_vars
        sens = prob.options.sens
        kw = dict(rtol=float(attrs["rtol"]), atol=float(attrs["atol"]), lu_precision="fp64")
        if sens is not None:
            hist, acc, rej, loop = oracle.solve("rodas5P", oracle.System.cascade(), y0[:, :n], times, params,
                                                sens=(sens[0] > 0, list(sens[1]), bool(sens[2])), **kw)
        else:
            hist, acc, rej, loop = oracle.solve("rodas5P", oracle.System.cascade(), y0, times, params, **kw)
        counters = np.stack([acc, rej, loop, np.zeros_like(acc)]).astype(np.int32)
        ckpt = np.zeros(specs[3].shape)
        if ckpt.size >= y0.size:
            ckpt[: y0.size] = y0.ravel()  # the stand-in reverse pass reads y0 back from here
        return (hist, counters, np.zeros(specs[2].shape, np.uint8), ckpt, acc.astype(np.int32)[: specs[4].shape[0]])

    def grad(specs, args, attrs):
        times, params, ckpt, count, g_hist, order = args
        assert sorted(order.tolist()) == list(range(len(count)))
        n_traj = len(count)
        y0 = ckpt[: n_traj * 2].reshape(n_traj, 2)
        hist, *_ = oracle.solve("rodas5P", oracle.System.cascade(), y0, times, params, rtol=1e-10, atol=1e-12,
                                lu_precision="fp64", sens=(True, [0, 1], False))
        s = hist[:, :, 2:].reshape(n_traj, len(times), 4, 2)
        g = np.einsum("nsj,nskj->nk", g_hist, s)
        return g[:, :2], g[:, 2:], np.zeros(n_traj, np.int32)

    handlers = {jax_api.SOLVE_TARGET: solve, jax_api.GRAD_TARGET: grad}

    def ffi_call(name, specs, has_side_effect=False):
        assert has_side_effect is False

        def run(*args, **attrs):
            calls.append((name, [np.asarray(a).shape for a in args], attrs))
            return handlers[name](specs, [np.asarray(a) for a in args], attrs)

        return run

    return ffi_call


@pytest.fixture
def fake_jax(monkeypatch, oracle):
    calls = []
    jax = types.ModuleType("jax")
    jax.numpy = np
    jax.ShapeDtypeStruct = namedtuple("ShapeDtypeStruct", "shape dtype")
    jax.ffi = types.SimpleNamespace(ffi_call=_fake_device(oracle, calls))
    jax.custom_batching = types.SimpleNamespace(custom_vmap=_Wrapped)
    jax.custom_jvp = _Wrapped
    jax.custom_vjp = _Wrapped
    jax.custom_derivatives = types.SimpleNamespace(SymbolicZero=_Symbolic)
    jax.dtypes = types.SimpleNamespace(float0=np.dtype([("float0", np.void, 0)]))
    monkeypatch.setitem(sys.modules, "jax", jax)
    monkeypatch.setattr(jax_api, "register_targets", lambda: None)
    return jax, calls


def _solver(**kw):
    from menodax_b200._problem import KernelOptions

    opts = dict(rtol=1e-10, atol=1e-12, first_step=None, max_steps=100000, sens_error_control=True,
                sens_param_columns=None, adjoint_capacity=64)
    opts.update(kw)
    return jax_api._Solver(systems.cascade, 2, 2, KernelOptions(lu_precision="fp64"), **opts)


def test_vmap_rule_folds_the_vmapped_axis_into_one_ensemble_call():
    seen = []

    def ensemble(y0, t, p):
        seen.append((y0.shape, p.shape))
        return np.zeros((y0.shape[0], len(t), 2)), np.zeros((4, y0.shape[0]), np.int32)

    out, batched = jax_api.vmap_rule(np, ensemble, 5, (True, False, False), np.ones((5, 2)), T, np.ones(2))
    assert seen == [((5, 2), (5, 2))]
    assert out[0].shape == (5, 1, len(T), 2) and out[1].shape == (5, 4, 1) and batched == (True, True)
    out, _ = jax_api.vmap_rule(np, ensemble, 3, (False, True, True), np.ones(2), np.tile(T, (3, 1)),
                               np.ones((3, 2)))
    assert out[0].shape == (3, 1, len(T), 2)
    with pytest.raises(NotImplementedError, match="already-ensembled y0"):
        jax_api.vmap_rule(np, ensemble, 2, (True, False, False), np.ones((2, 4, 2)), T, np.ones(2))
    with pytest.raises(NotImplementedError, match="nested t_span"):
        jax_api.vmap_rule(np, ensemble, 2, (False, True, False), np.ones(2), np.ones((2, 2, 3)), np.ones(2))
    with pytest.raises(ValueError, match="leading axis 4, expected 2"):
        jax_api.vmap_rule(np, ensemble, 2, (False, False, True), np.ones(2), T, np.ones((4, 2)))


def test_contraction_and_masks():
    rng = np.random.default_rng(0)
    sens = rng.normal(size=(3, 4, 2, 5))  # y0 directions 0-1, parameter columns 2-4
    dy0, dp = rng.normal(size=(3, 2)), rng.normal(size=(3, 6))
    got = jax_api.contract_tangent(np, sens, 2, dy0, dp, (5, 0, 3))
    want = np.einsum("nsij,nj->nsi", sens[..., :2], dy0) + np.einsum("nsik,nk->nsi", sens[..., 2:], dp[:, [5, 0, 3]])
    np.testing.assert_allclose(got, want)
    assert jax_api.sensitivity_blocks(True, False) == (False, True)
    gy, gp = jax_api.mask_adjoint(np, np.ones((3, 2)), np.ones((3, 4)), np.array([0, 4, 1]), (1, 3))
    assert np.isnan(gy[1]).all() and np.isnan(gp[1, [1, 3]]).all() and (gp[1, [0, 2]] == 0).all()
    assert (gp[0] == [0, 1, 0, 1]).all() and (gy[2] == 1).all()


def test_custom_call_arguments(fake_jax):
    solver = _solver()
    prob = solver.problem()
    outputs, attrs = jax_api.solve_call_args(prob, 7, 5, mode=1, dt0=0.0, rtol=1e-6, atol=1e-9, max_steps=50)
    assert [o[0] for o in outputs] == [(7, 5, 2), (4, 7), (jax_api.WORKSPACE_BYTES,), (1,), (1,)]
    assert attrs["plan"].dtype == np.int64 and attrs["plan"] == jax_api.plan_address(prob) != 0
    assert attrs["max_steps"].dtype == np.int32 and attrs["rtol"] == 1e-6 and attrs["ckpt_capacity"] == 0
    ck = solver.problem(checkpoint=True, adjoint=True, ckpt_stride=jax_api.ADJOINT_STRIDE)
    outputs, attrs = jax_api.solve_call_args(ck, 7, 5, mode=1, dt0=0.0, rtol=1e-6, atol=1e-9, max_steps=50,
                                             ckpt_capacity=64)
    assert outputs[3][0] == (ck.plan.checkpoint_size(7, 64) // 8,) and outputs[4][0] == (7,)


def test_primal_solve_is_one_ensemble_call(fake_jax, oracle):
    _, calls = fake_jax
    y0 = np.tile([2.0, 0.5], (4, 1))
    p = np.tile([A, B], (4, 1))
    hist, stats = jax_api.rodas5P_solve(systems.cascade, y0, T, p, rtol=1e-10, atol=1e-12, lu_precision="fp64",
                                        return_stats=True)
    ref, acc, *_ = oracle.solve("rodas5P", oracle.System.cascade(), y0, T, p, rtol=1e-10, atol=1e-12,
                                lu_precision="fp64")
    np.testing.assert_array_equal(hist, ref)
    np.testing.assert_array_equal(stats["accepted_steps"], acc)
    assert [c[0] for c in calls] == [jax_api.SOLVE_TARGET]
    assert calls[0][1][:3] == [(4, 2), (5,), (4, 2)]
    # A single trajectory: 1-D y0 and params become an ensemble of one.
    one = jax_api.rodas5P_solve(systems.cascade, y0[0], T, p[0], rtol=1e-10, atol=1e-12, lu_precision="fp64")
    assert one.shape == (1, 5, 2)


def test_jvp_rule_carries_only_the_tangent_blocks(fake_jax, oracle):
    """The custom_jvp rule: symbolic zeros decide the blocks, the joint solve's S is
    contracted with the tangents, the step counters get float0 tangents."""
    jax, calls = fake_jax
    fn = _solver().build()
    assert fn.symbolic_zeros is True
    y0, p = np.array([[2.0, 0.5]]), np.array([[A, B]])
    dp = np.array([[1.0, -2.0]])
    (state, counters), (tangent, ct) = fn.jvp((y0, T, p), (_Symbolic(), _Symbolic(), dp))
    assert ct.dtype == jax.dtypes.float0
    assert calls[-1][1][0] == (1, 2 + 2 * 2)  # y plus two parameter directions, no y0 block
    hist, *_ = oracle.solve("rodas5P", oracle.System.cascade(), y0, T, p, rtol=1e-10, atol=1e-12,
                            lu_precision="fp64", sens=(False, [0, 1], True))
    s = hist[:, :, 2:].reshape(1, len(T), 2, 2)
    np.testing.assert_allclose(tangent, np.einsum("nskj,nk->nsj", s, dp))
    np.testing.assert_allclose(state, hist[:, :, :2])
    with pytest.raises(NotImplementedError, match="t_span"):
        fn.jvp((y0, T, p), (_Symbolic(), np.ones_like(T), dp))


def test_vjp_backward_masks_and_reduces(fake_jax, oracle):
    """custom_vjp (sens_error_control=False): the forward pass records, the backward
    pass returns the reverse kernel's cotangents; inputs broadcast over the
    ensemble get the sum of their rows'; unlisted parameter columns get zeros."""
    fn = _solver(sens_error_control=False, sens_param_columns=[1]).build()
    y0 = np.array([2.0, 0.5])
    p = np.tile([A, B], (3, 1))
    (hist, counters), res = fn.fwd(y0, T, p)
    g_hist = np.random.default_rng(1).normal(size=hist.shape)
    gy0, g_t, gp = fn.bwd(res, (g_hist, None))
    assert g_t is None and gy0.shape == (2,) and gp.shape == (3, 2)
    full, *_ = oracle.solve("rodas5P", oracle.System.cascade(), np.tile(y0, (3, 1)), T, p, rtol=1e-10,
                            atol=1e-12, lu_precision="fp64", sens=(True, [0, 1], False))
    s = full[:, :, 2:].reshape(3, len(T), 4, 2)
    g = np.einsum("nsj,nskj->nk", g_hist, s)
    np.testing.assert_allclose(gy0, g[:, :2].sum(axis=0))
    assert (gp[:, 0] == 0).all()
    np.testing.assert_allclose(gp[:, 1], g[:, 3])


def test_front_end_needs_jax_and_says_so(monkeypatch):
    monkeypatch.setitem(sys.modules, "jax", None)
    with pytest.raises(ImportError, match="needs JAX"):
        jax_api.tsit5_solve(systems.cascade, np.ones(2), T, np.ones(2))
