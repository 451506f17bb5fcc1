"""The generated derivative code, compiled for the host with g++, against the
oracle's dual-number derivatives.

The kernels' right-hand side, coloured negated Jacobian, df/dt, VJP,
Hessian-vector product and df/dt-VJP are emitted as CUDA C++ by the tracer and
code generator.  The same text compiles as host C++ once the CUDA qualifiers are
defined away, so every piece is checked here without a GPU.
"""

import ctypes
import math
import subprocess

import numpy as np
import pytest

from workloads import systems
from menodax_b200._codegen import emit_adjoint_pieces, emit_neg_jac, emit_rhs
from menodax_b200._sparsity import dense_jacobian
from menodax_b200._trace import TraceError, evaluate, trace

PRELUDE = """
#include <cmath>
#include <cstring>
using std::exp; using std::log; using std::sqrt; using std::sin; using std::cos; using std::pow;
using std::tanh; using std::fabs; using std::atan2; using std::log1p; using std::expm1;
#define __device__
#define __forceinline__ inline
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
#define MDX_LU_T double
"""

WRAPPERS = """
extern "C" void h_rhs(const double* y, double t, const double* p, double* out) { mdx_rhs(y, t, p, out); }
extern "C" void h_neg_jac(const double* y, double t, const double* p, double* lu, double* dT) { mdx_neg_jac(y, t, p, lu, dT); }
extern "C" void h_vjp(const double* u, double t, const double* p, const double* rb, double* ub, double* pb) { mdx_vjp(u, t, p, rb, ub, pb); }
extern "C" void h_hvp(const double* y, double t, const double* p, const double* kv, const double* rb, double* yb, double* pb) { mdx_hvp(y, t, p, kv, rb, yb, pb); }
extern "C" void h_ft_vjp(const double* y, double t, const double* p, const double* db, double* yb, double* pb) { mdx_ft_vjp(y, t, p, db, yb, pb); }
"""


def _host_build(tmp_path, fn, n, np_):
    tr = trace(fn, n, np_)
    src = PRELUDE + emit_rhs(tr) + emit_neg_jac(tr, dense_jacobian(n), n * n) + emit_adjoint_pieces(tr) + WRAPPERS
    cpp = tmp_path / "gen.cpp"
    so = tmp_path / "gen.so"
    cpp.write_text(src)
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-w", str(cpp), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    return tr, lib


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.c_void_p)


def _call(lib, name, *args):
    getattr(lib, name)(*[(_p(a) if isinstance(a, np.ndarray) else ctypes.c_double(a)) for a in args])


def with_math(y, t, p):
    return (
        math.exp(-p[0] * y[0]) * math.sin(y[1]) + t * t,
        math.sqrt(1.0 + y[0] * y[0]) - p[1] * y[1] ** 3 + math.tanh(y[0] * t),
        y[0] / (1.0 + y[1] * y[1]) + p[0] ** 2.5 * math.log(2.0 + y[0] * y[0]),
    )


CASES = [
    ("robertson", systems.robertson, 3, 3, lambda O: O.System.robertson()),
    ("lorenz", systems.lorenz, 3, 1, lambda O: O.System.lorenz()),
    ("vdp3", systems.make_vdp_system(3, mu=1.0, d=0.1)[0], 6, 1, lambda O: O.System.vdp_ring(3, 1.0, 0.1)),
    ("brusselator4", systems.make_brusselator_b(4), 8, 1, lambda O: O.System.brusselator(4)),
    ("forced", systems.forced_decay, 1, 2, lambda O: O.System.forced()),
    ("with_math", with_math, 3, 2, lambda O: O.System.callback(with_math, 3, 2)),
]


@pytest.mark.parametrize("name,fn,n,np_,system", CASES, ids=[c[0] for c in CASES])
def test_generated_derivatives_match_dual_numbers(tmp_path, oracle, name, fn, n, np_, system):
    tr, lib = _host_build(tmp_path, fn, n, np_)
    sys_ = system(oracle)
    rng = np.random.default_rng(0)
    y = rng.uniform(0.5, 1.5, n)
    p = rng.uniform(0.5, 1.5, np_)
    t = 0.3
    out = np.empty(n)
    _call(lib, "h_rhs", y, t, p, out)
    np.testing.assert_allclose(out, evaluate(tr, y, t, p), rtol=1e-14, atol=1e-14)

    J = np.stack([oracle.jvp(sys_, y, t, p, np.eye(n)[c]) for c in range(n)], axis=1)
    Jp = np.stack([oracle.jvp(sys_, y, t, p, np.zeros(n), 0.0, np.eye(np_)[k]) for k in range(np_)], axis=1)
    ft = oracle.jvp(sys_, y, t, p, np.zeros(n), 1.0)
    lu = np.empty(n * n)
    dT = np.empty(n)
    _call(lib, "h_neg_jac", y, t, p, lu, dT)
    np.testing.assert_allclose(-lu.reshape(n, n), J, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(dT, ft, rtol=1e-12, atol=1e-12)

    r = rng.normal(size=n)
    ub = np.empty(n)
    pb = np.zeros(np_)
    _call(lib, "h_vjp", y, t, p, r, ub, pb)
    np.testing.assert_allclose(ub, J.T @ r, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(pb, Jp.T @ r, rtol=1e-12, atol=1e-12)

    kv = rng.normal(size=n)
    yb = np.zeros(n)
    pb = np.zeros(np_)
    _call(lib, "h_hvp", y, t, p, kv, r, yb, pb)
    ey = [r @ oracle.jvp2(sys_, y, t, p, kv, 0.0, np.zeros(np_), np.eye(n)[c], 0.0, np.zeros(np_)) for c in range(n)]
    ep = [r @ oracle.jvp2(sys_, y, t, p, kv, 0.0, np.zeros(np_), np.zeros(n), 0.0, np.eye(np_)[k]) for k in range(np_)]
    np.testing.assert_allclose(yb, ey, rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(pb, ep, rtol=1e-11, atol=1e-11)

    d = rng.normal(size=n)
    yb = np.zeros(n)
    pb = np.zeros(np_)
    _call(lib, "h_ft_vjp", y, t, p, d, yb, pb)
    ey = [d @ oracle.jvp2(sys_, y, t, p, np.zeros(n), 1.0, np.zeros(np_), np.eye(n)[c], 0.0, np.zeros(np_)) for c in range(n)]
    ep = [d @ oracle.jvp2(sys_, y, t, p, np.zeros(n), 1.0, np.zeros(np_), np.zeros(n), 0.0, np.eye(np_)[k]) for k in range(np_)]
    np.testing.assert_allclose(yb, ey, rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(pb, ep, rtol=1e-11, atol=1e-11)


def test_tracer_refuses_branching():
    def branchy(y, t, p):
        return (y[0] if y[0] > 0 else -y[0],)

    with pytest.raises(TraceError, match="branches"):
        trace(branchy, 1, 1)


def test_tracer_checks_component_count():
    with pytest.raises(ValueError, match="components"):
        trace(lambda y, t, p: (y[0], y[1]), 3, 0)


def test_tracer_requires_literal_indices():
    with pytest.raises(TraceError):
        trace(lambda y, t, p: (y[1.5], y[0]), 2, 0)


def test_common_subexpressions_collapse():
    def fn(y, t, p):
        a = y[0] * y[1]
        b = y[0] * y[1]
        return (a + b, a * b)

    tr = trace(fn, 2, 0)
    muls = [nd for nd in tr.graph.nodes if nd.op == "mul"]
    assert len(muls) == 2  # y0*y1 once, then a*b


def test_sensitivity_spec_sizes():
    """tests/test_sensitivity.py:124-161 in the reference: only requested blocks count."""
    from menodax_b200.sensitivity import SensitivitySpec

    params_only = SensitivitySpec(n_vars=4, n_params=2, wrt_y0=False, wrt_params=True)
    assert params_only.n_sens == 2 and params_only.n_aug == 12 and params_only.n_error == 12
    both = SensitivitySpec(n_vars=4, n_params=2, wrt_y0=True, wrt_params=True, error_control=False)
    assert both.n_sens == 6 and both.n_aug == 28 and both.n_error == 4
    cols = SensitivitySpec(n_vars=3, n_params=5, wrt_y0=False, wrt_params=True, param_columns=(4, 1))
    assert cols.param_seed_columns == (4, 1) and cols.n_sens == 2
    with pytest.raises(ValueError, match="at least one"):
        SensitivitySpec(n_vars=2, n_params=1, wrt_y0=False, wrt_params=False)
    with pytest.raises(ValueError, match="repeat"):
        SensitivitySpec(n_vars=2, n_params=3, wrt_y0=False, wrt_params=True, param_columns=(1, 1))


def test_augmented_layout():
    import torch

    from menodax_b200.sensitivity import SensitivitySpec, augmented_y0, split_augmented

    spec = SensitivitySpec(n_vars=2, n_params=1, wrt_y0=True, wrt_params=True)
    z = augmented_y0(torch.tensor([[1.0, 2.0]]), spec)
    assert z.tolist() == [[1.0, 2.0, 1.0, 0.0, 0.0, 1.0, 0.0, 0.0]]
    state, sens = split_augmented(z.reshape(1, 1, -1), spec)
    assert state.tolist() == [[[1.0, 2.0]]]
    assert sens[0, 0].tolist() == [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]


def test_tsit5_shared_stages_build_and_bounds():
    """The shared-memory placement of Tsit5's stages compiles (NVRTC, no GPU),
    is refused for Rodas5P, and is bounded by a block's static shared memory."""
    from menodax_b200._problem import KernelOptions, STATIC_SHARED_MAX, build_source, get_problem, tsit5_stage_bytes

    fn, _ = systems.make_vdp_system(8, mu=1.0, d=0.1)
    prob = get_problem(fn, 16, 1, KernelOptions(solver="tsit5", threads_per_block=32, shared_stages=True))
    assert "#define MDX_TSIT5_SHARED 1" in prob.source
    assert tsit5_stage_bytes(16, 32) == 6 * 16 * 32 * 8 <= STATIC_SHARED_MAX
    with pytest.raises(ValueError, match="shared memory"):
        build_source(fn, 16, 1, KernelOptions(solver="tsit5", threads_per_block=128, shared_stages=True))
    with pytest.raises(ValueError, match="team kernel"):
        build_source(fn, 16, 1, KernelOptions(solver="rodas5P", shared_stages=True))
