"""The team kernel's class loops, compiled for the host, against the thread kernel's code.

The team kernel evaluates f, -J and df/dt as loops over classes of structurally
identical components, each member's leaf indices and destination computed from
its position in the class.  Here those loops run on the host for every lane of
a team in turn and must write exactly what the thread kernel's straight-line
functions write (the same expressions, so bit for bit with contraction off).
"""

import ctypes
import math
import subprocess

import numpy as np
import pytest

from workloads import systems
from menodax_b200._codegen import emit_neg_jac, emit_rhs
from menodax_b200._sparse_direct import sparse_lu_for
from menodax_b200._sparsity import dense_jacobian, normalize_sparsity
from menodax_b200._team import dense_lda, emit_team_functions, group_items, index_expr, slice_bytes
from menodax_b200._trace import trace

PRELUDE = """
#include <cmath>
#include <cstring>
using std::exp; using std::log; using std::sqrt; using std::sin; using std::cos; using std::pow;
using std::tanh; using std::fabs; using std::atan2; using std::log1p; using std::expm1;
#define __device__
#define __forceinline__ inline
#define __restrict__
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
#define MDX_LU_T double
"""

WRAPPERS = """
extern "C" void h_rhs(const double* y, double t, const double* p, double* out) { mdx_rhs(y, t, p, out); }
extern "C" void h_neg_jac(const double* y, double t, const double* p, double* lu, double* dT) { mdx_neg_jac(y, t, p, lu, dT); }
extern "C" void h_team_rhs(const double* y, double t, const double* p, double* out) {
  for (int lane = 0; lane < MDX_TEAM; ++lane) mdx_team_rhs(y, t, p, out, lane);
}
extern "C" void h_team_neg_jac(const double* y, double t, const double* p, double* lu) {
  for (int lane = 0; lane < MDX_TEAM; ++lane) mdx_team_neg_jac(y, t, p, lu, lane);
}
extern "C" void h_team_dT(const double* y, double t, const double* p, double* dT) {
  for (int lane = 0; lane < MDX_TEAM; ++lane) mdx_team_dT(y, t, p, dT, lane);
}
"""


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.c_void_p)


def _build(tmp_path, tr, structure, lu_size, lu_slot, team, skip_zero):
    team_code = emit_team_functions(tr, structure, lu_slot, skip_zero=skip_zero)
    src = (PRELUDE + f"#define MDX_TEAM {team}\n" + emit_rhs(tr) + emit_neg_jac(tr, structure, lu_size)
           + team_code.source + WRAPPERS)
    cpp = tmp_path / "team.cpp"
    so = tmp_path / "team.so"
    cpp.write_text(src)
    subprocess.run(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-w", str(cpp),
                    "-o", str(so)], check=True)
    return ctypes.CDLL(str(so)), team_code


def forced_ring(y, t, p):
    """A non-autonomous ring: every component forced by sin(t) with its own phase."""
    n = 6
    return tuple(-p[0] * y[i] + 0.3 * (y[(i + 1) % n] - y[i]) + math.sin(t + 0.5 * i) for i in range(n))


SYSTEMS = [
    ("ring8", systems.make_vdp_system(4, mu=1.0, d=0.1, omega=1.0)[0], 8, 1, systems.vdp_sparsity(4)),
    ("ring32", systems.make_vdp_system(16, mu=1.0, d=0.1, omega=1.0)[0], 32, 1, systems.vdp_sparsity(16)),
    ("bruss16", systems.make_brusselator_b(8), 16, 1, systems.brusselator_pattern(8)),
    ("robertson", systems.robertson, 3, 3, None),
    ("forced_ring", forced_ring, 6, 1, None),
]


@pytest.mark.parametrize("team", [4, 32])
@pytest.mark.parametrize("layout", ["dense", "sparse"])
@pytest.mark.parametrize("name,fn,n,np_,pattern", SYSTEMS, ids=[s[0] for s in SYSTEMS])
def test_team_loops_write_what_the_thread_code_writes(tmp_path, name, fn, n, np_, pattern, layout, team):
    if layout == "sparse" and pattern is None:
        pytest.skip("no sparsity pattern for this system")
    tr = trace(fn, n, np_)
    if layout == "dense":
        structure = dense_jacobian(n)
        lda = dense_lda(n)
        team_size = n * lda

        def slot(row, col):
            return row * lda + col

        thread_slot = [(r, c, r * n + c, r * lda + c) for r in range(n) for c in range(n)]
        lib, code = _build(tmp_path, tr, structure, n * n, slot, team, skip_zero=True)
        clear = -0.0
        thread_size = n * n
    else:
        solver = sparse_lu_for(normalize_sparsity(pattern, n), "amd")
        structure = solver.slots
        store = structure.store_slots()

        def slot(row, colour):
            s = int(store[row * structure.n_colours + colour])
            return None if s < 0 else s

        lib, code = _build(tmp_path, tr, structure, structure.size, slot, team, skip_zero=False)
        team_size = thread_size = structure.size
        thread_slot = [(None, None, s, s) for s in range(structure.size)]
        clear = 0.0
    rng = np.random.default_rng(7)
    for _ in range(3):
        y = rng.uniform(0.2, 2.0, n)
        p = rng.uniform(0.5, 1.5, np_)
        t = float(rng.uniform(0.0, 3.0))
        f_thread = np.zeros(n)
        f_team = np.full(n, np.nan)
        lib.h_rhs(_p(y), ctypes.c_double(t), _p(p), _p(f_thread))
        lib.h_team_rhs(_p(y), ctypes.c_double(t), _p(p), _p(f_team))
        np.testing.assert_array_equal(f_team, f_thread)

        lu_thread = np.zeros(thread_size)
        if layout == "sparse":
            lu_thread[:] = 0.0
        dT_thread = np.zeros(n)
        lib.h_neg_jac(_p(y), ctypes.c_double(t), _p(p), _p(lu_thread), _p(dT_thread))
        lu_team = np.full(team_size, clear)
        lib.h_team_neg_jac(_p(y), ctypes.c_double(t), _p(p), _p(lu_team))
        for _, _, ts, ms in thread_slot:
            assert lu_team[ms] == lu_thread[ts] and math.copysign(1, lu_team[ms]) == math.copysign(1, lu_thread[ts])
        dT_team = np.zeros(n)
        lib.h_team_dT(_p(y), ctypes.c_double(t), _p(p), _p(dT_team))
        if code.autonomous:
            assert not dT_thread.any()
        else:
            np.testing.assert_array_equal(dT_team, dT_thread)


def test_repeated_components_form_few_classes():
    fn, _ = systems.make_vdp_system(64, mu=1.0, d=0.1, omega=1.0)
    tr = trace(fn, 128, 1)
    classes = group_items(tr.graph, [(o, j) for j, o in enumerate(tr.outputs)])
    assert len(classes) == 2
    assert sorted(len(c.members) for c in classes) == [64, 64]


def test_index_expressions():
    tables = []
    assert index_expr([5, 5, 5], 8, "t0", tables) == "5"
    assert index_expr([1, 3, 5, 7], 8, "t1", tables) == "(1 + 2 * m)"
    assert index_expr([6, 0, 2, 4], 8, "t2", tables) == "((6 + 2 * m) % 8)"
    expr = index_expr([3, 1, 4, 1], 8, "t3", tables)
    assert expr == "(int)t3[m]" and tables == ["__device__ const short t3[4] = {3, 1, 4, 1};"]


def test_slice_layout_sizes():
    # y, u, f, p (1) doubles; k[8][8] + lu[72] floats; perm[8] ints.
    assert slice_bytes(8, 1, 72, 4, dense=True, autonomous=True, fast=True) == 8 * 25 + 4 * (64 + 72) + 32
    # Non-autonomous and reference arithmetic add dT and two multiplier columns.
    assert slice_bytes(8, 1, 72, 4, dense=True, autonomous=False, fast=False) == 8 * 49 + 4 * 136 + 32
    assert dense_lda(8) == 9 and dense_lda(9) == 9


def test_team_block_threads_fit_shared_memory():
    from menodax_b200._problem import KernelOptions, team_block_threads

    pattern = normalize_sparsity(systems.vdp_sparsity(4), 8)
    assert team_block_threads(8, 1, KernelOptions(team=8, sparsity=pattern)) == 128
    # A dense 64-state FP32 slice is ~21 KB: eleven fit in a block.  With FP64
    # LUs it is ~41 KB, and a warp of eight 4-lane teams does not fit.
    assert team_block_threads(64, 1, KernelOptions(team=32, fast=True)) == 128
    assert team_block_threads(64, 1, KernelOptions(team=32, fast=True), preferred=1024) == 11 * 32
    with pytest.raises(ValueError, match="shared memory"):
        team_block_threads(64, 1, KernelOptions(team=4, lu_precision="fp64"))


def test_team_source_rejects_what_it_cannot_run():
    from menodax_b200._problem import KernelOptions, build_source

    fn = systems.make_vdp_system(4, mu=1.0, d=0.1)[0]
    for bad in (dict(solver="tsit5"), dict(sens=(8, (), True)), dict(checkpoint=True, adjoint=True)):
        with pytest.raises(ValueError):
            build_source(fn, 8, 1, KernelOptions(team=8, threads_per_block=128, **bad))
    with pytest.raises(ValueError, match="team must be"):
        build_source(fn, 8, 1, KernelOptions(team=3, threads_per_block=96))


def test_team_plan_builds_without_a_gpu():
    from menodax_b200._problem import KernelOptions, get_problem

    fn = systems.make_vdp_system(4, mu=1.0, d=0.1)[0]
    pattern = normalize_sparsity(systems.vdp_sparsity(4), 8)
    prob = get_problem(fn, 8, 1, KernelOptions(team=8, threads_per_block=128, sparsity=pattern, fast=True))
    assert prob.plan.team_size == 8
    assert prob.plan.shared_bytes == 16 * slice_bytes(8, 1, prob.lu_size, 4, dense=False, autonomous=True,
                                                     fast=True)
