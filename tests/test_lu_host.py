"""The in-kernel LU routines, compiled for the host and checked against NumPy.

The device headers are plain C++ apart from a few CUDA spellings, which the
prelude below maps to host equivalents (`__fdividef` becomes an IEEE division;
the device's approximate one is within 2 ulp of it).  Checked: the thread
kernel's dense LU in the reference's arithmetic (register-unrolled and looped
sizes) and in fast arithmetic, FP64 and FP32; the generated sparse LU in both
forms (straight-line and table-driven) and both arithmetics.  Each solves
M x = b and M^T x = b on random systems against numpy.linalg.solve; the dense
matrices have no dominant diagonal, so row pivoting is exercised.
"""

import ctypes
import subprocess

import numpy as np
import pytest

from menodax_b200._native import KERNEL_DIR
from menodax_b200._sparse_direct import analyse, emit_cuda
from menodax_b200._sparsity import normalize_sparsity

PRELUDE = """
#include <cmath>
#include <cstring>
using std::fabs; using std::sqrt; using std::pow; using std::isnan; using std::isfinite; using std::fma;
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__
#define __constant__
static inline float host_fdividef(float a, float b) { return a / b; }
static inline float host_powf(float a, float b) { return std::pow(a, b); }
#define __fdividef host_fdividef
#define __powf host_powf
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
#define MDX_NV 1
#include "mdx_common.cuh"
"""


def _compile(tmp_path, name, source):
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text(PRELUDE + source)
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-w", f"-I{KERNEL_DIR}", str(cpp),
                    "-o", str(so)], check=True)
    return ctypes.CDLL(str(so))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dense_wrapper(n, t, fast):
    fac, solve, solve_t = (("dense_factorize_fast", "dense_solve_fast", "dense_solve_t_fast") if fast else
                           ("dense_factorize", "dense_solve", "dense_solve_t"))
    return f"""
#include "mdx_dense_lu.cuh"
extern "C" void run(const double* a, const double* b, double* x, int transposed) {{
  {t} lu[{n * n}]; int piv[{n}]; {t} r[{n}];
  for (int i = 0; i < {n * n}; ++i) lu[i] = ({t})a[i];
  mdx::{fac}<{n}, {t}>(lu, piv);
  for (int i = 0; i < {n}; ++i) r[i] = ({t})b[i];
  if (transposed) mdx::{solve_t}<{n}, {t}>(lu, piv, r); else mdx::{solve}<{n}, {t}>(lu, piv, r);
  for (int i = 0; i < {n}; ++i) x[i] = (double)r[i];
}}
"""


def _check(run, matrix, tol, seed=3):
    n = len(matrix)
    rng = np.random.default_rng(seed)
    a = np.ascontiguousarray(matrix, dtype=np.float64)
    for transposed in (0, 1):
        for _ in range(3):
            b = rng.normal(size=n)
            x = np.zeros(n)
            run(_p(a), _p(b), _p(x), transposed)
            ref = np.linalg.solve(a.T if transposed else a, b)
            assert np.linalg.norm(x - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.parametrize("fast", [False, True])
@pytest.mark.parametrize("t", ["double", "float"])
@pytest.mark.parametrize("n", [3, 8, 12, 20])
def test_dense_lu_solves_with_pivoting(tmp_path, n, t, fast):
    if fast and n > 12:
        pytest.skip("the fast dense LU is for register-resident sizes")
    lib = _compile(tmp_path, f"dense_{n}_{t}_{int(fast)}", _dense_wrapper(n, t, fast))
    rng = np.random.default_rng(n)
    matrix = rng.normal(size=(n, n))
    matrix[0, 0] *= 0.01                                    # the first pivot is a row swap
    assert abs(matrix[0, 0]) < np.abs(matrix[1:, 0]).max()
    _check(lib.run, matrix, 1e-10 if t == "double" else 1e-3)


def _ring(n):
    m = np.zeros((n, n), dtype=bool)
    for i in range(n):
        m[i, i] = m[i, (i + 1) % n] = m[i, (i - 1) % n] = True
        m[i, (i + n // 2) % n] = True
    return m


@pytest.mark.parametrize("fast", [False, True])
@pytest.mark.parametrize("mode", ["unrolled", "tables"])
@pytest.mark.parametrize("t", ["double", "float"])
def test_generated_sparse_lu_solves(tmp_path, mode, t, fast):
    n = 16
    mask = _ring(n)
    layout = analyse(normalize_sparsity(mask, n), "amd")
    code = emit_cuda(layout, mode, fast=fast)
    source = code + f"""
extern "C" void run(const double* a, const double* b, double* x, int transposed) {{
  static const int slot[{n * n}] = {{{", ".join(str(int(v)) for v in layout.caller_slots().ravel())}}};
  {t} lu[{layout.nnz}]; {t} r[{n}];
  for (int i = 0; i < {layout.nnz}; ++i) lu[i] = 0;
  for (int i = 0; i < {n * n}; ++i) if (slot[i] >= 0) lu[slot[i]] = ({t})a[i];
  mdx_sparse_factorize<{t}>(lu);
  for (int i = 0; i < {n}; ++i) r[i] = ({t})b[i];
  if (transposed) mdx_sparse_solve_t<{t}>(lu, r); else mdx_sparse_solve<{t}>(lu, r);
  for (int i = 0; i < {n}; ++i) x[i] = (double)r[i];
}}
"""
    lib = _compile(tmp_path, f"sparse_{mode}_{t}_{int(fast)}", source)
    rng = np.random.default_rng(5)
    matrix = np.where(mask, rng.normal(size=(n, n)), 0.0) + 8.0 * np.eye(n)
    _check(lib.run, matrix, 1e-10 if t == "double" else 1e-5)
