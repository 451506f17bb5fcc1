// Dense LU with partial pivoting, one n x n system per thread, row-major.
//
// The algorithm is the reference's dense_lu_solver (modax/rodas5P.py:167-238):
// right-looking elimination, the largest remaining entry of the column as pivot,
// whole-row swaps recorded in ipiv, a zero pivot left alone (the Rosenbrock-W
// step controller rejects what comes out of it).  Arithmetic follows the
// reference's mixed typing: the multipliers and the rank-one update are formed in
// double and stored in the LU type T; the substitutions run in T.
//
// For N <= MDX_DENSE_UNROLL_MAX every index is a compile-time constant: the row
// swaps become predicated selects over the candidate rows, so the matrix stays in
// registers.  Larger systems use plain loops and the compiler places the matrix in
// local memory.
#pragma once

#ifndef MDX_DENSE_UNROLL_MAX
#define MDX_DENSE_UNROLL_MAX 12
#endif

namespace mdx {

template <typename T>
__device__ __forceinline__ void swap_vals(T& a, T& b) { T c = a; a = b; b = c; }

template <int N, typename T, class LU, class IP>
__device__ __forceinline__ void dense_factorize_unrolled(LU& lu, IP& ipiv) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T max_val = fabs(lu[i * N + i]);
    int pivot = i;
#pragma unroll
    for (int k = i + 1; k < N; ++k) {
      const T v = fabs(lu[k * N + i]);
      if (v > max_val) { max_val = v; pivot = k; }
    }
    ipiv[i] = pivot;
#pragma unroll
    for (int k = i + 1; k < N; ++k) {
      if (pivot == k) {
#pragma unroll
        for (int j = 0; j < N; ++j) swap_vals(lu[i * N + j], lu[k * N + j]);
      }
    }
    const T piv = lu[i * N + i];
    if (piv != T(0)) {
      const double inv_piv = 1.0 / (double)piv;
#pragma unroll
      for (int k = i + 1; k < N; ++k) {
        const double factor = (double)lu[k * N + i] * inv_piv;
        lu[k * N + i] = (T)factor;
#pragma unroll
        for (int j = i + 1; j < N; ++j)
          lu[k * N + j] = (T)((double)lu[k * N + j] - factor * (double)lu[i * N + j]);
      }
    }
  }
}

template <int N, typename T, class LU, class IP>
__device__ __forceinline__ void dense_factorize_loops(LU& lu, IP& ipiv) {
#pragma unroll 1
  for (int i = 0; i < N; ++i) {
    T max_val = fabs(lu[i * N + i]);
    int pivot = i;
    for (int k = i + 1; k < N; ++k) {
      const T v = fabs(lu[k * N + i]);
      if (v > max_val) { max_val = v; pivot = k; }
    }
    ipiv[i] = pivot;
    if (pivot != i) {
      for (int j = 0; j < N; ++j) swap_vals(lu[i * N + j], lu[pivot * N + j]);
    }
    const T piv = lu[i * N + i];
    if (piv != T(0)) {
      const double inv_piv = 1.0 / (double)piv;
#pragma unroll 1
      for (int k = i + 1; k < N; ++k) {
        const double factor = (double)lu[k * N + i] * inv_piv;
        lu[k * N + i] = (T)factor;
#pragma unroll 4
        for (int j = i + 1; j < N; ++j)
          lu[k * N + j] = (T)((double)lu[k * N + j] - factor * (double)lu[i * N + j]);
      }
    }
  }
}

template <int N, typename T, class LU, class IP>
__device__ __forceinline__ void dense_factorize(LU& lu, IP& ipiv) {
  if constexpr (N <= MDX_DENSE_UNROLL_MAX) dense_factorize_unrolled<N, T>(lu, ipiv);
  else dense_factorize_loops<N, T>(lu, ipiv);
}

// M x = rhs in place: forward through L applying the pivots as they come, then
// back through U (modax/rodas5P.py:218-236).
template <int N, typename T, class LU, class IP, class R>
__device__ __forceinline__ void dense_solve(const LU& lu, const IP& ipiv, R& rhs) {
  if constexpr (N <= MDX_DENSE_UNROLL_MAX) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int pivot = ipiv[i];
#pragma unroll
      for (int k = i + 1; k < N; ++k)
        if (pivot == k) swap_vals(rhs[i], rhs[k]);
      T acc = rhs[i];
#pragma unroll
      for (int j = 0; j < i; ++j) acc -= lu[i * N + j] * rhs[j];
      rhs[i] = acc;
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
      T acc = rhs[i];
#pragma unroll
      for (int j = i + 1; j < N; ++j) acc -= lu[i * N + j] * rhs[j];
      rhs[i] = acc / lu[i * N + i];
    }
  } else {
#pragma unroll 1
    for (int i = 0; i < N; ++i) {
      const int pivot = ipiv[i];
      if (pivot != i) swap_vals(rhs[i], rhs[pivot]);
      T acc = rhs[i];
      for (int j = 0; j < i; ++j) acc -= lu[i * N + j] * rhs[j];
      rhs[i] = acc;
    }
#pragma unroll 1
    for (int i = N - 1; i >= 0; --i) {
      T acc = rhs[i];
      for (int j = i + 1; j < N; ++j) acc -= lu[i * N + j] * rhs[j];
      rhs[i] = acc / lu[i * N + i];
    }
  }
}

// M^T x = rhs in place, for the discrete adjoint.  With M = P^-1 L U (P the
// product of the recorded row swaps): U^T z = rhs, L^T w = z, then the swaps
// undone in reverse order.
template <int N, typename T, class LU, class IP, class R>
__device__ __forceinline__ void dense_solve_t(const LU& lu, const IP& ipiv, R& rhs) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T acc = rhs[i];
#pragma unroll
    for (int k = 0; k < i; ++k) acc -= lu[k * N + i] * rhs[k];
    rhs[i] = acc / lu[i * N + i];
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    T acc = rhs[i];
#pragma unroll
    for (int k = i + 1; k < N; ++k) acc -= lu[k * N + i] * rhs[k];
    rhs[i] = acc;
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    const int pivot = ipiv[i];
    if constexpr (N <= MDX_DENSE_UNROLL_MAX) {
#pragma unroll
      for (int k = i + 1; k < N; ++k)
        if (pivot == k) swap_vals(rhs[i], rhs[k]);
    } else {
      if (pivot != i) swap_vals(rhs[i], rhs[pivot]);
    }
  }
}

// --- fast arithmetic (MDX_FAST): the FP32-LU path of the persistent kernel ------
// The factorisation runs entirely in T (no double multipliers, no conversions),
// the row swaps are folded into a permutation `perm` (perm[i] = the original
// row that ends at position i) so a solve permutes its right-hand side with
// selects instead of branches, and the diagonal is left holding 1/U_ii (the
// approximate reciprocal fast_recip) so the back substitution multiplies.  Same algorithm, different rounding: the FP32
// path is held to accuracy against the FP64 oracle, not to the reference's bits.
template <int N, typename T, class LU, class IP>
__device__ __forceinline__ void dense_factorize_fast(LU& lu, IP& perm) {
  static_assert(N <= MDX_DENSE_UNROLL_MAX, "the fast dense LU is for register-resident systems");
#pragma unroll
  for (int i = 0; i < N; ++i) perm[i] = i;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T max_val = fabs(lu[i * N + i]);
    int pivot = i;
#pragma unroll
    for (int k = i + 1; k < N; ++k) {
      const T v = fabs(lu[k * N + i]);
      if (v > max_val) { max_val = v; pivot = k; }
    }
#pragma unroll
    for (int k = i + 1; k < N; ++k) {
      const bool sw = pivot == k;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const T a = lu[i * N + j], b = lu[k * N + j];
        lu[i * N + j] = sw ? b : a;
        lu[k * N + j] = sw ? a : b;
      }
      const int pa = perm[i], pb = perm[k];
      perm[i] = sw ? pb : pa;
      perm[k] = sw ? pa : pb;
    }
    const T piv = lu[i * N + i];
    const T recip = fast_recip(piv);
    const T inv_piv = piv != T(0) ? recip : T(0);
#pragma unroll
    for (int k = i + 1; k < N; ++k) {
      const T factor = lu[k * N + i] * inv_piv;
      lu[k * N + i] = factor;
#pragma unroll
      for (int j = i + 1; j < N; ++j) lu[k * N + j] -= factor * lu[i * N + j];
    }
    lu[i * N + i] = recip;
  }
}

template <int N, typename T, class LU, class IP, class R>
__device__ __forceinline__ void dense_solve_fast(const LU& lu, const IP& perm, R& rhs) {
  T x[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T v = rhs[0];
#pragma unroll
    for (int k = 1; k < N; ++k) v = perm[i] == k ? rhs[k] : v;
    x[i] = v;
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T acc = x[i];
#pragma unroll
    for (int j = 0; j < i; ++j) acc -= lu[i * N + j] * x[j];
    x[i] = acc;
  }
  // Back substitution takes each row's terms latest-solved last (descending
  // column), so a row waits on one FMA after its last input.
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    T acc = x[i];
#pragma unroll
    for (int j = N - 1; j > i; --j) acc -= lu[i * N + j] * x[j];
    x[i] = acc * lu[i * N + i];
  }
#pragma unroll
  for (int i = 0; i < N; ++i) rhs[i] = x[i];
}

// Transposed solve for the fast factorisation: M^T x = b with M = P^T L U.
template <int N, typename T, class LU, class IP, class R>
__device__ __forceinline__ void dense_solve_t_fast(const LU& lu, const IP& perm, R& rhs) {
  T z[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T acc = rhs[i];
#pragma unroll
    for (int k = 0; k < i; ++k) acc -= lu[k * N + i] * z[k];
    z[i] = acc * lu[i * N + i];
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    T acc = z[i];
#pragma unroll
    for (int k = i + 1; k < N; ++k) acc -= lu[k * N + i] * z[k];
    z[i] = acc;
  }
  // x[perm[i]] = z[i]
#pragma unroll
  for (int j = 0; j < N; ++j) {
    T v = z[0];
#pragma unroll
    for (int i = 1; i < N; ++i) v = perm[i] == j ? z[i] : v;
    rhs[j] = perm[0] == j ? z[0] : v;
  }
}

}  // namespace mdx
