// Dense LU with partial pivoting for the team kernel: one n x n system per team
// of MDX_TEAM lanes, row-major in shared memory with an odd row stride LDA so a
// walk down a column touches 32 different banks.
//
// Same algorithm as the thread kernel's dense LU (the reference's
// dense_lu_solver, modax/rodas5P.py:167-238): right-looking elimination, the
// first largest-magnitude entry of the column at or below the diagonal as pivot,
// whole-row swaps.  Each entry sees the same operations in the same order as in
// the one-lane version; the lanes only split the work of one elimination step
// (pivot search by rows, multipliers by rows, the rank-one update by columns).
// The row swaps are folded into `perm` (perm[i] = original row now at i), which
// a solve applies as a gather.
//
// FAST (the FP32-LU product path): everything in T, the diagonal left holding
// 1/U_ii.  Otherwise the reference's mixed typing: double multipliers kept
// unrounded in `fac` for the update, U_ii divided in the back substitution.
#pragma once

namespace mdx {
namespace team {

template <typename T>
__device__ __forceinline__ T not_nan_or(T v, T fallback) { return v == v ? v : fallback; }

template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ void dense_factorize(T* __restrict__ a, int* __restrict__ perm,
                                                double* __restrict__ fac, const int lane,
                                                const unsigned mask) {
  for (int i = lane; i < N; i += MDX_TEAM) perm[i] = i;
  __syncwarp(mask);
#pragma unroll 1
  for (int c = 0; c < N; ++c) {
    // Pivot: lane-local first maximum over the lane's rows, then a butterfly
    // that prefers the larger magnitude and, on a tie, the smaller row -- the
    // serial scan's first maximum.  A NaN never wins (the serial scan keeps the
    // diagonal then; the step's error estimate is NaN either way and rejects).
    T best = T(-1);
    int bi = N;
    for (int r = c + lane; r < N; r += MDX_TEAM) {
      const T v = not_nan_or(fabs(a[r * LDA + c]), T(-1));
      if (v > best) { best = v; bi = r; }
    }
#pragma unroll
    for (int off = MDX_TEAM / 2; off > 0; off >>= 1) {
      const T ov = __shfl_xor_sync(mask, best, off, MDX_TEAM);
      const int oi = __shfl_xor_sync(mask, bi, off, MDX_TEAM);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if (bi >= N) bi = c;
    if (bi != c) {
      for (int j = lane; j < N; j += MDX_TEAM) {
        const T x = a[c * LDA + j];
        a[c * LDA + j] = a[bi * LDA + j];
        a[bi * LDA + j] = x;
      }
      if (lane == 0) {
        const int p = perm[c];
        perm[c] = perm[bi];
        perm[bi] = p;
      }
      __syncwarp(mask);
    }
    const T piv = a[c * LDA + c];
    if constexpr (FAST) {
      const T inv = piv != T(0) ? T(1) / piv : T(0);
      for (int r = c + 1 + lane; r < N; r += MDX_TEAM) a[r * LDA + c] *= inv;
      __syncwarp(mask);
      for (int j = c + 1 + lane; j < N; j += MDX_TEAM) {
        const T ucj = a[c * LDA + j];
#pragma unroll 4
        for (int r = c + 1; r < N; ++r) a[r * LDA + j] -= a[r * LDA + c] * ucj;
      }
      __syncwarp(mask);
      if (lane == 0) a[c * LDA + c] = T(1) / piv;
    } else {
      if (piv != T(0)) {
        const double inv = 1.0 / (double)piv;
        for (int r = c + 1 + lane; r < N; r += MDX_TEAM) {
          const double f = (double)a[r * LDA + c] * inv;
          a[r * LDA + c] = (T)f;
          fac[r] = f;
        }
        __syncwarp(mask);
        for (int j = c + 1 + lane; j < N; j += MDX_TEAM) {
          const double ucj = (double)a[c * LDA + j];
#pragma unroll 4
          for (int r = c + 1; r < N; ++r) a[r * LDA + j] = (T)((double)a[r * LDA + j] - fac[r] * ucj);
        }
        __syncwarp(mask);
      }
    }
  }
  __syncwarp(mask);
}

// M x = b in place on x (shared), M = P^T L U.  Rows are taken in blocks of
// MDX_TEAM, lane l owning row b0 + l of block b0: the contributions of earlier
// blocks are a dot product against finished values in shared memory, the
// in-block triangle a chain of shuffles from the lane whose row just finished.
// The forward sweep subtracts in ascending column order, as the serial
// substitution does; the backward sweep takes the later blocks first.
template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ void dense_solve(const T* __restrict__ a, const int* __restrict__ perm,
                                            T* __restrict__ x, const int lane, const unsigned mask) {
  constexpr int NB = (N + MDX_TEAM - 1) / MDX_TEAM;
  T r[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int i = b * MDX_TEAM + lane;
    r[b] = i < N ? x[perm[i]] : T(0);
  }
  __syncwarp(mask);
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int b0 = b * MDX_TEAM;
    const int nb = N - b0 < MDX_TEAM ? N - b0 : MDX_TEAM;
    const int i = b0 + lane;
    const bool live = i < N;
    T acc = r[b];
    if (live) {
      const T* row = a + i * LDA;
      for (int j = 0; j < b0; ++j) acc -= row[j] * x[j];
    }
#pragma unroll
    for (int jj = 0; jj < MDX_TEAM; ++jj) {
      if (jj < nb) {
        const T xj = __shfl_sync(mask, acc, jj, MDX_TEAM);
        if (live && lane > jj) acc -= a[i * LDA + b0 + jj] * xj;
      }
    }
    if (live) x[i] = acc;
    r[b] = acc;
    __syncwarp(mask);
  }
#pragma unroll
  for (int b = NB - 1; b >= 0; --b) {
    const int b0 = b * MDX_TEAM;
    const int nb = N - b0 < MDX_TEAM ? N - b0 : MDX_TEAM;
    const int i = b0 + lane;
    const bool live = i < N;
    T acc = r[b];
    if (live) {
      const T* row = a + i * LDA;
      for (int j = b0 + nb; j < N; ++j) acc -= row[j] * x[j];
    }
#pragma unroll
    for (int jj = MDX_TEAM - 1; jj >= 0; --jj) {
      if (jj < nb) {
        if (lane == jj) {
          if constexpr (FAST) acc = acc * a[i * LDA + i];
          else acc = acc / a[i * LDA + i];
        }
        const T xj = __shfl_sync(mask, acc, jj, MDX_TEAM);
        if (live && lane < jj) acc -= a[i * LDA + b0 + jj] * xj;
      }
    }
    if (live) x[i] = acc;
    __syncwarp(mask);
  }
}

}  // namespace team
}  // namespace mdx
