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
// unrounded in `fac` (two columns of them, 2N doubles) for the updates, U_ii
// divided in the back substitution.
#pragma once

namespace mdx {
namespace team {

template <typename T>
__device__ __forceinline__ T not_nan_or(T v, T fallback) { return v == v ? v : fallback; }

// Pivot of column c: lane-local first maximum over the lane's rows, then a
// butterfly that prefers the larger magnitude and, on a tie, the smaller row --
// the serial scan's first maximum.  A NaN never wins (the serial scan keeps the
// diagonal then; the step's error estimate is NaN either way and rejects).  The
// pivot row is swapped into place over every column, with the permutation and,
// when given, a pending multiplier column `fac0` that belongs to the rows.
template <int N, int LDA, typename T>
__device__ __forceinline__ void pivot_swap(T* __restrict__ a, int* __restrict__ perm,
                                           double* __restrict__ fac0, const int c, const int lane,
                                           const unsigned mask) {
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
      if (fac0) {
        const double f = fac0[c];
        fac0[c] = fac0[bi];
        fac0[bi] = f;
      }
    }
  }
  __syncwarp(mask);
}

// Multipliers of column c below the diagonal.  FAST: in T, stored in place, the
// diagonal replaced by its reciprocal.  Otherwise the reference's typing:
// double multipliers kept unrounded in `fac` for the updates, rounded into the
// matrix, nothing done for a zero pivot.  Returns whether updates from column c
// apply.
template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ bool multipliers(T* __restrict__ a, double* __restrict__ fac, const int c,
                                            const int lane, const unsigned mask) {
  const T piv = a[c * LDA + c];
  if constexpr (FAST) {
    const T inv = piv != T(0) ? T(1) / piv : T(0);
    for (int r = c + 1 + lane; r < N; r += MDX_TEAM) a[r * LDA + c] *= inv;
    __syncwarp(mask);
    if (lane == 0) a[c * LDA + c] = T(1) / piv;
    return true;
  } else {
    if (piv == T(0)) return false;
    const double inv = 1.0 / (double)piv;
    for (int r = c + 1 + lane; r < N; r += MDX_TEAM) {
      const double f = (double)a[r * LDA + c] * inv;
      a[r * LDA + c] = (T)f;
      fac[r] = f;
    }
    __syncwarp(mask);
    return true;
  }
}

// One elimination update a - l * u of an entry, with the rounding of the path.
template <typename T, bool FAST>
__device__ __forceinline__ T eliminate(T x, T l, double f, T u) {
  if constexpr (FAST) {
    return x - l * u;
  } else {
    return (T)((double)x - f * (double)u);
  }
}

// Columns are eliminated two at a time.  Column c is pivoted and scaled; its
// update is applied at once only to column c + 1 (which the next pivot search
// reads); column c + 1 is pivoted and scaled; row c + 1 takes column c's update;
// then one pass over the trailing rows applies both updates, entry by entry in
// the order the one-column algorithm applies them, so every entry rounds the same
// way.  A row swap between the two steps moves un-updated trailing entries
// together with the multipliers that update them.  The pass reads each trailing
// entry once and writes it once for two FMAs, with the two multipliers of its row
// read once for all of a lane's columns and the lane's two pivot-row entries held
// in registers -- half the shared-memory traffic per FMA of a one-column pass.
template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ void dense_factorize(T* __restrict__ a, int* __restrict__ perm,
                                                double* __restrict__ fac, const int lane,
                                                const unsigned mask) {
  constexpr int NB = (N + MDX_TEAM - 1) / MDX_TEAM;
  double* fac0 = FAST ? nullptr : fac;
  double* fac1 = FAST ? nullptr : fac + N;
  for (int i = lane; i < N; i += MDX_TEAM) perm[i] = i;
  __syncwarp(mask);
#pragma unroll 1
  for (int c = 0; c < N; c += 2) {
    pivot_swap<N, LDA, T>(a, perm, nullptr, c, lane, mask);
    const bool on0 = multipliers<N, LDA, T, FAST>(a, fac0, c, lane, mask);
    if (c + 1 >= N) break;
    const int c1 = c + 1;
    // Column c + 1 below row c takes column c's update.
    if (on0) {
      const T u = a[c * LDA + c1];
      for (int r = c1 + lane; r < N; r += MDX_TEAM)
        a[r * LDA + c1] = eliminate<T, FAST>(a[r * LDA + c1], a[r * LDA + c], FAST ? 0.0 : fac0[r], u);
    }
    __syncwarp(mask);
    pivot_swap<N, LDA, T>(a, perm, fac0, c1, lane, mask);
    const bool on1 = multipliers<N, LDA, T, FAST>(a, fac1, c1, lane, mask);
    // Row c + 1 right of the pair takes column c's update.
    if (on0) {
      const T l = a[c1 * LDA + c];
      const double f = FAST ? 0.0 : fac0[c1];
      for (int j = c1 + 1 + lane; j < N; j += MDX_TEAM)
        a[c1 * LDA + j] = eliminate<T, FAST>(a[c1 * LDA + j], l, f, a[c * LDA + j]);
    }
    __syncwarp(mask);
    // Rows below the pair, columns right of it: both updates in one pass.
    T u0[NB], u1[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int j = c1 + 1 + lane + q * MDX_TEAM;
      u0[q] = j < N ? a[c * LDA + j] : T(0);
      u1[q] = j < N ? a[c1 * LDA + j] : T(0);
    }
#pragma unroll 2
    for (int r = c1 + 1; r < N; ++r) {
      const T l0 = a[r * LDA + c];
      const T l1 = a[r * LDA + c1];
      const double f0 = FAST ? 0.0 : fac0[r];
      const double f1 = FAST ? 0.0 : fac1[r];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int j = c1 + 1 + lane + q * MDX_TEAM;
        if (j < N) {
          T x = a[r * LDA + j];
          if (on0) x = eliminate<T, FAST>(x, l0, f0, u0[q]);
          if (on1) x = eliminate<T, FAST>(x, l1, f1, u1[q]);
          a[r * LDA + j] = x;
        }
      }
    }
    __syncwarp(mask);
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
