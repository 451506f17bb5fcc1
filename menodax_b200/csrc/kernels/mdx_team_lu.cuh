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
// pivot row is swapped into place over every column, with the permutation and
// the `pending` multiplier columns fac[m * N + row] (m < pending) that belong to
// the rows.
template <int N, int LDA, typename T>
__device__ __forceinline__ void pivot_swap(T* __restrict__ a, int* __restrict__ perm,
                                           double* __restrict__ fac, const int pending, const int c,
                                           const int lane, const unsigned mask) {
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
      for (int m = 0; m < pending; ++m) {
        const double f = fac[m * N + c];
        fac[m * N + c] = fac[m * N + bi];
        fac[m * N + bi] = f;
      }
    }
  }
  __syncwarp(mask);
}

// Multipliers of column c below the diagonal.  FAST: in T, stored in place, the
// diagonal replaced by its reciprocal (fast_recip).  Otherwise the reference's typing:
// double multipliers kept unrounded in `fac` for the updates, rounded into the
// matrix, nothing done for a zero pivot.  Returns whether updates from column c
// apply.
template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ bool multipliers(T* __restrict__ a, double* __restrict__ fac, const int c,
                                            const int lane, const unsigned mask) {
  const T piv = a[c * LDA + c];
  if constexpr (FAST) {
    const T recip = fast_recip(piv);
    const T inv = piv != T(0) ? recip : T(0);
    for (int r = c + 1 + lane; r < N; r += MDX_TEAM) a[r * LDA + c] *= inv;
    __syncwarp(mask);
    if (lane == 0) a[c * LDA + c] = recip;
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

// Columns are eliminated in panels of W.  Within a panel, column c + k first
// takes the updates of the panel's earlier columns (its rows c+1 .. c+k-1 in
// order on one lane, then its rows from c + k down on all lanes), is pivoted and
// scaled, and row c + k right of the panel takes the earlier columns' updates.
// One pass over the trailing rows then applies the W updates, entry by entry in
// the order the one-column algorithm applies them, so every entry rounds the same
// way as there.  A row swap inside a panel moves un-updated entries together with
// the multipliers that update them.  The pass reads each trailing entry once and
// writes it once for W FMAs, the W multipliers of its row read once for all of a
// lane's columns and the lane's W pivot-row entries held in registers.
//
// FAST keeps no double multipliers and takes W = 4 (W = 2 when a lane's pivot-row
// entries would take too many registers); the reference's arithmetic takes W = 2
// with the two double multiplier columns in `fac`.
template <int N, int LDA, typename T, bool FAST>
__device__ __forceinline__ void dense_factorize(T* __restrict__ a, int* __restrict__ perm,
                                                double* __restrict__ fac, const int lane,
                                                const unsigned mask) {
  constexpr int NB = (N + MDX_TEAM - 1) / MDX_TEAM;
  constexpr int W = (FAST && NB <= 4) ? 4 : 2;
  for (int i = lane; i < N; i += MDX_TEAM) perm[i] = i;
  __syncwarp(mask);
#pragma unroll 1
  for (int c = 0; c < N; c += W) {
    const int w = N - c < W ? N - c : W;
    bool on[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      on[k] = false;
      if (k >= w) continue;
      const int ck = c + k;
      if (k > 0) {
        // Column ck, rows c+1 .. ck-1 (finished rows of U): serial in the row.
        if (lane == 0) {
#pragma unroll
          for (int ii = 1; ii < k; ++ii) {
            const int i = c + ii;
            T x = a[i * LDA + ck];
#pragma unroll
            for (int m = 0; m < ii; ++m)
              if (on[m]) x = eliminate<T, FAST>(x, a[i * LDA + c + m], FAST ? 0.0 : fac[m * N + i], a[(c + m) * LDA + ck]);
            a[i * LDA + ck] = x;
          }
        }
        __syncwarp(mask);
        // Column ck from row ck down: the pivot search reads these.
        for (int r = ck + lane; r < N; r += MDX_TEAM) {
          T x = a[r * LDA + ck];
#pragma unroll
          for (int m = 0; m < k; ++m)
            if (on[m]) x = eliminate<T, FAST>(x, a[r * LDA + c + m], FAST ? 0.0 : fac[m * N + r], a[(c + m) * LDA + ck]);
          a[r * LDA + ck] = x;
        }
        __syncwarp(mask);
      }
      pivot_swap<N, LDA, T>(a, perm, fac, FAST ? 0 : k, ck, lane, mask);
      on[k] = multipliers<N, LDA, T, FAST>(a, FAST ? nullptr : fac + k * N, ck, lane, mask);
      if (k > 0) {
        // Row ck right of the panel.
        for (int j = c + w + lane; j < N; j += MDX_TEAM) {
          T x = a[ck * LDA + j];
#pragma unroll
          for (int m = 0; m < k; ++m)
            if (on[m]) x = eliminate<T, FAST>(x, a[ck * LDA + c + m], FAST ? 0.0 : fac[m * N + ck], a[(c + m) * LDA + j]);
          a[ck * LDA + j] = x;
        }
        __syncwarp(mask);
      }
    }
    // Rows below the panel, columns right of it: the W updates in one pass.
    T u[W][NB];
#pragma unroll
    for (int m = 0; m < W; ++m) {
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int j = c + w + lane + q * MDX_TEAM;
        u[m][q] = (m < w && j < N) ? a[(c + m) * LDA + j] : T(0);
      }
    }
#pragma unroll 2
    for (int r = c + w; r < N; ++r) {
      T l[W];
      double f[W];
#pragma unroll
      for (int m = 0; m < W; ++m) {
        l[m] = m < w ? a[r * LDA + c + m] : T(0);
        f[m] = (FAST || m >= w) ? 0.0 : fac[m * N + r];
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int j = c + w + lane + q * MDX_TEAM;
        if (j < N) {
          T x = a[r * LDA + j];
#pragma unroll
          for (int m = 0; m < W; ++m)
            if (on[m]) x = eliminate<T, FAST>(x, l[m], f[m], u[m][q]);
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
