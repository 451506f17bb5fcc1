// Shared device helpers for the ensemble ODE kernels (sm_100a, NVRTC-compiled).
//
// Every kernel runs one trajectory per thread.  A problem header generated on
// the host (menodax_b200/_codegen.py) defines the sizes, the traced right-hand
// side and its derivatives as force-inlined templates; with every component
// index a compile-time constant the per-trajectory vectors live in registers.
#pragma once
#include "mdx_args.h"

#define MDX_FULL_MASK 0xffffffffu

#ifndef MDX_TPB
#define MDX_TPB 32
#endif
#ifndef MDX_MIN_BLOCKS
#define MDX_MIN_BLOCKS 1
#endif

namespace mdx {

// Python's max(a, b) on floats: the first argument unless the second is larger.
// It differs from fmax only on NaN, where the reference's comparison semantics
// (modax/rodas5P.py:907, modax/tsit5.py:297) are kept.
__device__ __forceinline__ double pymax(double a, double b) { return b > a ? b : a; }

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

__device__ __forceinline__ double nan_value() { return __longlong_as_double(0x7ff8000000000000LL); }

// x^e for the step-size factor in the fast path: the factor is a heuristic that
// is clamped to [0.2, 6] and multiplied by 0.9, so float precision (relative
// error ~1e-6) is ample; __powf is two special-function-unit instructions.
__device__ __forceinline__ double fast_pow(double x, double e) {
  return (double)__powf((float)x, (float)e);
}

// 1/x for the fast path's LU pivots.  In single precision the approximate
// reciprocal (__fdividef: within 2 ulp for |x| in [2^-126, 2^126], 1/0 = inf),
// whose error is below the FP32 factorisation's own rounding; double pivots keep
// the IEEE division.
__device__ __forceinline__ float fast_recip(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double fast_recip(double x) { return 1.0 / x; }

// 1/s in double for the fast path (the step's 1/h, the error scales): the
// single-precision reciprocal as a seed, refined by one Newton-Raphson step
// y <- y + y (1 - s y), which squares the seed's relative error (~1e-7 ->
// ~1e-14).  Values outside float's normal range keep the IEEE division.
__device__ __forceinline__ double recip_newton(double s) {
  if (s >= 1e-37 && s <= 1e37) {
    const double y = (double)__fdividef(1.0f, (float)s);
    return fma(y, fma(-s, y, 1.0), y);
  }
  return 1.0 / s;
}

// Step-size controller (modax/rodas5P.py:913-928, modax/tsit5.py:383-398):
// clamp the error into [1e-18, 1e18] (NaN counts as huge), form the PID factor
// from the error history, and clamp the factor.  E2 and E3 are compile-time
// constants, so the default I-controller multiplies by nothing extra.
__device__ __forceinline__ double controller_factor(double err_norm, double err_prev, double err_prev2,
                                                    double e1, double e2, double e3, bool use_e2,
                                                    bool use_e3, double& safe_err) {
  if (isnan(err_norm) || err_norm > 1e18) {
    safe_err = 1e18;
  } else if (err_norm == 0.0) {
    safe_err = 1e-18;
  } else {
    safe_err = err_norm;
  }
  double factor = 0.9 * pow(safe_err, e1);
  if (use_e2) factor = factor * pow(err_prev, e2);
  if (use_e3) factor = factor * pow(err_prev2, e3);
  return factor;
}

// The fast path's controller on the SQUARED weighted RMS error: the step is
// accepted on err^2 <= 1 and err^e = (err^2)^(e/2), so no square root is taken.
// The error history is kept squared too.  The clamp is [1e-36, 1e36] on err^2
// (the reference's [1e-18, 1e18] on err), applied below as well as at zero so
// that every power is taken of a normal float.
__device__ __forceinline__ double controller_factor_sq(double err_sq, double prev_sq, double prev2_sq,
                                                       double e1, double e2, double e3, bool use_e2,
                                                       bool use_e3, double& safe_sq) {
  if (isnan(err_sq) || err_sq > 1e36) {
    safe_sq = 1e36;
  } else if (err_sq < 1e-36) {
    safe_sq = 1e-36;
  } else {
    safe_sq = err_sq;
  }
  double factor = 0.9 * fast_pow(safe_sq, 0.5 * e1);
  if (use_e2) factor = factor * fast_pow(prev_sq, 0.5 * e2);
  if (use_e3) factor = factor * fast_pow(prev2_sq, 0.5 * e3);
  return factor;
}

// True when save time `ts` is reached by a step ending at `t_new`
// (modax/rodas5P.py:933-935): the 1e-12 relative slack keeps a save that
// rounding puts a hair past the end of the step from being missed.
__device__ __forceinline__ bool save_reached(double ts, double t_new) {
  return ts <= t_new + 1e-12 * pymax(1.0, fabs(ts));
}

#ifndef MDX_CKPT_SEG
#define MDX_CKPT_SEG 1
#endif

// Checkpoint layout of a MDX_CHECKPOINT solve: every accepted step's size h at
// ckpt[m * N + traj]; every MDX_CKPT_SEG-th step's start (t, y) as a record of
// n_vars + 1 doubles after them, segment-major so a warp in lockstep writes
// contiguous runs.  The reverse pass replays a segment from its start state.
__device__ __forceinline__ double* ckpt_state(double* ckpt, long long capacity, int n_traj, int seg, int traj) {
  return ckpt + (size_t)capacity * (size_t)n_traj +
         ((size_t)seg * (size_t)n_traj + (size_t)traj) * (size_t)(MDX_NV + 1);
}

template <class Y>
__device__ __forceinline__ void ckpt_write(const MdxSolveArgs& a, int traj, int m, double t, double h, const Y& y) {
  a.ckpt[(size_t)m * (size_t)a.n_traj + (size_t)traj] = h;
  if (m % MDX_CKPT_SEG == 0) {
    double* rec = ckpt_state(a.ckpt, a.ckpt_capacity, a.n_traj, m / MDX_CKPT_SEG, traj);
    rec[0] = t;
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) rec[1 + j] = y[j];
  }
}

}  // namespace mdx
