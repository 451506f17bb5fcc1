// Rodas5P (Rosenbrock-W, order 5), one trajectory per thread.
//
// Restates the reference kernel's step (modax/rodas5P.py:761-1005) as a
// state/step/finish triple so the same step body serves the one-launch kernel
// (one trajectory per thread for its whole life) and the persistent refill
// kernel (mdx_persistent.cuh), where a lane that finishes takes the next
// trajectory off a queue.
//
// Per step: -J and df/dt from the traced right-hand side (one forward sweep per
// colour, plus one in t), M = I/(h*gamma) - J on the diagonal slots, one LU, and
// eight stages "f -> stage right-hand side -> solve" against it; the error
// estimate is the eighth stage; PID control; dense output on accept.
//
// Precision split (modax/rodas5P.py:347-349, 713, 724): the state, f, J, the
// stage combinations, the error and the controller are double; the matrix, the
// solver's right-hand side and the stored stage increments k are MDX_LU_T.
//
// The problem header included before this file defines the sizes and the
// traced functions mdx_rhs / mdx_neg_jac / mdx_factorize / mdx_solve (and, with
// forward sensitivities, mdx_sens_coupling).
#pragma once
#include "mdx_common.cuh"
#include "mdx_rodas5p_coef.cuh"

namespace mdx {
namespace rodas5p {

typedef MDX_LU_T lu_t;
// A right-hand side with no explicit t dependence has df/dt = 0: its stages
// skip the h d_s df/dt terms, which are exact zeros added to the stage sums.
#ifndef MDX_AUTONOMOUS
#define MDX_AUTONOMOUS 0
#endif
// The triangular solves' type.  The reference solves in the LU type and rounds
// the stage increments to it (k_stages, modax/rodas5P.py:724), and so does the
// reference arithmetic here.  A fast-arithmetic build with MDX_WIDE_SOLVE (the
// host sets it for systems of up to 8 states, and for larger ones where it
// measured faster) factorises in FP32 as well but solves in double against the
// factors, widened once per step: one conversion per factor entry instead of
// two per component and stage, which on the B200's half-rate FP64 pipe costs
// less than the conversions it replaces, and the stages keep their full double
// values.
#ifndef MDX_SOLVE_T
#define MDX_SOLVE_T MDX_LU_T
#endif
#ifndef MDX_WIDE_SOLVE
#define MDX_WIDE_SOLVE 0
#endif
typedef MDX_SOLVE_T sol_t;
// Stage increments: small systems keep them in double registers (the rounded
// values, or the wide solve's own), larger ones in the LU type unless the
// solve is wide.
#if MDX_NS <= 8 || MDX_WIDE_SOLVE
typedef double k_t;
#else
typedef lu_t k_t;
#endif

// The matrix the stages solve against: the factors themselves, or their
// widened copy.
template <class LU, class SLU>
__device__ __forceinline__ void widen_factors(const LU& lu, SLU& lus) {
#pragma unroll
  for (int i = 0; i < MDX_LU_SIZE; ++i) lus[i] = (sol_t)lu[i];
}

struct State {
  double y[MDX_NS];
  double p[MDX_NP > 0 ? MDX_NP : 1];
  double t, dt, err_prev, err_prev2, tf_local;
  int save_idx, n_steps, accepted, rejected, traj;
#if MDX_CHECKPOINT
  int n_ckpt;
  bool ckpt_overflow;
#endif
};

__device__ __forceinline__ size_t hist_index(const MdxSolveArgs& a, int traj, int s, int j) {
  return ((size_t)traj * (size_t)a.n_save_hist + (size_t)s) * (size_t)MDX_NS + (size_t)j;
}

__device__ __forceinline__ double weight(const MdxSolveArgs& a, int traj, int j) {
#if MDX_WEIGHTS_RUNTIME
  return a.weights[(size_t)traj * MDX_NS + j];
#else
  return mdx_const_weight(j);
#endif
}

__device__ __forceinline__ void init(State& st, const MdxSolveArgs& a, int traj) {
  st.traj = traj;
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) st.y[j] = a.y0[(size_t)traj * MDX_NS + j];
#if MDX_SAVE_HISTORY
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) a.hist[hist_index(a, traj, 0, j)] = st.y[j];
#endif
#pragma unroll
  for (int k = 0; k < MDX_NP; ++k) st.p[k] = a.params[(size_t)traj * MDX_NP + k];
  const double t0 = a.times[0];
  const double tf = a.times[a.n_save - 1];
  st.t = t0;
  st.dt = a.dt0 > 0.0 ? a.dt0 : (tf - t0) * 1e-6;
  st.save_idx = 1;
  st.n_steps = 0;
  st.accepted = 0;
  st.rejected = 0;
  st.err_prev = 1.0;
  st.err_prev2 = 1.0;
#if MDX_TF_INDEX >= 0
  st.tf_local = st.p[MDX_TF_INDEX];
#else
  st.tf_local = tf;
#endif
#if MDX_CHECKPOINT
  st.n_ckpt = 0;
  st.ckpt_overflow = false;
#endif
#if MDX_HAS_HOOK
  // The hook's row starts at zero and accumulates over the trajectory's saves
  // (modax/rodas5P.py:753-756).
  double* acc = a.hook_out + (size_t)traj * MDX_HOOK_SIZE;
#pragma unroll 1
  for (int j = 0; j < MDX_HOOK_SIZE; ++j) acc[j] = 0.0;
  mdx_save_hook(0, st.y, t0, st.p, acc);
#endif
}

__device__ __forceinline__ bool running(const State& st, const MdxSolveArgs& a) {
  return st.save_idx < a.n_save && st.t < st.tf_local && st.n_steps < a.max_steps;
}

// One Rosenbrock stage: its right-hand side from the tableau row, then the
// solve against the step's factorisation.  State rows go to the solver's
// buffer; with forward sensitivities the sensitivity rows wait in `work` until
// the coupling term L_k k_y of their block is known (modax/rodas5P.py:513-583).
template <int S, class LU, class IP, class K, class W, class DT, class RB>
__device__ __forceinline__ void stage(const LU& lu, const IP& ipiv, RB& rhs, K& k, W& work,
                                      const DT& dT, const State& st, double dt_use,
                                      double inv_dt) {
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) {
    double value;
    if constexpr (S == 0) {
      if constexpr (MDX_AUTONOMOUS) value = work[j];
      else value = work[j] + dt_use * coef_d(0) * dT[j];
    } else {
      double acc = coef_c(S, 0) * (double)k[0][j];
#pragma unroll
      for (int m = 1; m < S; ++m) acc += coef_c(S, m) * (double)k[m][j];
      if constexpr (coef_d(S) != 0.0 && !MDX_AUTONOMOUS) {
        value = work[j] + dt_use * coef_d(S) * dT[j] + acc * inv_dt;
      } else {
        value = work[j] + acc * inv_dt;
      }
    }
    if (j < MDX_NV) rhs[j] = (sol_t)value;
    else work[j] = value;
  }
  mdx_solve(lu, ipiv, rhs);
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) k[S][j] = (k_t)rhs[j];
#if MDX_NSENS > 0
  double kstate[MDX_NV];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) kstate[j] = (double)k[S][j];
  double coupling[MDX_NSENS * MDX_NV];
  mdx_sens_coupling(st.y, st.t, st.p, kstate, coupling);
#pragma unroll
  for (int s = 0; s < MDX_NSENS; ++s) {
    const int base = MDX_NV + s * MDX_NV;
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) rhs[j] = (sol_t)(work[base + j] + coupling[s * MDX_NV + j]);
    mdx_solve(lu, ipiv, rhs);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) k[S][base + j] = (k_t)rhs[j];
  }
#endif
}

template <int S, class U, class K>
__device__ __forceinline__ void advance(U& u, const State& st, const K& k) {
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) {
    double acc = coef_a(S, 0) * (double)k[0][j];
#pragma unroll
    for (int m = 1; m <= S; ++m) acc += coef_a(S, m) * (double)k[m][j];
    u[j] = st.y[j] + acc;
  }
}

// 1/h and 1/(h gamma) of a step; the discrete adjoint recomputes steps with
// the same two numbers.
__device__ __forceinline__ void step_reciprocals(double h, double& inv_dt, double& dtgamma_inv) {
#if MDX_FAST
  inv_dt = recip_newton(h);
  dtgamma_inv = inv_dt * (1.0 / GAMMA);
#else
  inv_dt = 1.0 / h;
  dtgamma_inv = 1.0 / (h * GAMMA);
#endif
}

__device__ __forceinline__ void step(State& st, const MdxSolveArgs& a) {
  double dt_use = st.dt;
  if (dt_use > st.tf_local - st.t) dt_use = st.tf_local - st.t;
  if (dt_use < 1e-30) dt_use = 1e-30;
  const double t = st.t;
  const double t_end = t + dt_use;
  double inv_dt, dtgamma_inv;
  step_reciprocals(dt_use, inv_dt, dtgamma_inv);

  lu_t lu[MDX_LU_SIZE];
  int ipiv[MDX_IPIV];
  double dT[MDX_NS];
  mdx_neg_jac(st.y, t, st.p, lu, dT);
#pragma unroll
  for (int d = 0; d < MDX_NV; ++d) lu[mdx_diag_slot(d)] += (lu_t)dtgamma_inv;
  mdx_factorize(lu, ipiv);
#if MDX_WIDE_SOLVE
  sol_t lus[MDX_LU_SIZE];
  widen_factors(lu, lus);
#else
  lu_t (&lus)[MDX_LU_SIZE] = lu;
#endif

  sol_t rhs[MDX_NV];
  k_t k[8][MDX_NS];
  double u[MDX_NS];
  double work[MDX_NS];

  mdx_rhs(st.y, t, st.p, work);
  stage<0>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
  advance<0>(u, st, k);
  mdx_rhs(u, t + coef_ct(0) * dt_use, st.p, work);
  stage<1>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
  advance<1>(u, st, k);
  mdx_rhs(u, t + coef_ct(1) * dt_use, st.p, work);
  stage<2>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
  advance<2>(u, st, k);
  mdx_rhs(u, t + coef_ct(2) * dt_use, st.p, work);
  stage<3>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
  advance<3>(u, st, k);
  mdx_rhs(u, t + coef_ct(3) * dt_use, st.p, work);
  stage<4>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
  advance<4>(u, st, k);
  mdx_rhs(u, t_end, st.p, work);
  stage<5>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) u[j] += (double)k[5][j];
  mdx_rhs(u, t_end, st.p, work);
  stage<6>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) u[j] += (double)k[6][j];
  mdx_rhs(u, t_end, st.p, work);
  stage<7>(lus, ipiv, rhs, k, work, dT, st, dt_use, inv_dt);

  // Weighted RMS of the embedded error estimate k8 (modax/rodas5P.py:903-911).
  double err_local = 0.0;
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) {
    const double y_new_j = u[j] + (double)k[7][j];
    const double scale = a.atol + a.rtol * pymax(fabs(st.y[j]), fabs(y_new_j));
#if MDX_FAST
    const double r = weight(a, st.traj, j) * (double)k[7][j] * recip_newton(scale);
#else
    const double r = weight(a, st.traj, j) * (double)k[7][j] / scale;
#endif
    err_local += r * r;
  }
  double safe_err;
#if MDX_FAST
  // Squared norm and history (controller_factor_sq): no square root.
  const double err_sq = err_local * (1.0 / MDX_NERR);
  const bool accept = err_sq <= 1.0;
  double factor = controller_factor_sq(err_sq, st.err_prev, st.err_prev2, MDX_E1, MDX_E2, MDX_E3,
                                       MDX_USE_E2, MDX_USE_E3, safe_err);
#else
  const double err_norm = sqrt(err_local / MDX_NERR);
  const bool accept = err_norm <= 1.0 && !isnan(err_norm);
  double factor = controller_factor(err_norm, st.err_prev, st.err_prev2, MDX_E1, MDX_E2, MDX_E3,
                                    MDX_USE_E2, MDX_USE_E3, safe_err);
#endif
  if (accept) {
    st.err_prev2 = st.err_prev;
    st.err_prev = safe_err;
  }
  if (factor < FACTOR_MIN) factor = FACTOR_MIN;
  else if (factor > FACTOR_MAX) factor = FACTOR_MAX;
  st.dt = dt_use * factor;

  if (accept) {
#if MDX_CHECKPOINT
    if (st.n_ckpt < a.ckpt_capacity) {
      ckpt_write(a, st.traj, st.n_ckpt, t, dt_use, st.y);
      ++st.n_ckpt;
    } else {
      st.ckpt_overflow = true;
    }
#endif
    const double t_new = t + dt_use;
    while (st.save_idx < a.n_save && save_reached(a.times[st.save_idx], t_new)) {
#if MDX_FAST
      const double theta = (a.times[st.save_idx] - t) * inv_dt;
#else
      const double theta = (a.times[st.save_idx] - t) / dt_use;
#endif
      const double theta1 = 1.0 - theta;
#if MDX_FAST
      // h1 + theta (h2 + theta h3) = sum_m w_m k_m, w_m = H0m + theta (H1m + theta H2m):
      // eight weights shared by every component.  A warp runs this whenever any
      // of its lanes passes a save time, which is most steps.
      double w[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) w[m] = coef_h(0, m) + theta * (coef_h(1, m) + theta * coef_h(2, m));
#endif
#if MDX_HAS_HOOK
      double y_save[MDX_NS];
#endif
#pragma unroll
      for (int j = 0; j < MDX_NS; ++j) {
#if MDX_FAST
        double hsum = w[0] * (double)k[0][j];
#pragma unroll
        for (int m = 1; m < 8; ++m) hsum += w[m] * (double)k[m][j];
        const double y_new_j = u[j] + (double)k[7][j];
        const double val = theta1 * st.y[j] + theta * (y_new_j + theta1 * hsum);
#else
        double h1 = coef_h(0, 0) * (double)k[0][j];
        double h2 = coef_h(1, 0) * (double)k[0][j];
        double h3 = coef_h(2, 0) * (double)k[0][j];
#pragma unroll
        for (int m = 1; m < 8; ++m) {
          h1 += coef_h(0, m) * (double)k[m][j];
          h2 += coef_h(1, m) * (double)k[m][j];
          h3 += coef_h(2, m) * (double)k[m][j];
        }
        const double y_new_j = u[j] + (double)k[7][j];
        const double val = theta1 * st.y[j] + theta * (y_new_j + theta1 * (h1 + theta * (h2 + theta * h3)));
#endif
#if MDX_SAVE_HISTORY
        a.hist[hist_index(a, st.traj, st.save_idx, j)] = val;
#endif
#if MDX_HAS_HOOK
        y_save[j] = val;
#endif
      }
#if MDX_HAS_HOOK
      mdx_save_hook(st.save_idx, y_save, a.times[st.save_idx], st.p,
                    a.hook_out + (size_t)st.traj * MDX_HOOK_SIZE);
#endif
      ++st.save_idx;
    }
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) st.y[j] = u[j] + (double)k[7][j];
    st.t += dt_use;
    ++st.accepted;
  } else {
    ++st.rejected;
  }
  ++st.n_steps;
}

__device__ __forceinline__ void finish(State& st, const MdxSolveArgs& a) {
  const bool hit_max = st.save_idx < a.n_save && st.t < st.tf_local;
  // Save times past this trajectory's own end hold its final state
  // (modax/rodas5P.py:991-1002).
  while (st.save_idx < a.n_save) {
#if MDX_SAVE_HISTORY
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) a.hist[hist_index(a, st.traj, st.save_idx, j)] = st.y[j];
#endif
#if MDX_HAS_HOOK
    mdx_save_hook(st.save_idx, st.y, a.times[st.save_idx], st.p,
                  a.hook_out + (size_t)st.traj * MDX_HOOK_SIZE);
#endif
    ++st.save_idx;
  }
#if !MDX_SAVE_HISTORY
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) a.hist[hist_index(a, st.traj, 0, j)] = st.y[j];
#endif
  a.accepted[st.traj] = st.accepted;
  a.rejected[st.traj] = st.rejected;
  a.loop_steps[st.traj] = st.n_steps;
#if MDX_CHECKPOINT
  if (a.ckpt_count) a.ckpt_count[st.traj] = st.n_ckpt;
#endif
  if (a.status) {
    int status = hit_max ? MDX_STATUS_MAX_STEPS : MDX_STATUS_OK;
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j)
      if (!isfinite(st.y[j])) status |= MDX_STATUS_NONFINITE;
#if MDX_CHECKPOINT
    if (st.ckpt_overflow) status |= MDX_STATUS_CKPT_OVERFLOW;
#endif
    a.status[st.traj] = status;
  }
}

}  // namespace rodas5p

struct Rodas5P {
  typedef rodas5p::State State;
  static __device__ __forceinline__ void init(State& s, const MdxSolveArgs& a, int i) { rodas5p::init(s, a, i); }
  static __device__ __forceinline__ bool running(const State& s, const MdxSolveArgs& a) { return rodas5p::running(s, a); }
  static __device__ __forceinline__ void step(State& s, const MdxSolveArgs& a) { rodas5p::step(s, a); }
  static __device__ __forceinline__ void finish(State& s, const MdxSolveArgs& a) { rodas5p::finish(s, a); }
};

}  // namespace mdx
