// Discrete adjoint of a checkpointed ensemble solve, one trajectory per thread.
//
// The forward solve (MDX_CHECKPOINT) records every accepted step's size h_m and,
// every MDX_CKPT_SEG steps, the step's start (t_m, y_m).  This kernel walks the
// steps backwards a segment at a time: it replays the segment forward from its
// recorded start to recover each step's start state, then recomputes step m --
// Jacobian, df/dt, LU and the eight stages (Rodas5P) or the seven stages
// (Tsit5) -- and back-propagates the cotangent of the step's end state and of
// the saves that fell inside the step into the cotangent of y_m and of the
// parameters.  Rejected steps leave no trace in the
// solution and none here; step sizes are constants of the discrete map, so the
// gradient is the exact derivative of the solution the forward pass produced.
//
// Reverse-mode pieces of the traced right-hand side come from the generated
// problem source: mdx_vjp (J^T r, f_p^T r at a stage point), mdx_hvp
// (grad (r . J(y, p) k), the dependence of the iteration matrix on y and p) and
// mdx_ft_vjp (grad (d . df/dt)).  The discrete adjoint has no counterpart in
// the reference, whose gradients come from forward sensitivities
// (modax/_sensitivity.py:331-413); for a fixed step sequence the two are the
// transposes of one linear map, which is what the tests check.
#pragma once

namespace mdx {
namespace adjoint {

__device__ __forceinline__ double ckpt_h(const MdxGradArgs& a, int m, int traj) {
  return a.ckpt[(size_t)m * (size_t)a.n_traj + (size_t)traj];
}

__device__ __forceinline__ const double* ckpt_seg_state(const MdxGradArgs& a, int seg, int traj) {
  return a.ckpt + (size_t)a.ckpt_capacity * (size_t)a.n_traj +
         ((size_t)seg * (size_t)a.n_traj + (size_t)traj) * (size_t)(MDX_NV + 1);
}

// The highest save index whose time a step ending at `t_end` reaches, searching
// down from `hi` (the forward pass's save rule, mdx_common.cuh::save_reached).
__device__ __forceinline__ int last_save_reached(const double* times, int hi, double t_end) {
  int s = hi;
  while (s > 0 && !save_reached(times[s], t_end)) --s;
  return s;
}

__device__ __forceinline__ const double* grad_row(const MdxGradArgs& a, int traj, int s) {
  return a.grad_hist + ((size_t)traj * (size_t)a.n_save + (size_t)s) * MDX_NV;
}

}  // namespace adjoint
}  // namespace mdx

#if defined(MDX_ADJOINT_RODAS5P)
namespace mdx {
namespace adjoint {
using namespace mdx::rodas5p;

// Recompute one accepted Rodas5P step from its start state exactly as the
// forward step did (the same 1/h and 1/(h gamma), step_reciprocals): the
// factorised iteration matrix, the eight stages and the point each stage's f was
// evaluated at.  The end state is us[7] + k[7].
// `lus` receives the matrix the solves use: the factors, or (MDX_WIDE_SOLVE)
// their widened copy, as in the forward step.
template <class SLU, class IP, class K, class US, class DTV>
__device__ __forceinline__ void recompute(double t, double h, const double (&y)[MDX_NV], const double* p,
                                          SLU& lus, IP& ipiv, K& k, US& us, DTV& dT) {
  typedef MDX_LU_T T;
  double inv_dt, dtgamma_inv;
  step_reciprocals(h, inv_dt, dtgamma_inv);
  const double t_end = t + h;
#if MDX_WIDE_SOLVE
  T lu[MDX_LU_SIZE];
#else
  SLU& lu = lus;
#endif
  mdx_neg_jac(y, t, p, lu, dT);
#pragma unroll
  for (int d = 0; d < MDX_NV; ++d) lu[mdx_diag_slot(d)] += (T)dtgamma_inv;
  mdx_factorize(lu, ipiv);
#if MDX_WIDE_SOLVE
  widen_factors(lu, lus);
#endif
  double u[MDX_NV], work[MDX_NV];
  sol_t rhs[MDX_NV];
  const double tstage[8] = {t, t + coef_ct(0) * h, t + coef_ct(1) * h, t + coef_ct(2) * h,
                            t + coef_ct(3) * h, t_end, t_end, t_end};
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    if (s == 0) {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) u[j] = y[j];
    } else if (s <= 5) {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) {
        double acc = coef_a(s - 1, 0) * (double)k[0][j];
#pragma unroll
        for (int m = 1; m < s; ++m) acc += coef_a(s - 1, m) * (double)k[m][j];
        u[j] = y[j] + acc;
      }
    } else {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) u[j] += (double)k[s - 1][j];
    }
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) us[s][j] = u[j];
    mdx_rhs(u, tstage[s], p, work);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      double value;
      if (s == 0) {
        value = MDX_AUTONOMOUS ? work[j] : work[j] + h * coef_d(0) * dT[j];
      } else {
        double acc = coef_c(s, 0) * (double)k[0][j];
#pragma unroll
        for (int m = 1; m < s; ++m) acc += coef_c(s, m) * (double)k[m][j];
        if (coef_d(s) != 0.0 && !MDX_AUTONOMOUS) value = work[j] + h * coef_d(s) * dT[j] + acc * inv_dt;
        else value = work[j] + acc * inv_dt;
      }
      rhs[j] = (sol_t)value;
    }
    mdx_solve(lus, ipiv, rhs);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) k[s][j] = rhs[j];
  }
}

// The end state of one accepted step, for replaying a segment forward.
__device__ __forceinline__ void replay_step(double t, double h, const double (&y)[MDX_NV], const double* p,
                                            double (&y_next)[MDX_NV]) {
  sol_t lu[MDX_LU_SIZE];
  int ipiv[MDX_IPIV];
  sol_t k[8][MDX_NV];
  double us[8][MDX_NV];
  double dT[MDX_NV];
  recompute(t, h, y, p, lu, ipiv, k, us, dT);
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) y_next[j] = us[7][j] + (double)k[7][j];
}

// Reverse of one accepted Rodas5P step.  On entry ybar holds the cotangent of
// the step's end state; on exit the cotangent of its start state; pbar
// accumulates.  Saves s_lo < s <= s_hi fell inside this step.
__device__ __forceinline__ void reverse_step(const MdxGradArgs& a, int traj, double t, double h,
                                             const double (&y)[MDX_NV], const double* p,
                                             int s_lo, int s_hi, double (&ybar)[MDX_NV],
                                             double (&pbar)[MDX_NP > 0 ? MDX_NP : 1]) {
  double inv_dt, dtgamma_inv;
  step_reciprocals(h, inv_dt, dtgamma_inv);
  const double t_end = t + h;
  sol_t lu[MDX_LU_SIZE];
  int ipiv[MDX_IPIV];
  sol_t k[8][MDX_NV];
  double us[8][MDX_NV];
  double dT[MDX_NV];
  recompute(t, h, y, p, lu, ipiv, k, us, dT);
  const double tstage[8] = {t, t + coef_ct(0) * h, t + coef_ct(1) * h, t + coef_ct(2) * h,
                            t + coef_ct(3) * h, t_end, t_end, t_end};

  // Cotangents of the stages, starting from the end state and the saves.
  double kbar[8][MDX_NV];
  double ynew_bar[MDX_NV];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ynew_bar[j] = ybar[j];
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) kbar[s][j] = 0.0;
  double ystart_bar[MDX_NV];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ystart_bar[j] = 0.0;
  for (int sv = s_lo + 1; sv <= s_hi; ++sv) {
    const double theta = (a.times[sv] - t) / h;
    const double theta1 = 1.0 - theta;
    const double* g = grad_row(a, traj, sv);
    const double w1 = theta * theta1, w2 = theta * theta * theta1, w3 = theta * theta * theta * theta1;
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      const double gj = g[j];
      ystart_bar[j] += theta1 * gj;
      ynew_bar[j] += theta * gj;
#pragma unroll
      for (int m = 0; m < 8; ++m)
        kbar[m][j] += (coef_h(0, m) * w1 + coef_h(1, m) * w2 + coef_h(2, m) * w3) * gj;
    }
  }
  // y_new = y + sum_{m<=4} A[4][m] k_m + k5 + k6 + k7
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) {
    ystart_bar[j] += ynew_bar[j];
#pragma unroll
    for (int m = 0; m < 5; ++m) kbar[m][j] += coef_a(4, m) * ynew_bar[j];
    kbar[5][j] += ynew_bar[j];
    kbar[6][j] += ynew_bar[j];
    kbar[7][j] += ynew_bar[j];
  }

  double dTbar[MDX_NV];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) dTbar[j] = 0.0;
  double uchain[MDX_NV];  // cotangent flowing down the u5 -> u6 -> u7 chain
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) uchain[j] = 0.0;

#pragma unroll
  for (int s = 7; s >= 0; --s) {
    sol_t rb_t[MDX_NV];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) rb_t[j] = (sol_t)kbar[s][j];
    mdx_solve_t(lu, ipiv, rb_t);
    double rbar[MDX_NV];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) rbar[j] = (double)rb_t[j];
    // k_s = W^-1 r_s with W = I/(h gamma) - J(y, p): J-bar = rbar k_s^T.
    double kd[MDX_NV];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) kd[j] = (double)k[s][j];
    mdx_hvp(y, t, p, kd, rbar, ystart_bar, pbar);
    // r_s = f(u_s) + h d_s dT + (sum_m C[s][m] k_m) / h
    if (coef_d(s) != 0.0) {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) dTbar[j] += h * coef_d(s) * rbar[j];
    }
#pragma unroll
    for (int m = 0; m < s; ++m)
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) kbar[m][j] += coef_c(s, m) * inv_dt * rbar[j];
    double ubar[MDX_NV];
    mdx_vjp(us[s], tstage[s], p, rbar, ubar, pbar);
    if (s >= 5) {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) ubar[j] += uchain[j];
    }
    if (s == 7 || s == 6) {
      // u_s = u_{s-1} + k_{s-1}
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) {
        uchain[j] = ubar[j];
        kbar[s - 1][j] += ubar[j];
      }
    } else if (s >= 1) {
      // u_s = y + sum_{m<s} A[s-1][m] k_m
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) {
        ystart_bar[j] += ubar[j];
#pragma unroll
        for (int m = 0; m < s; ++m) kbar[m][j] += coef_a(s - 1, m) * ubar[j];
      }
    } else {
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) ystart_bar[j] += ubar[j];
    }
  }
  mdx_ft_vjp(y, t, p, dTbar, ystart_bar, pbar);
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ybar[j] = ystart_bar[j];
}

}  // namespace adjoint
}  // namespace mdx
#endif

#if defined(MDX_ADJOINT_TSIT5)
namespace mdx {
namespace adjoint {
using namespace mdx::tsit5;

// Tsit5 rows: u_s = y + h * sum_{m<s} a[s][m] k_m, k_s = f(u_s, t + c_s h);
// y_new = u_7 (the B row), k_7 = f(y_new, t + h).
__device__ __forceinline__ double arow(int s, int m) {
  const double r[7][6] = {
      {0, 0, 0, 0, 0, 0},
      {A21, 0, 0, 0, 0, 0},
      {A31, A32, 0, 0, 0, 0},
      {A41, A42, A43, 0, 0, 0},
      {A51, A52, A53, A54, 0, 0},
      {A61, A62, A63, A64, A65, 0},
      {B1, B2, B3, B4, B5, B6},
  };
  return r[s][m];
}

__device__ __forceinline__ double cstage(int s) {
  const double c[7] = {0.0, C2, C3, C4, C5, 1.0, 1.0};
  return c[s];
}

template <class K, class US>
__device__ __forceinline__ void recompute(double t, double h, const double (&y)[MDX_NV], const double* p,
                                          K& k, US& us) {
#pragma unroll
  for (int s = 0; s < 7; ++s) {
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      if (s == 0) {
        us[s][j] = y[j];
      } else {
        double acc = arow(s, 0) * k[0][j];
#pragma unroll
        for (int m = 1; m < s; ++m) acc += arow(s, m) * k[m][j];
        us[s][j] = y[j] + h * acc;
      }
    }
    mdx_rhs(us[s], t + cstage(s) * h, p, k[s]);
  }
}

__device__ __forceinline__ void replay_step(double t, double h, const double (&y)[MDX_NV], const double* p,
                                            double (&y_next)[MDX_NV]) {
  double k[7][MDX_NV], us[7][MDX_NV];
  recompute(t, h, y, p, k, us);
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) y_next[j] = us[6][j];
}

__device__ __forceinline__ void reverse_step(const MdxGradArgs& a, int traj, double t, double h,
                                             const double (&y)[MDX_NV], const double* p,
                                             int s_lo, int s_hi, double (&ybar)[MDX_NV],
                                             double (&pbar)[MDX_NP > 0 ? MDX_NP : 1]) {
  double k[7][MDX_NV], us[7][MDX_NV];
  recompute(t, h, y, p, k, us);
  // k[6] is f(y_new, t + h); the end state is us[6].
  double kbar[7][MDX_NV], ystart_bar[MDX_NV], ynew_bar[MDX_NV];
#pragma unroll
  for (int s = 0; s < 7; ++s)
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) kbar[s][j] = 0.0;
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) {
    ystart_bar[j] = 0.0;
    ynew_bar[j] = ybar[j];
  }
  for (int sv = s_lo + 1; sv <= s_hi; ++sv) {
    const double theta = (a.times[sv] - t) / h;
    double b[7];
    dense_weights(theta, b);
    const double* g = grad_row(a, traj, sv);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      ystart_bar[j] += g[j];
#pragma unroll
      for (int m = 0; m < 7; ++m) kbar[m][j] += h * b[m] * g[j];
    }
  }
  // k7 = f(y_new): its cotangent flows into y_new first.
  double ub[MDX_NV];
  mdx_vjp(us[6], t + h, p, kbar[6], ub, pbar);
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ynew_bar[j] += ub[j];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) {
    ystart_bar[j] += ynew_bar[j];
#pragma unroll
    for (int m = 0; m < 6; ++m) kbar[m][j] += h * arow(6, m) * ynew_bar[j];
  }
#pragma unroll
  for (int s = 5; s >= 0; --s) {
    mdx_vjp(us[s], t + cstage(s) * h, p, kbar[s], ub, pbar);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      ystart_bar[j] += ub[j];
#pragma unroll
      for (int m = 0; m < s; ++m) kbar[m][j] += h * arow(s, m) * ub[j];
    }
  }
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ybar[j] = ystart_bar[j];
}

}  // namespace adjoint
}  // namespace mdx
#endif

// The reverse pass.  Segments of MDX_CKPT_SEG accepted steps are visited last
// to first: each is replayed forward from its recorded start state (with the
// recorded step sizes) to recover every step's start state, then reversed step
// by step.  Saves after the last accepted step hold the final state (Rodas5P's
// frozen saves); save 0 is y0 itself.
//
// reverse_segments reverses segments [seg_lo, seg_hi) of one trajectory with
// `steps` recorded steps, ybar holding the cotangent at the end of segment
// seg_hi - 1 on entry and at the start of segment seg_lo on exit; pbar
// accumulates.  With `inject` the saves' cotangents (grad_hist) inside the range
// are added as their steps are reversed, and, when the range ends with the last
// step, those of the frozen saves first; without it the pass is the homogeneous
// linear map, which a split trajectory's chunks are composed from.
namespace mdx {
namespace adjoint {

// Small systems load the segment below's start record and step sizes while the
// current segment is being reversed: a sweep that has the SM to itself (the
// longest trajectories, last) would otherwise wait on each segment's loads.
#define MDX_SEG_PREFETCH (MDX_NV <= 8 && MDX_CKPT_SEG <= 8)

struct SegmentData {
  double rec[MDX_NV + 1];  // t, y at the segment's first step
  double h[MDX_SEG_PREFETCH ? MDX_CKPT_SEG : 1];
};

__device__ __forceinline__ void load_segment(const MdxGradArgs& a, int seg, int traj, int steps, SegmentData& d) {
  const double* rec = ckpt_seg_state(a, seg, traj);
#pragma unroll
  for (int j = 0; j <= MDX_NV; ++j) d.rec[j] = __ldg(rec + j);
#if MDX_SEG_PREFETCH
  const int m0 = seg * MDX_CKPT_SEG;
#pragma unroll
  for (int k = 0; k < MDX_CKPT_SEG; ++k)
    if (m0 + k < steps) d.h[k] = __ldg(a.ckpt + (size_t)(m0 + k) * (size_t)a.n_traj + (size_t)traj);
#endif
}

__device__ __forceinline__ double segment_h(const MdxGradArgs& a, const SegmentData& d, int m, int m0, int traj) {
#if MDX_SEG_PREFETCH
  (void)a;
  (void)traj;
  double h = d.h[0];
#pragma unroll
  for (int k = 1; k < MDX_CKPT_SEG; ++k)
    if (m - m0 == k) h = d.h[k];
  return h;
#else
  (void)d;
  (void)m0;
  return ckpt_h(a, m, traj);
#endif
}

__device__ __forceinline__ void reverse_segments(const MdxGradArgs& a, int traj, const double* p, int steps,
                                                 int seg_lo, int seg_hi, bool inject,
                                                 double (&ybar)[MDX_NV],
                                                 double (&pbar)[MDX_NP > 0 ? MDX_NP : 1]) {
  double yseg[MDX_CKPT_SEG][MDX_NV];
  double tseg[MDX_CKPT_SEG];
  int s_hi = 0;
  SegmentData cur;
  if (seg_hi > seg_lo) load_segment(a, seg_hi - 1, traj, steps, cur);
  for (int seg = seg_hi - 1; seg >= seg_lo; --seg) {
    const int m0 = seg * MDX_CKPT_SEG;
    const int m1 = (m0 + MDX_CKPT_SEG < steps) ? m0 + MDX_CKPT_SEG : steps;
    SegmentData next;
#if MDX_SEG_PREFETCH
    if (seg > seg_lo) load_segment(a, seg - 1, traj, steps, next);
#endif
    double y[MDX_NV];
    double t = cur.rec[0];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) y[j] = cur.rec[1 + j];
    for (int m = m0; m < m1; ++m) {
      tseg[m - m0] = t;
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) yseg[m - m0][j] = y[j];
      const double h = segment_h(a, cur, m, m0, traj);
      if (m + 1 < m1) {
        double y_next[MDX_NV];
        replay_step(t, h, y, p, y_next);
#pragma unroll
        for (int j = 0; j < MDX_NV; ++j) y[j] = y_next[j];
      }
      t += h;
    }
    if (seg == seg_hi - 1) {
      // t is now the end time of the range's last step: the saves it reached
      // are the ones its steps own.
      s_hi = last_save_reached(a.times, a.n_save - 1, t);
      if (inject && m1 == steps) {
        // Later saves are frozen at the final state.
        for (int sv = s_hi + 1; sv < a.n_save; ++sv) {
          const double* g = grad_row(a, traj, sv);
#pragma unroll
          for (int j = 0; j < MDX_NV; ++j) ybar[j] += g[j];
        }
      }
    }
    for (int m = m1 - 1; m >= m0; --m) {
      const double tm = tseg[m - m0];
      const double h = segment_h(a, cur, m, m0, traj);
      double ym[MDX_NV];
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) ym[j] = yseg[m - m0][j];
      const int s_lo = m == 0 ? 0 : last_save_reached(a.times, s_hi, tm);
      reverse_step(a, traj, tm, h, ym, p, inject ? s_lo : s_hi, s_hi, ybar, pbar);
      s_hi = s_lo;
    }
    if (seg > seg_lo) {
#if MDX_SEG_PREFETCH
      cur = next;
#else
      load_segment(a, seg - 1, traj, steps, cur);
#endif
    }
  }
}

}  // namespace adjoint
}  // namespace mdx

extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_grad_reverse(const MdxGradArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_run) return;
  int traj, seg_lo = 0, seg_hi = 0, kind = -2, slot = -1;
  if (a.tasks) {
    const int* task = a.tasks + (size_t)i * 5;
    traj = task[0];
    seg_lo = task[1];
    seg_hi = task[2];
    kind = task[3];
    slot = task[4];
  } else {
    traj = a.order ? a.order[i] : i;
  }
  if (traj < 0 || traj >= a.n_traj || kind < -2 || kind >= MDX_NV) return;
  double p[MDX_NP > 0 ? MDX_NP : 1];
#pragma unroll
  for (int k = 0; k < MDX_NP; ++k) p[k] = a.params[(size_t)traj * MDX_NP + k];
  double pbar[MDX_NP > 0 ? MDX_NP : 1];
#pragma unroll
  for (int k = 0; k < MDX_NP; ++k) pbar[k] = 0.0;
  double ybar[MDX_NV];
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) ybar[j] = kind == j ? 1.0 : 0.0;
  const int n_steps = a.ckpt_count[traj];
  const int steps = n_steps < a.ckpt_capacity ? n_steps : (int)a.ckpt_capacity;
  const int n_seg = (steps + MDX_CKPT_SEG - 1) / MDX_CKPT_SEG;
  if (kind == -2) {
    seg_lo = 0;
    seg_hi = n_seg;
  } else if (seg_lo < 0 || seg_hi > n_seg || seg_lo >= seg_hi || slot < 0 || slot >= a.n_slots) {
    return;
  }
  const bool inject = kind < 0;
  if (steps == 0 && inject) {
    for (int sv = 1; sv < a.n_save; ++sv) {
      const double* g = mdx::adjoint::grad_row(a, traj, sv);
#pragma unroll
      for (int j = 0; j < MDX_NV; ++j) ybar[j] += g[j];
    }
  }
  mdx::adjoint::reverse_segments(a, traj, p, steps, seg_lo, seg_hi, inject, ybar, pbar);
  if (inject && seg_lo == 0) {
    const double* g0 = mdx::adjoint::grad_row(a, traj, 0);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) ybar[j] += g0[j];
  }
  if (kind == -2) {
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) a.grad_y0[(size_t)traj * MDX_NV + j] = ybar[j];
#pragma unroll
    for (int k = 0; k < MDX_NP; ++k) a.grad_params[(size_t)traj * MDX_NP + k] = pbar[k];
    if (a.status) a.status[traj] = n_steps > a.ckpt_capacity ? MDX_STATUS_CKPT_OVERFLOW : 0;
  } else {
    double* out = a.task_out + (size_t)slot * (MDX_NV + MDX_NP);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) out[j] = ybar[j];
#pragma unroll
    for (int k = 0; k < MDX_NP; ++k) out[MDX_NV + k] = pbar[k];
  }
}

// Composes each split trajectory's chunks, last to first: with the cotangent
// lambda at a chunk's end, its start gets A lambda + b and the parameters
// P lambda + q, where column j of [A; P] is the chunk's unit task j and [b; q]
// its injecting task.
extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_grad_combine(const MdxGradArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n_combine) return;
  const int traj = a.combine[(size_t)k * 3];
  const int first = a.combine[(size_t)k * 3 + 1];
  const int chunks = a.combine[(size_t)k * 3 + 2];
  constexpr int W = MDX_NV + MDX_NP;
  constexpr int PER_CHUNK = MDX_NV + 1;
  if (traj < 0 || traj >= a.n_traj || chunks < 1 || first < 0 || first + chunks * PER_CHUNK > a.n_slots) return;
  double lam[MDX_NV];
  double pb[MDX_NP > 0 ? MDX_NP : 1];
  const double* last = a.task_out + (size_t)(first + (chunks - 1) * PER_CHUNK) * W;
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) lam[j] = last[j];
#pragma unroll
  for (int q = 0; q < MDX_NP; ++q) pb[q] = last[MDX_NV + q];
  for (int c = chunks - 2; c >= 0; --c) {
    const double* base = a.task_out + (size_t)(first + c * PER_CHUNK) * W;
    double next[MDX_NV];
#pragma unroll
    for (int i = 0; i < MDX_NV; ++i) next[i] = base[i];
#pragma unroll
    for (int q = 0; q < MDX_NP; ++q) pb[q] += base[MDX_NV + q];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) {
      const double* col = base + (size_t)(j + 1) * W;
#pragma unroll
      for (int i = 0; i < MDX_NV; ++i) next[i] += col[i] * lam[j];
#pragma unroll
      for (int q = 0; q < MDX_NP; ++q) pb[q] += col[MDX_NV + q] * lam[j];
    }
#pragma unroll
    for (int i = 0; i < MDX_NV; ++i) lam[i] = next[i];
  }
#pragma unroll
  for (int j = 0; j < MDX_NV; ++j) a.grad_y0[(size_t)traj * MDX_NV + j] = lam[j];
#pragma unroll
  for (int q = 0; q < MDX_NP; ++q) a.grad_params[(size_t)traj * MDX_NP + q] = pb[q];
  if (a.status) a.status[traj] = a.ckpt_count[traj] > a.ckpt_capacity ? MDX_STATUS_CKPT_OVERFLOW : 0;
}
