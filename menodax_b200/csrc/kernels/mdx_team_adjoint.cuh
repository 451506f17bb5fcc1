// Discrete adjoint of a checkpointed Rodas5P solve with a team of MDX_TEAM lanes
// per trajectory: the thread kernel's reverse sweep (mdx_adjoint.cuh) with the
// per-trajectory vectors in a shared-memory slice and the work of each phase
// split across the team, the way mdx_team.cuh splits the forward step.
//
// A thread reverse sweep keeps the eight stages, their cotangents and the
// segment's start states of one trajectory -- several KB for a 16-state system --
// in local memory, and each step is a long serial chain through it.  Here those
// arrays live in the team's slice; component j of every vector operation runs
// on lane j % MDX_TEAM; the right-hand side, -J and the reverse-mode pieces
// (J^T r, f_p^T r, grad (r . J k), grad (d . df/dt)) are the generated class
// loops; the sparse factorisation and the forward and transposed solves are the
// thread kernel's generated code on the first lane, as in the forward team step.
//
// Recomputed steps use the forward team step's own arithmetic (mdx_team.cuh's
// stage / advance / rhs / factorize), with the recorded step sizes, so the
// gradient is the derivative of the solution the team forward pass produced.
#pragma once

// The block's reverse-sweep slices; a host build of this kernel (lanes as
// contexts on one thread) defines it to a static so all lanes see one copy.
#ifndef MDX_BLOCK_SHARED
#define MDX_BLOCK_SHARED __shared__
#endif

namespace mdx {
namespace team_adjoint {

using namespace mdx::team;

struct GradSlice {
  Slice s;                      // the recomputed step: y, u, f, (dT), p, k, lu
  double kbar[8][MDX_NV];       // stage cotangents
  double ystart[MDX_NV];        // cotangent of the step's start state
  double ynew[MDX_NV];          // cotangent of the step's end state
  double uchain[MDX_NV];        // cotangent flowing down u5 -> u6 -> u7
  double rbar[MDX_NV];          // M^-T kbar[s]
  double ubar[MDX_NV];          // J(u_s)^T rbar
  double kd[MDX_NV];            // k_s in double, the direction of the hvp
#if !MDX_TEAM_AUTONOMOUS
  double dTbar[MDX_NV];
#endif
  double pbar[MDX_NP > 0 ? MDX_NP : 1];
  double yseg[MDX_CKPT_SEG][MDX_NV];
  double tseg[MDX_CKPT_SEG];
};

constexpr int GRAD_TEAMS_PER_BLOCK = MDX_TPB / MDX_TEAM;

__device__ __forceinline__ double ckpt_h(const MdxGradArgs& a, int m, int traj) {
  return a.ckpt[(size_t)m * (size_t)a.n_traj + (size_t)traj];
}

__device__ __forceinline__ const double* ckpt_seg_state(const MdxGradArgs& a, int seg, int traj) {
  return a.ckpt + (size_t)a.ckpt_capacity * (size_t)a.n_traj +
         ((size_t)seg * (size_t)a.n_traj + (size_t)traj) * (size_t)(MDX_NV + 1);
}

__device__ __forceinline__ int last_save_reached(const double* times, int hi, double t_end) {
  int sv = hi;
  while (sv > 0 && !save_reached(times[sv], t_end)) --sv;
  return sv;
}

__device__ __forceinline__ const double* grad_row(const MdxGradArgs& a, int traj, int sv) {
  return a.grad_hist + ((size_t)traj * (size_t)a.n_save + (size_t)sv) * MDX_NV;
}

// Recompute the accepted step (t, h) from s.y: the factorised matrix and the
// eight stages, exactly as the forward team step computed them.
__device__ __forceinline__ void recompute(Slice& s, const Lanes& L, double t, double h, double& inv_dt) {
#if MDX_FAST
  inv_dt = recip_newton(h);
  const double dtgamma_inv = inv_dt * (1.0 / GAMMA);
#else
  inv_dt = 1.0 / h;
  const double dtgamma_inv = 1.0 / (h * GAMMA);
#endif
  const double t_end = t + h;
  for (int q = L.lane; q < MDX_TEAM_LU_SIZE; q += MDX_TEAM) s.lu[q] = (lu_t)(MDX_TEAM_LU_CLEAR);
  __syncwarp(L.mask);
  mdx_team_neg_jac(s.y, t, s.p, s.lu, L.lane);
#if !MDX_TEAM_AUTONOMOUS
  mdx_team_dT(s.y, t, s.p, s.dT, L.lane);
#endif
  __syncwarp(L.mask);
  for (int d = L.lane; d < MDX_NV; d += MDX_TEAM) s.lu[mdx_team_diag_slot(d)] += (lu_t)dtgamma_inv;
  __syncwarp(L.mask);
  factorize(s, L);
  rhs(s, L, s.y, t);
  stage<0>(s, L, h, inv_dt);
  advance<0>(s, L);
  rhs(s, L, s.u, t + coef_ct(0) * h);
  stage<1>(s, L, h, inv_dt);
  advance<1>(s, L);
  rhs(s, L, s.u, t + coef_ct(1) * h);
  stage<2>(s, L, h, inv_dt);
  advance<2>(s, L);
  rhs(s, L, s.u, t + coef_ct(2) * h);
  stage<3>(s, L, h, inv_dt);
  advance<3>(s, L);
  rhs(s, L, s.u, t + coef_ct(3) * h);
  stage<4>(s, L, h, inv_dt);
  advance<4>(s, L);
  rhs(s, L, s.u, t_end);
  stage<5>(s, L, h, inv_dt);
  accumulate(s, L, 5);
  rhs(s, L, s.u, t_end);
  stage<6>(s, L, h, inv_dt);
  accumulate(s, L, 6);
  rhs(s, L, s.u, t_end);
  stage<7>(s, L, h, inv_dt);
}

// The point stage S's right-hand side was evaluated at, into s.u (the forward
// step's own sums: u0 = y, u_S = y + sum_{m<S} A[S-1][m] k_m up to S = 5, then
// u6 = u5 + k5 and u7 = u6 + k6).
__device__ __forceinline__ void stage_point(Slice& s, const Lanes& L, int S) {
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    double u = s.y[j];
    if (S >= 1) {
      const int row = S <= 5 ? S - 1 : 4;
      double acc = coef_a(row, 0) * (double)s.k[0][j];
#pragma unroll
      for (int m = 1; m <= row; ++m) acc += coef_a(row, m) * (double)s.k[m][j];
      u = s.y[j] + acc;
      if (S >= 6) u += (double)s.k[5][j];
      if (S >= 7) u += (double)s.k[6][j];
    }
    s.u[j] = u;
  }
  __syncwarp(L.mask);
}

// rbar = M^-T kbar[S] on the team's first lane (the generated transposed solve).
__device__ __noinline__ void solve_t(GradSlice& g, int S, const Lanes L) {
  if (L.lane == 0) {
    lu_t r[MDX_NV];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) r[j] = (lu_t)g.kbar[S][j];
    mdx_sparse_solve_t<lu_t>(g.s.lu, r);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) g.rbar[j] = (double)r[j];
  }
  __syncwarp(L.mask);
}

// Reverse one accepted step: on entry ynew holds the cotangent of the step's end
// state, on exit ystart holds that of its start; pbar accumulates.  Saves
// s_lo < sv <= s_hi fell inside the step (the thread kernel's reverse_step).
__device__ __forceinline__ void reverse_step(GradSlice& g, const Lanes& L, const MdxGradArgs& a, int traj,
                                             double t, double h, int s_lo, int s_hi) {
  Slice& s = g.s;
  double inv_dt;
  recompute(s, L, t, h, inv_dt);
  const double t_end = t + h;
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    g.ystart[j] = 0.0;
    g.uchain[j] = 0.0;
#if !MDX_TEAM_AUTONOMOUS
    g.dTbar[j] = 0.0;
#endif
#pragma unroll
    for (int m = 0; m < 8; ++m) g.kbar[m][j] = 0.0;
  }
  for (int sv = s_lo + 1; sv <= s_hi; ++sv) {
    const double theta = (a.times[sv] - t) / h;
    const double theta1 = 1.0 - theta;
    const double* gr = grad_row(a, traj, sv);
    const double w1 = theta * theta1, w2 = theta * theta * theta1, w3 = theta * theta * theta * theta1;
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
      const double gj = gr[j];
      g.ystart[j] += theta1 * gj;
      g.ynew[j] += theta * gj;
#pragma unroll
      for (int m = 0; m < 8; ++m) g.kbar[m][j] += (coef_h(0, m) * w1 + coef_h(1, m) * w2 + coef_h(2, m) * w3) * gj;
    }
  }
  // y_new = y + sum_{m<=4} A[4][m] k_m + k5 + k6 + k7
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    const double yn = g.ynew[j];
    g.ystart[j] += yn;
#pragma unroll
    for (int m = 0; m < 5; ++m) g.kbar[m][j] += coef_a(4, m) * yn;
    g.kbar[5][j] += yn;
    g.kbar[6][j] += yn;
    g.kbar[7][j] += yn;
  }
  __syncwarp(L.mask);
  const double tstage[8] = {t, t + coef_ct(0) * h, t + coef_ct(1) * h, t + coef_ct(2) * h,
                            t + coef_ct(3) * h, t_end, t_end, t_end};
#pragma unroll 1
  for (int S = 7; S >= 0; --S) {
    solve_t(g, S, L);
    // k_S = M^-1 r_S with M = I/(h gamma) - J(y, p): the matrix's dependence on y, p.
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.kd[j] = (double)s.k[S][j];
    __syncwarp(L.mask);
    mdx_team_hvp(s.y, t, s.p, g.kd, g.rbar, g.ystart, g.pbar, L.lane);
    // r_S = f(u_S) + h d_S dT + (sum_{m<S} C[S][m] k_m) / h
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
#if !MDX_TEAM_AUTONOMOUS
      g.dTbar[j] += h * coef_d(S) * g.rbar[j];
#endif
      for (int m = 0; m < S; ++m) g.kbar[m][j] += coef_c(S, m) * inv_dt * g.rbar[j];
    }
    stage_point(s, L, S);
    mdx_team_vjp(s.u, tstage[S], s.p, g.rbar, g.ubar, g.pbar, L.lane);
    __syncwarp(L.mask);
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
      double ub = g.ubar[j];
      if (S >= 5) ub += g.uchain[j];
      if (S == 7 || S == 6) {
        // u_S = u_{S-1} + k_{S-1}
        g.uchain[j] = ub;
        g.kbar[S - 1][j] += ub;
      } else if (S >= 1) {
        // u_S = y + sum_{m<S} A[S-1][m] k_m
        g.ystart[j] += ub;
        for (int m = 0; m < S; ++m) g.kbar[m][j] += coef_a(S - 1, m) * ub;
      } else {
        g.ystart[j] += ub;
      }
    }
    __syncwarp(L.mask);
  }
#if !MDX_TEAM_AUTONOMOUS
  mdx_team_ft_vjp(s.y, t, s.p, g.dTbar, g.ystart, g.pbar, L.lane);
  __syncwarp(L.mask);
#endif
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.ynew[j] = g.ystart[j];
  __syncwarp(L.mask);
}

}  // namespace team_adjoint
}  // namespace mdx

// The reverse pass, one team per trajectory, segments last to first (the thread
// kernel's mdx_grad_reverse).  The launch takes order[0..n_run) in blocks of
// MDX_TPB / MDX_TEAM trajectories.
extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_grad_reverse(const MdxGradArgs a) {
  using namespace mdx::team_adjoint;
  MDX_BLOCK_SHARED GradSlice slices[GRAD_TEAMS_PER_BLOCK];
  const Lanes L = lanes();
  GradSlice& g = slices[threadIdx.x / MDX_TEAM];
  Slice& s = g.s;
  const int i = blockIdx.x * GRAD_TEAMS_PER_BLOCK + (int)(threadIdx.x / MDX_TEAM);
  if (i >= a.n_run) return;  // whole teams leave together
  const int traj = a.order ? a.order[i] : i;
  for (int k = L.lane; k < MDX_NP; k += MDX_TEAM) {
    s.p[k] = a.params[(size_t)traj * MDX_NP + k];
    g.pbar[k] = 0.0;
  }
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.ynew[j] = 0.0;
  const int n_steps = a.ckpt_count[traj];
  int status = 0;
  if (n_steps > a.ckpt_capacity) status |= MDX_STATUS_CKPT_OVERFLOW;
  const int steps = n_steps < a.ckpt_capacity ? n_steps : (int)a.ckpt_capacity;
  __syncwarp(L.mask);
  int s_hi = 0;
  if (steps == 0) {
    for (int sv = 1; sv < a.n_save; ++sv) {
      const double* gr = grad_row(a, traj, sv);
      for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.ynew[j] += gr[j];
    }
    __syncwarp(L.mask);
  }
  for (int seg = (steps - 1) / MDX_CKPT_SEG; steps > 0 && seg >= 0; --seg) {
    const int m0 = seg * MDX_CKPT_SEG;
    const int m1 = (m0 + MDX_CKPT_SEG < steps) ? m0 + MDX_CKPT_SEG : steps;
    const double* rec = ckpt_seg_state(a, seg, traj);
    double t = rec[0];
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) s.y[j] = rec[1 + j];
    __syncwarp(L.mask);
    for (int m = m0; m < m1; ++m) {
      if (L.lane == 0) g.tseg[m - m0] = t;
      for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.yseg[m - m0][j] = s.y[j];
      const double h = ckpt_h(a, m, traj);
      if (m + 1 < m1) {
        double inv_dt;
        recompute(s, L, t, h, inv_dt);
        for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) s.y[j] = s.u[j] + (double)s.k[7][j];
        __syncwarp(L.mask);
      }
      t += h;
    }
    __syncwarp(L.mask);
    if (m1 == steps) {
      // t is the end time of the last accepted step: later saves are frozen.
      s_hi = last_save_reached(a.times, a.n_save - 1, t);
      for (int sv = s_hi + 1; sv < a.n_save; ++sv) {
        const double* gr = grad_row(a, traj, sv);
        for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) g.ynew[j] += gr[j];
      }
      __syncwarp(L.mask);
    }
    for (int m = m1 - 1; m >= m0; --m) {
      const double tm = g.tseg[m - m0];
      const double h = ckpt_h(a, m, traj);
      for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) s.y[j] = g.yseg[m - m0][j];
      __syncwarp(L.mask);
      const int s_lo = m == 0 ? 0 : last_save_reached(a.times, s_hi, tm);
      reverse_step(g, L, a, traj, tm, h, s_lo, s_hi);
      s_hi = s_lo;
    }
  }
  const double* g0 = grad_row(a, traj, 0);
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) a.grad_y0[(size_t)traj * MDX_NV + j] = g.ynew[j] + g0[j];
  for (int k = L.lane; k < MDX_NP; k += MDX_TEAM) a.grad_params[(size_t)traj * MDX_NP + k] = g.pbar[k];
  if (a.status && L.lane == 0) a.status[traj] = status;
}
