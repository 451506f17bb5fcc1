// Rodas5P with a team of MDX_TEAM lanes per trajectory (4 to 32 lanes, a power
// of two, so a team never straddles a warp).
//
// The step is the thread kernel's (mdx_rodas5p.cuh, the reference's
// modax/rodas5P.py:761-1005) with the per-trajectory vectors moved from
// registers to a shared-memory slice and the work of each phase split across
// the team:
//
//   * right-hand side, -J and df/dt: the generated class loops (member m of a
//     class of structurally identical components on lane m % MDX_TEAM);
//   * vector algebra (stage right-hand sides, stage combinations, the error
//     terms, dense output, the history rows): component j on lane j % MDX_TEAM,
//     so history stores are contiguous across the team;
//   * dense LU and solves: mdx_team_lu.cuh;
//   * sparse LU and solves: the generated straight-line (or table) routines of
//     the thread kernel, run by the team's first lane on the shared matrix with
//     the right-hand side in its registers -- the other lanes of a warp serve
//     the other teams' trajectories, so a warp of 4-lane teams runs 8
//     factorisations side by side;
//   * scalars (t, h, the controller, the accept decision) on every lane, from
//     identical inputs, so every lane of a team takes the same branches.
//
// The error norm sums its squared terms in component order on every lane, the
// thread kernel's order.  A __syncwarp over the team's lanes separates every
// write of the slice from the reads of other lanes that follow it.
#pragma once
#include "mdx_common.cuh"
#include "mdx_rodas5p_coef.cuh"
#if MDX_TEAM_DENSE
#include "mdx_team_lu.cuh"
#endif

namespace mdx {
namespace team {

using rodas5p::coef_a;
using rodas5p::coef_c;
using rodas5p::coef_ct;
using rodas5p::coef_d;
using rodas5p::coef_h;
using rodas5p::FACTOR_MAX;
using rodas5p::FACTOR_MIN;
using rodas5p::GAMMA;

typedef MDX_LU_T lu_t;
constexpr int TEAMS_PER_BLOCK = MDX_TPB / MDX_TEAM;
static_assert(MDX_TEAM == 4 || MDX_TEAM == 8 || MDX_TEAM == 16 || MDX_TEAM == 32,
              "a team is 4, 8, 16 or 32 lanes");
static_assert(MDX_TPB % 32 == 0, "blocks are whole warps");
static_assert(MDX_NS == MDX_NV, "the team kernel integrates the plain system");

// One trajectory's shared-memory slice.  Doubles first, then the LU-typed
// arrays, then the permutation; the host sizes the launch with the same layout.
struct Slice {
  double y[MDX_NV];
  double u[MDX_NV];
  double f[MDX_NV];  // f(u) of the current stage; the scaled error terms at the end
#if !MDX_TEAM_AUTONOMOUS
  double dT[MDX_NV];
#endif
  double p[MDX_NP > 0 ? MDX_NP : 1];
#if MDX_TEAM_DENSE && !MDX_FAST
  double fac[2 * MDX_NV];
#endif
  lu_t k[8][MDX_NV];
  lu_t lu[MDX_TEAM_LU_SIZE];
#if MDX_TEAM_DENSE
  int perm[MDX_NV];
#endif
};
static_assert(sizeof(Slice) == MDX_TEAM_SLICE_BYTES, "host and device disagree on the slice layout");

struct Lanes {
  int lane;       // lane within the team
  unsigned mask;  // the team's lanes within the warp
};

__device__ __forceinline__ Lanes lanes() {
  Lanes l;
  l.lane = (int)(threadIdx.x % MDX_TEAM);
  if constexpr (MDX_TEAM == 32) {
    l.mask = MDX_FULL_MASK;
  } else {
    const unsigned first = (threadIdx.x & 31u) / MDX_TEAM * MDX_TEAM;
    l.mask = ((1u << MDX_TEAM) - 1u) << first;
  }
  return l;
}

__device__ __forceinline__ Slice* slice_of_team() {
  extern __shared__ __align__(16) unsigned char mdx_team_smem[];
  return reinterpret_cast<Slice*>(mdx_team_smem + (size_t)(threadIdx.x / MDX_TEAM) * MDX_TEAM_SLICE_BYTES);
}

// Scalars every lane of a team holds identically.
struct State {
  double t, dt, err_prev, err_prev2, tf_local;
  int save_idx, n_steps, accepted, rejected, traj;
#if MDX_CHECKPOINT
  int n_ckpt;
  bool ckpt_overflow;
#endif
};

__device__ __forceinline__ size_t hist_index(const MdxSolveArgs& a, int traj, int s, int j) {
  return ((size_t)traj * (size_t)a.n_save_hist + (size_t)s) * (size_t)MDX_NV + (size_t)j;
}

__device__ __forceinline__ double weight(const MdxSolveArgs& a, int traj, int j) {
#if MDX_WEIGHTS_RUNTIME
  return a.weights[(size_t)traj * MDX_NV + j];
#else
  (void)a; (void)traj;
  return mdx_const_weight(j);
#endif
}

__device__ __forceinline__ void factorize(Slice& s, const Lanes& L) {
#if MDX_TEAM_DENSE
#if MDX_FAST
  dense_factorize<MDX_NV, MDX_TEAM_LDA, lu_t, true>(s.lu, s.perm, nullptr, L.lane, L.mask);
#else
  dense_factorize<MDX_NV, MDX_TEAM_LDA, lu_t, false>(s.lu, s.perm, s.fac, L.lane, L.mask);
#endif
#else
  if (L.lane == 0) mdx_sparse_factorize<lu_t>(s.lu);
  __syncwarp(L.mask);
#endif
}

// Solve M x = x in place on stage row x.  One copy serves the eight stages: the
// substitutions are the largest straight-line code of a step, and eight inlined
// copies overflow the instruction cache (ncu: "no instruction" stalls).
__device__ __noinline__ void solve(Slice& s, lu_t* x, const Lanes L) {
#if MDX_TEAM_DENSE
  dense_solve<MDX_NV, MDX_TEAM_LDA, lu_t, MDX_FAST != 0>(s.lu, s.perm, x, L.lane, L.mask);
#else
  if (L.lane == 0) {
#if MDX_TEAM_SPARSE_REGISTERS
    lu_t r[MDX_NV];
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) r[j] = x[j];
    mdx_sparse_solve<lu_t>(s.lu, r);
#pragma unroll
    for (int j = 0; j < MDX_NV; ++j) x[j] = r[j];
#else
    mdx_sparse_solve<lu_t>(s.lu, x);
#endif
  }
  __syncwarp(L.mask);
#endif
}

__device__ __forceinline__ void init(State& st, Slice& s, const Lanes& L, const MdxSolveArgs& a, int traj) {
  st.traj = traj;
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    const double v = a.y0[(size_t)traj * MDX_NV + j];
    s.y[j] = v;
#if MDX_SAVE_HISTORY
    a.hist[hist_index(a, traj, 0, j)] = v;
#endif
  }
  for (int k = L.lane; k < MDX_NP; k += MDX_TEAM) s.p[k] = a.params[(size_t)traj * MDX_NP + k];
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
  st.tf_local = a.params[(size_t)traj * MDX_NP + MDX_TF_INDEX];
#else
  st.tf_local = tf;
#endif
#if MDX_CHECKPOINT
  st.n_ckpt = 0;
  st.ckpt_overflow = false;
#endif
  __syncwarp(L.mask);
#if MDX_HAS_HOOK
  // The hook (the thread kernel's generated code) runs on the team's first lane
  // on the slice's state; its row starts at zero (modax/rodas5P.py:753-756).
  if (L.lane == 0) {
    double* acc = a.hook_out + (size_t)traj * MDX_HOOK_SIZE;
    for (int j = 0; j < MDX_HOOK_SIZE; ++j) acc[j] = 0.0;
    mdx_save_hook(0, s.y, t0, s.p, acc);
  }
  __syncwarp(L.mask);
#endif
}

__device__ __forceinline__ bool running(const State& st, const MdxSolveArgs& a) {
  return st.save_idx < a.n_save && st.t < st.tf_local && st.n_steps < a.max_steps;
}

// Stage S's right-hand side into k[S] (rounded to the LU type), then the solve.
template <int S>
__device__ __forceinline__ void stage(Slice& s, const Lanes& L, double dt_use, double inv_dt) {
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    double value;
    if constexpr (S == 0) {
#if MDX_TEAM_AUTONOMOUS
      value = s.f[j];
#else
      value = s.f[j] + dt_use * coef_d(0) * s.dT[j];
#endif
    } else {
      double acc = coef_c(S, 0) * (double)s.k[0][j];
#pragma unroll
      for (int m = 1; m < S; ++m) acc += coef_c(S, m) * (double)s.k[m][j];
#if !MDX_TEAM_AUTONOMOUS
      if constexpr (coef_d(S) != 0.0) {
        value = s.f[j] + dt_use * coef_d(S) * s.dT[j] + acc * inv_dt;
      } else {
        value = s.f[j] + acc * inv_dt;
      }
#else
      value = s.f[j] + acc * inv_dt;
#endif
    }
    s.k[S][j] = (lu_t)value;
  }
  __syncwarp(L.mask);
  solve(s, s.k[S], L);
}

template <int S>
__device__ __forceinline__ void advance(Slice& s, const Lanes& L) {
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    double acc = coef_a(S, 0) * (double)s.k[0][j];
#pragma unroll
    for (int m = 1; m <= S; ++m) acc += coef_a(S, m) * (double)s.k[m][j];
    s.u[j] = s.y[j] + acc;
  }
  __syncwarp(L.mask);
}

__device__ __forceinline__ void accumulate(Slice& s, const Lanes& L, int S) {
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) s.u[j] += (double)s.k[S][j];
  __syncwarp(L.mask);
}

__device__ __forceinline__ void rhs(Slice& s, const Lanes& L, const double* y, double t) {
  mdx_team_rhs(y, t, s.p, s.f, L.lane);
  __syncwarp(L.mask);
}

__device__ __forceinline__ void step(State& st, Slice& s, const Lanes& L, const MdxSolveArgs& a) {
  double dt_use = st.dt;
  if (dt_use > st.tf_local - st.t) dt_use = st.tf_local - st.t;
  if (dt_use < 1e-30) dt_use = 1e-30;
  const double t = st.t;
  const double t_end = t + dt_use;
#if MDX_FAST
  const double inv_dt = recip_newton(dt_use);
  const double dtgamma_inv = inv_dt * (1.0 / GAMMA);
#else
  const double inv_dt = 1.0 / dt_use;
  const double dtgamma_inv = 1.0 / (dt_use * GAMMA);
#endif

  // M = I/(h gamma) - J.
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
  stage<0>(s, L, dt_use, inv_dt);
  advance<0>(s, L);
  rhs(s, L, s.u, t + coef_ct(0) * dt_use);
  stage<1>(s, L, dt_use, inv_dt);
  advance<1>(s, L);
  rhs(s, L, s.u, t + coef_ct(1) * dt_use);
  stage<2>(s, L, dt_use, inv_dt);
  advance<2>(s, L);
  rhs(s, L, s.u, t + coef_ct(2) * dt_use);
  stage<3>(s, L, dt_use, inv_dt);
  advance<3>(s, L);
  rhs(s, L, s.u, t + coef_ct(3) * dt_use);
  stage<4>(s, L, dt_use, inv_dt);
  advance<4>(s, L);
  rhs(s, L, s.u, t_end);
  stage<5>(s, L, dt_use, inv_dt);
  accumulate(s, L, 5);
  rhs(s, L, s.u, t_end);
  stage<6>(s, L, dt_use, inv_dt);
  accumulate(s, L, 6);
  rhs(s, L, s.u, t_end);
  stage<7>(s, L, dt_use, inv_dt);

  // Weighted RMS of k8 (modax/rodas5P.py:903-911): scaled terms by component on
  // the owning lanes, then the sum of squares in component order on every lane.
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
    const double k7 = (double)s.k[7][j];
    const double y_new_j = s.u[j] + k7;
    const double scale = a.atol + a.rtol * pymax(fabs(s.y[j]), fabs(y_new_j));
#if MDX_FAST
    s.f[j] = weight(a, st.traj, j) * k7 * recip_newton(scale);
#else
    s.f[j] = weight(a, st.traj, j) * k7 / scale;
#endif
  }
  __syncwarp(L.mask);
  double err_local = 0.0;
#pragma unroll 8
  for (int j = 0; j < MDX_NV; ++j) err_local += s.f[j] * s.f[j];
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
    // The thread kernel's checkpoint layout (mdx_common.cuh::ckpt_write): the
    // step size, and every MDX_CKPT_SEG-th step's start (t, y), y by component.
    if (st.n_ckpt < a.ckpt_capacity) {
      if (L.lane == 0) a.ckpt[(size_t)st.n_ckpt * (size_t)a.n_traj + (size_t)st.traj] = dt_use;
      if (st.n_ckpt % MDX_CKPT_SEG == 0) {
        double* rec = ckpt_state(a.ckpt, a.ckpt_capacity, a.n_traj, st.n_ckpt / MDX_CKPT_SEG, st.traj);
        if (L.lane == 0) rec[0] = t;
        for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) rec[1 + j] = s.y[j];
      }
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
#if MDX_HAS_HOOK
      // Every lane has read the error terms in f before any lane overwrites them
      // with this save's state.
      __syncwarp(L.mask);
#endif
#if MDX_FAST
      // The thread kernel's shared stage weights (mdx_rodas5p.cuh).
      double w[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) w[m] = coef_h(0, m) + theta * (coef_h(1, m) + theta * coef_h(2, m));
#endif
      for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) {
#if MDX_FAST
        double hsum = w[0] * (double)s.k[0][j];
#pragma unroll
        for (int m = 1; m < 8; ++m) hsum += w[m] * (double)s.k[m][j];
        const double y_new_j = s.u[j] + (double)s.k[7][j];
        const double val = theta1 * s.y[j] + theta * (y_new_j + theta1 * hsum);
#else
        double h1 = coef_h(0, 0) * (double)s.k[0][j];
        double h2 = coef_h(1, 0) * (double)s.k[0][j];
        double h3 = coef_h(2, 0) * (double)s.k[0][j];
#pragma unroll
        for (int m = 1; m < 8; ++m) {
          h1 += coef_h(0, m) * (double)s.k[m][j];
          h2 += coef_h(1, m) * (double)s.k[m][j];
          h3 += coef_h(2, m) * (double)s.k[m][j];
        }
        const double y_new_j = s.u[j] + (double)s.k[7][j];
        const double val = theta1 * s.y[j] + theta * (y_new_j + theta1 * (h1 + theta * (h2 + theta * h3)));
#endif
#if MDX_SAVE_HISTORY
        a.hist[hist_index(a, st.traj, st.save_idx, j)] = val;
#endif
#if MDX_HAS_HOOK
        s.f[j] = val;  // the error terms in f are no longer needed
#else
        (void)val;
#endif
      }
#if MDX_HAS_HOOK
      __syncwarp(L.mask);
      if (L.lane == 0)
        mdx_save_hook(st.save_idx, s.f, a.times[st.save_idx], s.p, a.hook_out + (size_t)st.traj * MDX_HOOK_SIZE);
      __syncwarp(L.mask);
#endif
      ++st.save_idx;
    }
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) s.y[j] = s.u[j] + (double)s.k[7][j];
    st.t += dt_use;
    ++st.accepted;
  } else {
    ++st.rejected;
  }
  ++st.n_steps;
  __syncwarp(L.mask);
}

__device__ __forceinline__ void finish(State& st, Slice& s, const Lanes& L, const MdxSolveArgs& a) {
  const bool hit_max = st.save_idx < a.n_save && st.t < st.tf_local;
  // Saves past this trajectory's end hold its final state (modax/rodas5P.py:991-1002).
  while (st.save_idx < a.n_save) {
#if MDX_SAVE_HISTORY
    for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) a.hist[hist_index(a, st.traj, st.save_idx, j)] = s.y[j];
#endif
#if MDX_HAS_HOOK
    if (L.lane == 0)
      mdx_save_hook(st.save_idx, s.y, a.times[st.save_idx], s.p, a.hook_out + (size_t)st.traj * MDX_HOOK_SIZE);
#endif
    ++st.save_idx;
  }
#if !MDX_SAVE_HISTORY
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) a.hist[hist_index(a, st.traj, 0, j)] = s.y[j];
#endif
  bool bad = false;
  for (int j = L.lane; j < MDX_NV; j += MDX_TEAM) bad |= !isfinite(s.y[j]);
  bad = __any_sync(L.mask, bad);
  if (L.lane == 0) {
    a.accepted[st.traj] = st.accepted;
    a.rejected[st.traj] = st.rejected;
    a.loop_steps[st.traj] = st.n_steps;
    int status = (hit_max ? MDX_STATUS_MAX_STEPS : MDX_STATUS_OK) | (bad ? MDX_STATUS_NONFINITE : 0);
#if MDX_CHECKPOINT
    if (a.ckpt_count) a.ckpt_count[st.traj] = st.n_ckpt;
    if (st.ckpt_overflow) status |= MDX_STATUS_CKPT_OVERFLOW;
#endif
    if (a.status) a.status[st.traj] = status;
  }
  __syncwarp(L.mask);
  if (a.hist_host != nullptr) {
    // The team copies its finished row to the page-locked host copy; the barrier
    // above ordered every lane's history stores before these L2 reads.
    const size_t row = (size_t)a.n_save_hist * (size_t)MDX_NV;
    const double* src = a.hist + (size_t)st.traj * row;
    double* dst = a.hist_host + (size_t)st.traj * row;
    for (size_t k = L.lane; k < row; k += MDX_TEAM) dst[k] = __ldcg(src + k);
  }
}

}  // namespace team
}  // namespace mdx

// One trajectory per team for its whole life; blockDim.x / MDX_TEAM
// trajectories per block.
extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_plain(const MdxSolveArgs a) {
  using namespace mdx::team;
  const int traj = blockIdx.x * TEAMS_PER_BLOCK + (int)(threadIdx.x / MDX_TEAM);
  if (traj >= a.n_traj) return;  // whole teams leave together
  const Lanes L = lanes();
  Slice& s = *slice_of_team();
  State st;
  init(st, s, L, a, traj);
  while (running(st, a)) step(st, s, L, a);
  finish(st, s, L, a);
}

// A device-sized grid whose teams take trajectories off an atomic queue until it
// runs dry: one atomicAdd per trajectory by the team's first lane, broadcast to
// the team.  Nothing waits on another team.
extern "C" __global__ void __launch_bounds__(MDX_TPB, MDX_MIN_BLOCKS)
mdx_solve_persistent(const MdxSolveArgs a) {
  using namespace mdx::team;
  const Lanes L = lanes();
  Slice& s = *slice_of_team();
  while (true) {
    int slot = 0;
    if (L.lane == 0) slot = atomicAdd(a.work_counter, 1);
    slot = __shfl_sync(L.mask, slot, 0, MDX_TEAM);
    if (slot >= a.n_traj) break;
    const int traj = a.order ? a.order[slot] : slot;
    State st;
    init(st, s, L, a, traj);
    while (running(st, a)) step(st, s, L, a);
    finish(st, s, L, a);
  }
}
