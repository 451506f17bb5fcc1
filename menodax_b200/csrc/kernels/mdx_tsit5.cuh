// Tsit5 (explicit Runge-Kutta 5(4), FSAL), one trajectory per thread.
//
// Restates the reference body (modax/tsit5.py:193-404) as a state/step/finish
// triple shared by the one-launch and the persistent refill kernels.  The nine
// per-trajectory vectors (y, u, k1..k7) are register arrays: every component
// index is a compile-time constant.  State kept across steps: y, k7 (the FSAL
// stage), t, dt, the PID error history, the save cursor and the counters.
//
// With MDX_TSIT5_SHARED the stages k1..k6 live in shared memory instead, the
// reference's "shared" backend (modax/tsit5.py:117-139, 433-602): a
// (6, n, MDX_TPB) array per block, each thread one column, so a warp's access to
// component j of a stage is 32 consecutive doubles.  It takes 6n doubles per
// trajectory out of the register file, which matters once n reaches ~16.
#pragma once
#include "mdx_common.cuh"

namespace mdx {
namespace tsit5 {

// Tsitouras (2011) coefficients, as tabulated in modax/tsit5.py:33-82.
constexpr double C2 = 0.161, C3 = 0.327, C4 = 0.9, C5 = 0.9800255409045097;
constexpr double A21 = 0.161;
constexpr double A31 = -0.008480655492356989, A32 = 0.335480655492357;
constexpr double A41 = 2.8971530571054935, A42 = -6.359448489975075, A43 = 4.3622954328695815;
constexpr double A51 = 5.325864828439257, A52 = -11.748883564062828, A53 = 7.4955393428898365,
                 A54 = -0.09249506636175525;
constexpr double A61 = 5.86145544294642, A62 = -12.92096931784711, A63 = 8.159367898576159,
                 A64 = -0.071584973281401, A65 = -0.028269050394068383;
constexpr double B1 = 0.09646076681806523, B2 = 0.01, B3 = 0.4798896504144996,
                 B4 = 1.379008574103742, B5 = -3.2900695154360807, B6 = 2.324710524099774;
constexpr double E1 = 0.0017800110522257773, E2 = 0.0008164344596567463,
                 E3 = -0.007880878010261994, E4 = 0.1447110071732629,
                 E5 = -0.5823571654525552, E6 = 0.45808210592918686, E7 = -1.0 / 66.0;
constexpr double FACTOR_MIN = 0.2;
constexpr double FACTOR_MAX = 10.0;

struct State {
  double y[MDX_NS];
  double k7[MDX_NS];
  double p[MDX_NP > 0 ? MDX_NP : 1];
  double t, dt, tf, err_prev, err_prev2;
  int save_idx, n_steps, accepted, rejected, traj;
  bool has_fsal;
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

// Dense-output weights b1..b7 at theta (Tsitouras 2011 continuous extension,
// modax/tsit5.py:307-344).
__device__ __forceinline__ void dense_weights(double th, double b[7]) {
  b[0] = -1.0530884977290216 * th * (th - 1.3299890189751412) *
         (th * th - 1.4364028541716351 * th + 0.7139816917074209);
  b[1] = 0.1017 * th * th * (th * th - 2.1966568338249754 * th + 1.2949852507374631);
  b[2] = 2.490627285651252793 * th * th * (th * th - 2.38535645472061657 * th + 1.57803468208092486);
  b[3] = -16.54810288924490272 * (th - 1.21712927295533244) * (th - 0.61620406037800089) * th * th;
  b[4] = 47.37952196281928122 * (th - 1.203071208372362603) * (th - 0.658047292653547382) * th * th;
  b[5] = -34.87065786149660974 * (th - 1.2) * (th - 0.666666666666666667) * th * th;
  b[6] = 2.5 * (th - 1.0) * (th - 0.6) * th * th;
}

__device__ __forceinline__ void init(State& st, const MdxSolveArgs& a, int traj) {
  st.traj = traj;
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) {
    st.y[j] = a.y0[(size_t)traj * MDX_NS + j];
    a.hist[hist_index(a, traj, 0, j)] = st.y[j];
    st.k7[j] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < MDX_NP; ++k) st.p[k] = a.params[(size_t)traj * MDX_NP + k];
  st.t = a.times[0];
  st.tf = a.times[a.n_save - 1];
  st.dt = a.dt0 > 0.0 ? a.dt0 : (st.tf - st.t) * 1e-6;
  st.save_idx = 1;
  st.n_steps = 0;
  st.accepted = 0;
  st.rejected = 0;
  st.has_fsal = false;
  st.err_prev = 1.0;
  st.err_prev2 = 1.0;
#if MDX_CHECKPOINT
  st.n_ckpt = 0;
  st.ckpt_overflow = false;
#endif
}

__device__ __forceinline__ bool running(const State& st, const MdxSolveArgs& a) {
  return st.save_idx < a.n_save && st.t < st.tf && st.n_steps < a.max_steps;
}

#if MDX_TSIT5_SHARED
// One thread's column of a stage array in shared memory.  The accesses are
// volatile so every use reads shared memory: otherwise the compiler keeps the
// loaded stage values in registers, which is the pressure the placement is
// there to remove (at 16 components: 236 registers and no spills, against 255
// registers and 450 B of local-memory spills with the stages in registers).
struct StageColumn {
  volatile double* base;
  __device__ __forceinline__ volatile double& operator[](int j) const { return base[j * MDX_TPB]; }
};

__device__ __forceinline__ StageColumn stage_column(int s) {
  __shared__ double mdx_tsit5_stages[6][MDX_NS][MDX_TPB];
  return StageColumn{&mdx_tsit5_stages[s][0][threadIdx.x]};
}
#endif

__device__ __forceinline__ void step(State& st, const MdxSolveArgs& a) {
  double dt_use = st.dt;
  if (dt_use > st.tf - st.t) dt_use = st.tf - st.t;
  if (dt_use < 1e-30) dt_use = 1e-30;
  const double t = st.t;

#if MDX_TSIT5_SHARED
  const StageColumn k1 = stage_column(0), k2 = stage_column(1), k3 = stage_column(2),
                    k4 = stage_column(3), k5 = stage_column(4), k6 = stage_column(5);
  double u[MDX_NS];
#else
  double k1[MDX_NS], k2[MDX_NS], k3[MDX_NS], k4[MDX_NS], k5[MDX_NS], k6[MDX_NS], u[MDX_NS];
#endif
  if (st.has_fsal) {
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) k1[j] = st.k7[j];
  } else {
    mdx_rhs(st.y, t, st.p, k1);
  }
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) u[j] = st.y[j] + dt_use * (A21 * k1[j]);
  mdx_rhs(u, t + C2 * dt_use, st.p, k2);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) u[j] = st.y[j] + dt_use * (A31 * k1[j] + A32 * k2[j]);
  mdx_rhs(u, t + C3 * dt_use, st.p, k3);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j)
    u[j] = st.y[j] + dt_use * (A41 * k1[j] + A42 * k2[j] + A43 * k3[j]);
  mdx_rhs(u, t + C4 * dt_use, st.p, k4);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j)
    u[j] = st.y[j] + dt_use * (A51 * k1[j] + A52 * k2[j] + A53 * k3[j] + A54 * k4[j]);
  mdx_rhs(u, t + C5 * dt_use, st.p, k5);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j)
    u[j] = st.y[j] + dt_use * (A61 * k1[j] + A62 * k2[j] + A63 * k3[j] + A64 * k4[j] + A65 * k5[j]);
  mdx_rhs(u, t + 1.0 * dt_use, st.p, k6);
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j)
    u[j] = st.y[j] + dt_use * (B1 * k1[j] + B2 * k2[j] + B3 * k3[j] + B4 * k4[j] + B5 * k5[j] +
                               B6 * k6[j]);
  mdx_rhs(u, t + 1.0 * dt_use, st.p, st.k7);

  double err_sum = 0.0;
#pragma unroll
  for (int j = 0; j < MDX_NS; ++j) {
    const double err_est = dt_use * (E1 * k1[j] + E2 * k2[j] + E3 * k3[j] + E4 * k4[j] +
                                     E5 * k5[j] + E6 * k6[j] + E7 * st.k7[j]);
    const double scale = a.atol + a.rtol * pymax(fabs(st.y[j]), fabs(u[j]));
    const double r = weight(a, st.traj, j) * err_est / scale;
    err_sum += r * r;
  }
  const double err_norm = sqrt(err_sum / MDX_NERR);
  const bool accept = err_norm <= 1.0 && !isnan(err_norm);

  double t_new = t;
  if (accept) {
#if MDX_CHECKPOINT
    if (st.n_ckpt < a.ckpt_capacity) {
      ckpt_write(a, st.traj, st.n_ckpt, t, dt_use, st.y);
      ++st.n_ckpt;
    } else {
      st.ckpt_overflow = true;
    }
#endif
    t_new = t + dt_use;
    while (st.save_idx < a.n_save && save_reached(a.times[st.save_idx], t_new)) {
      const double theta = (a.times[st.save_idx] - t) / dt_use;
      double b[7];
      dense_weights(theta, b);
#pragma unroll
      for (int j = 0; j < MDX_NS; ++j) {
        a.hist[hist_index(a, st.traj, st.save_idx, j)] =
            st.y[j] + dt_use * (b[0] * k1[j] + b[1] * k2[j] + b[2] * k3[j] + b[3] * k4[j] +
                                b[4] * k5[j] + b[5] * k6[j] + b[6] * st.k7[j]);
      }
      ++st.save_idx;
    }
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) st.y[j] = u[j];
    ++st.accepted;
    st.has_fsal = true;
  } else {
    ++st.rejected;
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) st.k7[j] = 0.0;
    st.has_fsal = false;
  }

  double safe_err;
  double factor = controller_factor(err_norm, st.err_prev, st.err_prev2, MDX_E1, MDX_E2, MDX_E3,
                                    MDX_USE_E2, MDX_USE_E3, safe_err);
  if (accept) {
    st.err_prev2 = st.err_prev;
    st.err_prev = safe_err;
  }
  if (factor < FACTOR_MIN) factor = FACTOR_MIN;
  else if (factor > FACTOR_MAX) factor = FACTOR_MAX;
  st.dt = dt_use * factor;
  st.t = t_new;
  ++st.n_steps;
}

__device__ __forceinline__ void finish(State& st, const MdxSolveArgs& a) {
  const bool hit_max = st.save_idx < a.n_save;
  // The reference leaves unreached save rows unwritten (modax/tsit5.py:238);
  // here they read NaN and the status says why.
  for (int s = st.save_idx; s < a.n_save; ++s) {
#pragma unroll
    for (int j = 0; j < MDX_NS; ++j) a.hist[hist_index(a, st.traj, s, j)] = nan_value();
  }
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

}  // namespace tsit5

struct Tsit5 {
  typedef tsit5::State State;
  static __device__ __forceinline__ void init(State& s, const MdxSolveArgs& a, int i) { tsit5::init(s, a, i); }
  static __device__ __forceinline__ bool running(const State& s, const MdxSolveArgs& a) { return tsit5::running(s, a); }
  static __device__ __forceinline__ void step(State& s, const MdxSolveArgs& a) { tsit5::step(s, a); }
  static __device__ __forceinline__ void finish(State& s, const MdxSolveArgs& a) { tsit5::finish(s, a); }
};

}  // namespace mdx
