// TEST INFRASTRUCTURE -- the CPU oracle.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this; the product never does.
//
// A line-by-line CPU restatement of the reference solvers:
//   Tsit5   : modax/tsit5.py:193-404 (tableau 33-82, controller 85-90)
//   Rodas5P : modax/rodas5P.py:761-1005 (tableau 44-105, controller 108-113,
//             913-928; dense output 930-982; frozen saves 991-1005)
//   dense LU: modax/rodas5P.py:167-238 (partial pivoting, mixed typing)
//   sparse LU: modax/_sparse_direct.py:472-622 (up-looking, no pivot,
//             reciprocal diagonal), read straight off the CSR image
//   forward sensitivities: modax/_sensitivity.py:198-243,
//             modax/rodas5P.py:403-437, 513-583
// The LU type T (float or double) is rounded at the reference's points:
// -J and the diagonal shift stored in T, the stage right-hand side cast to T,
// the solves in T, the stage increments k stored in T.
//
// Right-hand sides are C++ templates over the scalar type, so exact first and
// second directional derivatives come from dual numbers (forward mode), the way
// the reference's Enzyme jvp / jvp-of-jvp supplies them -- independent of the
// product's own tracer.  A ctypes callback system covers ad-hoc test problems.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- dual numbers
template <class T>
struct Dual {
  T v, d;
  Dual() : v(0), d(0) {}
  Dual(double x) : v(x), d(0) {}
  Dual(T a, T b) : v(a), d(b) {}
};
template <class T> Dual<T> operator+(const Dual<T>& a, const Dual<T>& b) { return {a.v + b.v, a.d + b.d}; }
template <class T> Dual<T> operator-(const Dual<T>& a, const Dual<T>& b) { return {a.v - b.v, a.d - b.d}; }
template <class T> Dual<T> operator-(const Dual<T>& a) { return {-a.v, -a.d}; }
template <class T> Dual<T> operator*(const Dual<T>& a, const Dual<T>& b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
template <class T> Dual<T> operator/(const Dual<T>& a, const Dual<T>& b) {
  T q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
template <class T> Dual<T> operator+(const Dual<T>& a, double b) { return a + Dual<T>(b); }
template <class T> Dual<T> operator+(double a, const Dual<T>& b) { return Dual<T>(a) + b; }
template <class T> Dual<T> operator-(const Dual<T>& a, double b) { return a - Dual<T>(b); }
template <class T> Dual<T> operator-(double a, const Dual<T>& b) { return Dual<T>(a) - b; }
template <class T> Dual<T> operator*(const Dual<T>& a, double b) { return a * Dual<T>(b); }
template <class T> Dual<T> operator*(double a, const Dual<T>& b) { return Dual<T>(a) * b; }
template <class T> Dual<T> operator/(const Dual<T>& a, double b) { return a / Dual<T>(b); }
template <class T> Dual<T> operator/(double a, const Dual<T>& b) { return Dual<T>(a) / b; }

typedef Dual<double> D1;
typedef Dual<D1> D2;

// ---------------------------------------------------------------- systems
enum { SYS_LORENZ = 1, SYS_ROBERTSON = 2, SYS_VDP_RING = 3, SYS_BRUSSELATOR = 4,
       SYS_CASCADE = 5, SYS_FORCED = 6, SYS_EXP_DECAY = 7, SYS_CALLBACK = 100 };

typedef void (*f_cb_t)(const double* y, double t, const double* p, double* out);
typedef void (*jvp_cb_t)(const double* y, double t, const double* p, const double* vy, double vt,
                         const double* vp, double* out);
typedef void (*jvp2_cb_t)(const double* y, double t, const double* p, const double* uy, double ut,
                          const double* up, const double* vy, double vt, const double* vp,
                          double* out);

struct SystemDesc {
  int kind;
  int n, np;
  const double* cfg;
  int n_cfg;
  f_cb_t f_cb;
  jvp_cb_t jvp_cb;
  jvp2_cb_t jvp2_cb;
};

// Lorenz: sigma = 10, beta = 8/3, p0 = rho (reference/systems/python/lorenz.py:36-43).
template <class T>
void lorenz(const T* y, T t, const T* p, T* out) {
  (void)t;
  const double sigma = 10.0, beta = 8.0 / 3.0;
  out[0] = sigma * (y[1] - y[0]);
  out[1] = y[0] * (p[0] - y[2]) - y[1];
  out[2] = y[0] * y[1] - beta * y[2];
}

// Robertson, rate order of reference/systems/python/robertson.py:13-22.
template <class T>
void robertson(const T* y, T t, const T* p, T* out) {
  (void)t;
  out[0] = -p[0] * y[0] + p[1] * y[1] * y[2];
  out[1] = p[0] * y[0] - p[1] * y[1] * y[2] - p[2] * (y[1] * y[1]);
  out[2] = p[2] * (y[1] * y[1]);
}

// Ring of Van der Pol oscillators, nearest-neighbour diffusive coupling on x
// (reference/systems/python/vdp.py:63-79); cfg = {n_osc, mu, d, omega}.  Each
// component ends in "+ 0.0" as the generated callbacks do (_tuple_codegen.py:30).
template <class T>
void vdp_ring(const T* y, T t, const T* p, T* out, const double* cfg) {
  (void)t;
  const int n_osc = (int)cfg[0];
  const double mu = cfg[1], d = cfg[2], omega = cfg[3];
  for (int osc = 0; osc < n_osc; ++osc) {
    const int b = 2 * osc;
    const T x = y[b], v = y[b + 1];
    int others[2];
    int n_others = 0;
    const int left = (osc - 1 + n_osc) % n_osc, right = (osc + 1) % n_osc;
    if (left != osc) others[n_others++] = left;
    if (right != osc) others[n_others++] = right;
    T lap;
    if (n_others == 0) {
      lap = (-0.0) * x;
    } else {
      lap = y[2 * others[0]];
      for (int k = 1; k < n_others; ++k) lap = lap + y[2 * others[k]];
      lap = lap + (-((double)n_others)) * x;
    }
    out[b] = v + 0.0;
    out[b + 1] = p[0] * mu * (1.0 - x * x) * v + (-(omega * omega)) * x + d * lap + 0.0;
  }
}

// 1-D periodic Brusselator, interleaved u_i = y[2i], v_i = y[2i+1];
// cfg = {n_grid, A, alpha}; p0 = B.  du = A + u^2 v - (B + 1) u + D lap(u),
// dv = B u - u^2 v + D lap(v), D = alpha / dx^2 (reference/systems/python/
// brusselator.py:143-165, with B taken from p0 and A fixed).
template <class T>
void brusselator(const T* y, T t, const T* p, T* out, const double* cfg) {
  (void)t;
  const int ng = (int)cfg[0];
  const double A = cfg[1], alpha = cfg[2];
  const double dx = 1.0 / ng;
  const double D = alpha / (dx * dx);
  for (int g = 0; g < ng; ++g) {
    const int l = (g - 1 + ng) % ng, r = (g + 1) % ng;
    const int u = 2 * g, v = u + 1;
    const T u2v = y[u] * y[u] * y[v];
    out[u] = A + u2v - (p[0] + 1.0) * y[u] + D * (y[2 * l] + (-2.0) * y[u] + y[2 * r]) + 0.0;
    out[v] = p[0] * y[u] - u2v + D * (y[2 * l + 1] + (-2.0) * y[v] + y[2 * r + 1]) + 0.0;
  }
}

// Linear cascade y0' = -a y0, y1' = a y0 - b y1 (tests/test_sensitivity.py:41-42).
template <class T>
void cascade(const T* y, T t, const T* p, T* out) {
  (void)t;
  out[0] = -p[0] * y[0];
  out[1] = p[0] * y[0] - p[1] * y[1];
}

// Forced decay y' = -lam y + F t (tests/test_solver_options.py:29-31).
template <class T>
void forced(const T* y, T t, const T* p, T* out) {
  out[0] = -p[0] * y[0] + p[1] * t;
}

template <class T>
void exp_decay(const T* y, T t, const T* p, T* out, int n) {
  (void)t;
  for (int i = 0; i < n; ++i) out[i] = -p[0] * y[i];
}

template <class T>
void eval(const SystemDesc& s, const T* y, T t, const T* p, T* out) {
  switch (s.kind) {
    case SYS_LORENZ: lorenz(y, t, p, out); break;
    case SYS_ROBERTSON: robertson(y, t, p, out); break;
    case SYS_VDP_RING: vdp_ring(y, t, p, out, s.cfg); break;
    case SYS_BRUSSELATOR: brusselator(y, t, p, out, s.cfg); break;
    case SYS_CASCADE: cascade(y, t, p, out); break;
    case SYS_FORCED: forced(y, t, p, out); break;
    case SYS_EXP_DECAY: exp_decay(y, t, p, out, s.n); break;
    default: break;
  }
}

void f(const SystemDesc& s, const double* y, double t, const double* p, double* out) {
  if (s.kind == SYS_CALLBACK) { s.f_cb(y, t, p, out); return; }
  eval<double>(s, y, t, p, out);
}

// D f(y, t, p)[vy, vt, vp]
void jvp(const SystemDesc& s, const double* y, double t, const double* p, const double* vy,
         double vt, const double* vp, double* out) {
  if (s.kind == SYS_CALLBACK) { s.jvp_cb(y, t, p, vy, vt, vp, out); return; }
  std::vector<D1> yy(s.n), pp(s.np > 0 ? s.np : 1), oo(s.n);
  for (int i = 0; i < s.n; ++i) yy[i] = D1(y[i], vy ? vy[i] : 0.0);
  for (int k = 0; k < s.np; ++k) pp[k] = D1(p[k], vp ? vp[k] : 0.0);
  eval<D1>(s, yy.data(), D1(t, vt), pp.data(), oo.data());
  for (int i = 0; i < s.n; ++i) out[i] = oo[i].d;
}

// D^2 f(y, t, p)[u, v]
void jvp2(const SystemDesc& s, const double* y, double t, const double* p, const double* uy,
          double ut, const double* up, const double* vy, double vt, const double* vp, double* out) {
  if (s.kind == SYS_CALLBACK) { s.jvp2_cb(y, t, p, uy, ut, up, vy, vt, vp, out); return; }
  std::vector<D2> yy(s.n), pp(s.np > 0 ? s.np : 1), oo(s.n);
  for (int i = 0; i < s.n; ++i) yy[i] = D2(D1(y[i], uy ? uy[i] : 0.0), D1(vy ? vy[i] : 0.0, 0.0));
  for (int k = 0; k < s.np; ++k) pp[k] = D2(D1(p[k], up ? up[k] : 0.0), D1(vp ? vp[k] : 0.0, 0.0));
  eval<D2>(s, yy.data(), D2(D1(t, ut), D1(vt, 0.0)), pp.data(), oo.data());
  for (int i = 0; i < s.n; ++i) out[i] = oo[i].d.d;
}

// ---------------------------------------------------------------- problem
struct Layout {
  int n_colours;
  const int* colour;   // (n,)
  int lu_size;
  const int* store;    // (n * n_colours) slot of each (row, colour), -1 none; NULL: grid
  const int* diag;     // (n,)
  int sparse;
  const int* row_ptr;  // CSR of L+U in elimination order
  const int* col_ind;
  const int* diag_ptr;
  const int* order;
};

struct Sens {
  int n_sens;          // 0: plain solve
  int n_y0_dirs;
  const int* param_cols;
  int error_control;
};

struct Controls {
  double dt0, rtol, atol;
  int max_steps;
  double pcoeff, icoeff, dcoeff;
  int tf_index;
};

struct Ensemble {
  int N, n_system, np, S;
  const double* y0;
  const double* times;
  const double* params;
  const double* weights;  // NULL: ones
  double* hist;
  int* accepted;
  int* rejected;
  int* loop;
};

// The augmented right-hand side [f, J S_k + J_p,k] (modax/_sensitivity.py:198-243).
void f_system(const SystemDesc& s, const Sens& sens, const double* z, double t, const double* p,
              double* out, std::vector<double>& tmp_dir_p) {
  const int n = s.n;
  f(s, z, t, p, out);
  for (int k = 0; k < sens.n_sens; ++k) {
    const int base = n + k * n;
    std::fill(tmp_dir_p.begin(), tmp_dir_p.end(), 0.0);
    if (k >= sens.n_y0_dirs) tmp_dir_p[sens.param_cols[k - sens.n_y0_dirs]] = 1.0;
    jvp(s, z, t, p, z + base, 0.0, tmp_dir_p.data(), out + base);
  }
}

inline double pymax(double a, double b) { return b > a ? b : a; }

// ---------------------------------------------------------------- Tsit5
void tsit5_one(const SystemDesc& s, const Sens& sens, const Controls& c, const Ensemble& e, int i) {
  const double A21 = 161.0 / 1000.0;
  const double A31 = -0.008480655492356989, A32 = 0.335480655492357;
  const double A41 = 2.8971530571054935, A42 = -6.359448489975075, A43 = 4.3622954328695815;
  const double A51 = 5.325864828439257, A52 = -11.748883564062828, A53 = 7.4955393428898365,
               A54 = -0.09249506636175525;
  const double A61 = 5.86145544294642, A62 = -12.92096931784711, A63 = 8.159367898576159,
               A64 = -0.071584973281401, A65 = -0.028269050394068383;
  const double B1 = 0.09646076681806523, B2 = 0.01, B3 = 0.4798896504144996,
               B4 = 1.379008574103742, B5 = -3.2900695154360807, B6 = 2.324710524099774;
  const double E1 = 0.0017800110522257773, E2 = 0.0008164344596567463,
               E3 = -0.007880878010261994, E4 = 0.1447110071732629, E5 = -0.5823571654525552,
               E6 = 0.45808210592918686, E7 = -1.0 / 66.0;
  const double C2 = 161.0 / 1000.0, C3 = 327.0 / 1000.0, C4 = 9.0 / 10.0,
               C5 = 0.9800255409045097;
  const double EXPONENT = -1.0 / 5.0;
  const double e1 = EXPONENT * (c.icoeff + c.pcoeff + c.dcoeff);
  const double e2 = -EXPONENT * (c.pcoeff + 2.0 * c.dcoeff);
  const double e3 = EXPONENT * c.dcoeff;
  const int ns = e.n_system;
  const int n_error = sens.n_sens == 0 ? s.n : (sens.error_control ? ns : s.n);
  const double* prow = e.params + (size_t)i * e.np;
  std::vector<double> y(ns), u(ns), k1(ns), k2(ns), k3(ns), k4(ns), k5(ns), k6(ns), k7(ns);
  std::vector<double> tmp(e.np > 0 ? e.np : 1);
  double* hist = e.hist + (size_t)i * e.S * ns;
  for (int j = 0; j < ns; ++j) {
    y[j] = e.y0[(size_t)i * ns + j];
    hist[j] = y[j];
    k7[j] = 0.0;
  }
  const double* times = e.times;
  double t = times[0];
  const double tf = times[e.S - 1];
  double dt = c.dt0 > 0.0 ? c.dt0 : (tf - t) * 1e-6;
  int save_idx = 1, n_steps = 0, acc = 0, rej = 0;
  bool has_fsal = false;
  double err_prev = 1.0, err_prev2 = 1.0;
  auto w = [&](int j) { return e.weights ? e.weights[(size_t)i * ns + j] : (j < s.n ? 1.0 : (sens.error_control ? 1.0 : 0.0)); };
  while (save_idx < e.S && t < tf && n_steps < c.max_steps) {
    double h = dt;
    if (h > tf - t) h = tf - t;
    if (h < 1e-30) h = 1e-30;
    if (has_fsal) k1 = k7;
    else f_system(s, sens, y.data(), t, prow, k1.data(), tmp);
    for (int j = 0; j < ns; ++j) u[j] = y[j] + h * (A21 * k1[j]);
    f_system(s, sens, u.data(), t + C2 * h, prow, k2.data(), tmp);
    for (int j = 0; j < ns; ++j) u[j] = y[j] + h * (A31 * k1[j] + A32 * k2[j]);
    f_system(s, sens, u.data(), t + C3 * h, prow, k3.data(), tmp);
    for (int j = 0; j < ns; ++j) u[j] = y[j] + h * (A41 * k1[j] + A42 * k2[j] + A43 * k3[j]);
    f_system(s, sens, u.data(), t + C4 * h, prow, k4.data(), tmp);
    for (int j = 0; j < ns; ++j) u[j] = y[j] + h * (A51 * k1[j] + A52 * k2[j] + A53 * k3[j] + A54 * k4[j]);
    f_system(s, sens, u.data(), t + C5 * h, prow, k5.data(), tmp);
    for (int j = 0; j < ns; ++j)
      u[j] = y[j] + h * (A61 * k1[j] + A62 * k2[j] + A63 * k3[j] + A64 * k4[j] + A65 * k5[j]);
    f_system(s, sens, u.data(), t + 1.0 * h, prow, k6.data(), tmp);
    for (int j = 0; j < ns; ++j)
      u[j] = y[j] + h * (B1 * k1[j] + B2 * k2[j] + B3 * k3[j] + B4 * k4[j] + B5 * k5[j] + B6 * k6[j]);
    f_system(s, sens, u.data(), t + 1.0 * h, prow, k7.data(), tmp);
    double err_sum = 0.0;
    for (int j = 0; j < ns; ++j) {
      double est = h * (E1 * k1[j] + E2 * k2[j] + E3 * k3[j] + E4 * k4[j] + E5 * k5[j] + E6 * k6[j] + E7 * k7[j]);
      double scale = c.atol + c.rtol * pymax(std::fabs(y[j]), std::fabs(u[j]));
      double r = w(j) * est / scale;
      err_sum += r * r;
    }
    double err = std::sqrt(err_sum / n_error);
    bool accept = err <= 1.0 && !std::isnan(err);
    double t_new = t;
    if (accept) {
      t_new = t + h;
      while (save_idx < e.S && times[save_idx] <= t_new + 1e-12 * pymax(1.0, std::fabs(times[save_idx]))) {
        double th = (times[save_idx] - t) / h;
        double b1 = -1.0530884977290216 * th * (th - 1.3299890189751412) * (th * th - 1.4364028541716351 * th + 0.7139816917074209);
        double b2 = 0.1017 * th * th * (th * th - 2.1966568338249754 * th + 1.2949852507374631);
        double b3 = 2.490627285651252793 * th * th * (th * th - 2.38535645472061657 * th + 1.57803468208092486);
        double b4 = -16.54810288924490272 * (th - 1.21712927295533244) * (th - 0.61620406037800089) * th * th;
        double b5 = 47.37952196281928122 * (th - 1.203071208372362603) * (th - 0.658047292653547382) * th * th;
        double b6 = -34.87065786149660974 * (th - 1.2) * (th - 0.666666666666666667) * th * th;
        double b7 = 2.5 * (th - 1.0) * (th - 0.6) * th * th;
        for (int j = 0; j < ns; ++j)
          hist[(size_t)save_idx * ns + j] = y[j] + h * (b1 * k1[j] + b2 * k2[j] + b3 * k3[j] + b4 * k4[j] + b5 * k5[j] + b6 * k6[j] + b7 * k7[j]);
        ++save_idx;
      }
      y = u;
      ++acc;
      has_fsal = true;
    } else {
      ++rej;
      std::fill(k7.begin(), k7.end(), 0.0);
      has_fsal = false;
    }
    double safe;
    if (std::isnan(err) || err > 1e18) safe = 1e18;
    else if (err == 0.0) safe = 1e-18;
    else safe = err;
    double factor = 0.9 * std::pow(safe, e1) * std::pow(err_prev, e2) * std::pow(err_prev2, e3);
    if (accept) { err_prev2 = err_prev; err_prev = safe; }
    if (factor < 0.2) factor = 0.2;
    else if (factor > 10.0) factor = 10.0;
    dt = h * factor;
    t = t_new;
    ++n_steps;
  }
  for (int si = save_idx; si < e.S; ++si)
    for (int j = 0; j < ns; ++j) hist[(size_t)si * ns + j] = NAN;
  e.accepted[i] = acc;
  e.rejected[i] = rej;
  e.loop[i] = n_steps;
}

// ---------------------------------------------------------------- LU
template <class T>
void dense_factorize(T* lu, int* ipiv, int n) {
  for (int i = 0; i < n; ++i) {
    T max_val = std::fabs(lu[i * n + i]);
    int pivot = i;
    for (int k = i + 1; k < n; ++k) {
      T v = std::fabs(lu[k * n + i]);
      if (v > max_val) { max_val = v; pivot = k; }
    }
    ipiv[i] = pivot;
    if (pivot != i)
      for (int j = 0; j < n; ++j) std::swap(lu[i * n + j], lu[pivot * n + j]);
    T piv = lu[i * n + i];
    if (piv != T(0)) {
      double inv_piv = 1.0 / (double)piv;
      for (int k = i + 1; k < n; ++k) {
        double factor = (double)lu[k * n + i] * inv_piv;
        lu[k * n + i] = (T)factor;
        for (int j = i + 1; j < n; ++j) lu[k * n + j] = (T)((double)lu[k * n + j] - factor * (double)lu[i * n + j]);
      }
    }
  }
}

template <class T>
void dense_solve(const T* lu, const int* ipiv, T* rhs, int n) {
  for (int i = 0; i < n; ++i) {
    int pivot = ipiv[i];
    if (pivot != i) std::swap(rhs[i], rhs[pivot]);
    T acc = rhs[i];
    for (int j = 0; j < i; ++j) acc -= lu[i * n + j] * rhs[j];
    rhs[i] = acc;
  }
  for (int i = n - 1; i >= 0; --i) {
    T acc = rhs[i];
    for (int j = i + 1; j < n; ++j) acc -= lu[i * n + j] * rhs[j];
    rhs[i] = acc / lu[i * n + i];
  }
}

// Up-looking unpivoted LU over the CSR image, diagonal left holding 1/U_ii
// (modax/_sparse_direct.py:472-546).  The destination of each update is found
// by a search of row i, not taken from precomputed tables.
template <class T>
void sparse_factorize(T* lu, const Layout& L, int n) {
  for (int i = 0; i < n; ++i) {
    const int pivot = L.diag_ptr[i];
    for (int p = L.row_ptr[i]; p < pivot; ++p) {
      const int k = L.col_ind[p];
      const int above = L.diag_ptr[k];
      const T factor = lu[p] * lu[above];
      lu[p] = factor;
      for (int q = above + 1; q < L.row_ptr[k + 1]; ++q) {
        const int col = L.col_ind[q];
        int dst = -1;
        for (int r = L.row_ptr[i]; r < L.row_ptr[i + 1]; ++r)
          if (L.col_ind[r] == col) { dst = r; break; }
        lu[dst] -= factor * lu[q];
      }
    }
    lu[pivot] = (T)(1.0 / (double)lu[pivot]);
  }
}

template <class T>
void sparse_solve(const T* lu, const Layout& L, T* rhs, int n) {
  for (int i = 0; i < n; ++i) {
    const int row = L.order[i];
    T acc = rhs[row];
    for (int p = L.row_ptr[i]; p < L.diag_ptr[i]; ++p) acc -= lu[p] * rhs[L.order[L.col_ind[p]]];
    rhs[row] = acc;
  }
  for (int i = n - 1; i >= 0; --i) {
    const int row = L.order[i];
    const int pivot = L.diag_ptr[i];
    T acc = rhs[row];
    for (int p = pivot + 1; p < L.row_ptr[i + 1]; ++p) acc -= lu[p] * rhs[L.order[L.col_ind[p]]];
    rhs[row] = acc * lu[pivot];
  }
}

// ---------------------------------------------------------------- Rodas5P
const double GAMMA = 0.21193756319429014;
const double RA[5][5] = {
    {3.0, 0, 0, 0, 0},
    {2.849394379747939, 0.45842242204463923, 0, 0, 0},
    {-6.954028509809101, 2.489845061869568, -10.358996098473584, 0, 0},
    {2.8029986275628964, 0.5072464736228206, -0.3988312541770524, -0.04721187230404641, 0},
    {-7.502846399306121, 2.561846144803919, -11.627539656261098, -0.18268767659942256, 0.030198172008377946}};
const double RC[8][7] = {
    {0, 0, 0, 0, 0, 0, 0},
    {-14.155112264123755, 0, 0, 0, 0, 0, 0},
    {-17.97296035885952, -2.859693295451294, 0, 0, 0, 0, 0},
    {147.12150275711716, -1.41221402718213, 71.68940251302358, 0, 0, 0, 0},
    {165.43517024871676, -0.4592823456491126, 42.90938336958603, -5.961986721573306, 0, 0, 0},
    {24.854864614690072, -3.0009227002832186, 47.4931110020768, 5.5814197821558125, -0.6610691825249471, 0, 0},
    {30.91273214028599, -3.1208243349937974, 77.79954646070892, 34.28646028294783, -19.097331116725623, -28.087943162872662, 0},
    {37.80277123390563, -3.2571969029072276, 112.26918849496327, 66.9347231244047, -40.06618937091002, -54.66780262877968, -9.48861652309627}};
const double RCT[4] = {0.6358126895828704, 0.4095798393397535, 0.9769306725060716, 0.4288403609558664};
const double RD[8] = {0.21193756319429014, -0.42387512638858027, -0.3384627126235924, 1.8046452872882734, 2.325825639765069, 0, 0, 0};
const double RH[3][8] = {
    {25.948786856663858, -2.5579724845846235, 10.433815404888879, -2.3679251022685204, 0.524948541321073, 1.1241088310450404, 0.4272876194431874, -0.17202221070155493},
    {-9.91568850695171, -0.9689944594115154, 3.0438037242978453, -24.495224566215796, 20.176138334709044, 15.98066361424651, -6.789040303419874, -6.710236069923372},
    {11.419903575922262, 2.8879645146136994, 72.92137995996029, 80.12511834622643, -52.072871366152654, -59.78993625266729, -0.15582684282751913, 4.883087185713722}};

template <class T>
void rodas_one(const SystemDesc& s, const Sens& sens, const Layout& L, const Controls& c,
               const Ensemble& e, int i) {
  const int n = s.n;
  const int ns = e.n_system;
  const int n_error = sens.n_sens == 0 ? n : (sens.error_control ? ns : n);
  const double EXPONENT = -1.0 / 6.0;
  const double e1 = EXPONENT * (c.icoeff + c.pcoeff + c.dcoeff);
  const double e2 = -EXPONENT * (c.pcoeff + 2.0 * c.dcoeff);
  const double e3 = EXPONENT * c.dcoeff;
  const double* prow = e.params + (size_t)i * e.np;
  const int np1 = e.np > 0 ? e.np : 1;
  std::vector<T> lu(L.lu_size), rhs(n), k(8 * (size_t)ns);
  std::vector<int> ipiv(n);
  std::vector<double> y(ns), u(ns), work(ns), dT(ns), col(n), seed(n), tmpp(np1), zero_p(np1, 0.0),
      kstate(n), coupling(n);
  double* hist = e.hist + (size_t)i * e.S * ns;
  for (int j = 0; j < ns; ++j) {
    y[j] = e.y0[(size_t)i * ns + j];
    hist[j] = y[j];
  }
  const double* times = e.times;
  const double tf = times[e.S - 1];
  const double dt_init = c.dt0 > 0.0 ? c.dt0 : (tf - times[0]) * 1e-6;
  double t = times[0], dt = dt_init, err_prev = 1.0, err_prev2 = 1.0;
  int save_idx = 1, n_steps = 0, acc = 0, rej = 0;
  const double tf_local = c.tf_index >= 0 ? prow[c.tf_index] : tf;
  auto w = [&](int j) { return e.weights ? e.weights[(size_t)i * ns + j] : (j < n ? 1.0 : (sens.error_control ? 1.0 : 0.0)); };
  auto sens_pdir = [&](int kk) {
    std::fill(tmpp.begin(), tmpp.end(), 0.0);
    if (kk >= sens.n_y0_dirs) tmpp[sens.param_cols[kk - sens.n_y0_dirs]] = 1.0;
  };

  while (save_idx < e.S && t < tf_local && n_steps < c.max_steps) {
    double h = dt;
    if (h > tf_local - t) h = tf_local - t;
    if (h < 1e-30) h = 1e-30;
    const double inv_dt = 1.0 / h;
    const double t_end = t + h;
    const double dtgamma_inv = 1.0 / (h * GAMMA);
    // -J by colour sweeps into the slots, df/dt into dT (modax/rodas5P.py:251-303).
    if (L.store) {
      int claimed = 0;
      for (int q = 0; q < n * L.n_colours; ++q) claimed += L.store[q] >= 0;
      if (L.lu_size > claimed) std::fill(lu.begin(), lu.end(), T(0));
    }
    for (int g = 0; g < L.n_colours; ++g) {
      for (int cc = 0; cc < n; ++cc) seed[cc] = L.colour[cc] == g ? 1.0 : 0.0;
      jvp(s, y.data(), t, prow, seed.data(), 0.0, zero_p.data(), col.data());
      for (int row = 0; row < n; ++row) {
        int slot = L.store ? L.store[row * L.n_colours + g] : row * L.n_colours + g;
        if (slot >= 0) lu[slot] = (T)(-col[row]);
      }
    }
    jvp(s, y.data(), t, prow, nullptr, 1.0, zero_p.data(), col.data());
    for (int row = 0; row < n; ++row) dT[row] = col[row];
    for (int kk = 0; kk < sens.n_sens; ++kk) {
      const int base = n + kk * n;
      sens_pdir(kk);
      jvp2(s, y.data(), t, prow, y.data() + base, 0.0, tmpp.data(), nullptr, 1.0, zero_p.data(), col.data());
      for (int row = 0; row < n; ++row) dT[base + row] = col[row];
    }
    for (int d = 0; d < n; ++d) lu[L.diag[d]] += (T)dtgamma_inv;
    if (L.sparse) sparse_factorize<T>(lu.data(), L, n);
    else dense_factorize<T>(lu.data(), ipiv.data(), n);

    auto solve = [&](T* r) {
      if (L.sparse) sparse_solve<T>(lu.data(), L, r, n);
      else dense_solve<T>(lu.data(), ipiv.data(), r, n);
    };
    auto K = [&](int st, int j) -> T& { return k[(size_t)st * ns + j]; };
    auto stage = [&](int st) {
      for (int j = 0; j < ns; ++j) {
        double value;
        if (st == 0) {
          value = work[j] + h * RD[0] * dT[j];
        } else {
          double a = RC[st][0] * (double)K(0, j);
          for (int m = 1; m < st; ++m) a += RC[st][m] * (double)K(m, j);
          if (RD[st] != 0.0) value = work[j] + h * RD[st] * dT[j] + a * inv_dt;
          else value = work[j] + a * inv_dt;
        }
        if (j < n) rhs[j] = (T)value;
        else work[j] = value;
      }
      solve(rhs.data());
      for (int j = 0; j < n; ++j) K(st, j) = rhs[j];
      if (sens.n_sens) {
        for (int j = 0; j < n; ++j) kstate[j] = (double)K(st, j);
        for (int kk = 0; kk < sens.n_sens; ++kk) {
          const int base = n + kk * n;
          sens_pdir(kk);
          jvp2(s, y.data(), t, prow, y.data() + base, 0.0, tmpp.data(), kstate.data(), 0.0, zero_p.data(), coupling.data());
          for (int j = 0; j < n; ++j) rhs[j] = (T)(work[base + j] + coupling[j]);
          solve(rhs.data());
          for (int j = 0; j < n; ++j) K(st, base + j) = rhs[j];
        }
      }
    };
    auto advance = [&](int st) {
      for (int j = 0; j < ns; ++j) {
        double a = RA[st][0] * (double)K(0, j);
        for (int m = 1; m <= st; ++m) a += RA[st][m] * (double)K(m, j);
        u[j] = y[j] + a;
      }
    };
    f_system(s, sens, y.data(), t, prow, work.data(), tmpp);
    stage(0);
    advance(0);
    f_system(s, sens, u.data(), t + RCT[0] * h, prow, work.data(), tmpp);
    stage(1);
    advance(1);
    f_system(s, sens, u.data(), t + RCT[1] * h, prow, work.data(), tmpp);
    stage(2);
    advance(2);
    f_system(s, sens, u.data(), t + RCT[2] * h, prow, work.data(), tmpp);
    stage(3);
    advance(3);
    f_system(s, sens, u.data(), t + RCT[3] * h, prow, work.data(), tmpp);
    stage(4);
    advance(4);
    f_system(s, sens, u.data(), t_end, prow, work.data(), tmpp);
    stage(5);
    for (int j = 0; j < ns; ++j) u[j] += (double)K(5, j);
    f_system(s, sens, u.data(), t_end, prow, work.data(), tmpp);
    stage(6);
    for (int j = 0; j < ns; ++j) u[j] += (double)K(6, j);
    f_system(s, sens, u.data(), t_end, prow, work.data(), tmpp);
    stage(7);

    double err_local = 0.0;
    for (int j = 0; j < ns; ++j) {
      double y_new = u[j] + (double)K(7, j);
      double scale = c.atol + c.rtol * pymax(std::fabs(y[j]), std::fabs(y_new));
      double r = w(j) * (double)K(7, j) / scale;
      err_local += r * r;
    }
    double err = std::sqrt(err_local / n_error);
    bool accept = err <= 1.0 && !std::isnan(err);
    double safe;
    if (std::isnan(err) || err > 1e18) safe = 1e18;
    else if (err == 0.0) safe = 1e-18;
    else safe = err;
    double factor = 0.9 * std::pow(safe, e1) * std::pow(err_prev, e2) * std::pow(err_prev2, e3);
    if (accept) { err_prev2 = err_prev; err_prev = safe; }
    if (factor < 0.2) factor = 0.2;
    else if (factor > 6.0) factor = 6.0;
    dt = h * factor;
    if (accept) {
      const double t_old = t;
      const double t_new = t_old + h;
      while (save_idx < e.S && times[save_idx] <= t_new + 1e-12 * pymax(1.0, std::fabs(times[save_idx]))) {
        const double th = (times[save_idx] - t_old) / h;
        const double th1 = 1.0 - th;
        for (int j = 0; j < ns; ++j) {
          double h1 = RH[0][0] * (double)K(0, j), h2 = RH[1][0] * (double)K(0, j), h3 = RH[2][0] * (double)K(0, j);
          for (int m = 1; m < 8; ++m) {
            h1 += RH[0][m] * (double)K(m, j);
            h2 += RH[1][m] * (double)K(m, j);
            h3 += RH[2][m] * (double)K(m, j);
          }
          double y_new = u[j] + (double)K(7, j);
          hist[(size_t)save_idx * ns + j] = th1 * y[j] + th * (y_new + th1 * (h1 + th * (h2 + th * h3)));
        }
        ++save_idx;
      }
      for (int j = 0; j < ns; ++j) y[j] = u[j] + (double)K(7, j);
      t += h;
      ++acc;
    } else {
      ++rej;
    }
    ++n_steps;
  }
  while (save_idx < e.S) {
    for (int j = 0; j < ns; ++j) hist[(size_t)save_idx * ns + j] = y[j];
    ++save_idx;
  }
  e.accepted[i] = acc;
  e.rejected[i] = rej;
  e.loop[i] = n_steps;
}

void set_threads(int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}

}  // namespace

extern "C" {

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_tsit5(const SystemDesc* s, const Sens* sens, const Controls* c, const Ensemble* e, int threads) {
  set_threads(threads);
  const bool serial = s->kind == SYS_CALLBACK;
#pragma omp parallel for schedule(dynamic, 16) if (!serial)
  for (int i = 0; i < e->N; ++i) tsit5_one(*s, *sens, *c, *e, i);
  return 0;
}

int oracle_rodas5p(const SystemDesc* s, const Sens* sens, const Layout* L, const Controls* c,
                   const Ensemble* e, int lu_fp32, int threads) {
  set_threads(threads);
  const bool serial = s->kind == SYS_CALLBACK;
  if (lu_fp32) {
#pragma omp parallel for schedule(dynamic, 16) if (!serial)
    for (int i = 0; i < e->N; ++i) rodas_one<float>(*s, *sens, *L, *c, *e, i);
  } else {
#pragma omp parallel for schedule(dynamic, 16) if (!serial)
    for (int i = 0; i < e->N; ++i) rodas_one<double>(*s, *sens, *L, *c, *e, i);
  }
  return 0;
}

// The right-hand side and its directional derivatives, for checking the
// product's traced derivatives against independent dual-number ones.
int oracle_eval(const SystemDesc* s, const double* y, double t, const double* p, double* out) {
  f(*s, y, t, p, out);
  return 0;
}
int oracle_jvp(const SystemDesc* s, const double* y, double t, const double* p, const double* vy,
               double vt, const double* vp, double* out) {
  jvp(*s, y, t, p, vy, vt, vp, out);
  return 0;
}

int oracle_jvp2(const SystemDesc* s, const double* y, double t, const double* p, const double* uy,
                double ut, const double* up, const double* vy, double vt, const double* vp,
                double* out) {
  jvp2(*s, y, t, p, uy, ut, up, vy, vt, vp, out);
  return 0;
}

}  // extern "C"
