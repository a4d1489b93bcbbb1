// TEST INFRASTRUCTURE ONLY — the oracle (checker) of the per-ray hot path.
//
// A CPU restatement, operation by operation and in the same floating-point
// order, of KerrRay's scalar ray kernel (src/kerrray/raytracing/backends/
// numba_kernel.py:111-463) and of its host-side constant packing
// (src/kerrray/raytracing/backends/numba_backend.py:87-128).  It is compiled
// without floating-point contraction (-ffp-contract=off) so that, like the
// Numba kernel (fastmath=False, numba_kernel.py:466), every product and sum
// is rounded separately; sin, cos, pow and sqrt come from the C library as in
// the Numba build.  Only the tests, the smoke check and the CPU-baseline leg of
// the benchmark load this file's library; the product path never does.
//
// The scalar type is a template parameter so that the same source also runs
// with a counting type (krr_oracle_count_flops) that pins the algorithmic
// floating-point work per step attempt used by the roofline figures.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum : int { RUNNING = 0, ESCAPED = 1, CAPTURED = 2, MAX_AFFINE = 3, FAILURE = 4, OUT_OF_DOMAIN = 5, DISK_HIT = 6 };
enum : int { T = 0, R = 1, TH = 2, PH = 3, PT = 4, PR = 5, PTH = 6, PPH = 7 };

// ---------------------------------------------------------------------------------------------
// Counting scalar: behaves like double and tallies every arithmetic operation by kind.
// ---------------------------------------------------------------------------------------------
struct Tally {
  int64_t add = 0, mul = 0, div = 0, sqrt_ = 0, trig = 0, pow_ = 0;
};
thread_local Tally* g_tally = nullptr;
inline void tick(int64_t Tally::*f) { if (g_tally) ++(g_tally->*f); }

struct CD {
  double v;
  CD() : v(0.0) {}
  CD(double x) : v(x) {}  // NOLINT: implicit like a double
  explicit operator double() const { return v; }
};
inline CD operator+(CD a, CD b) { tick(&Tally::add); return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { tick(&Tally::add); return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { tick(&Tally::mul); return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { tick(&Tally::div); return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
inline bool operator<(CD a, CD b) { return a.v < b.v; }
inline bool operator>(CD a, CD b) { return a.v > b.v; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { return a.v >= b.v; }
inline bool operator==(CD a, CD b) { return a.v == b.v; }
inline bool operator!=(CD a, CD b) { return a.v != b.v; }
inline CD k_sin(CD a) { tick(&Tally::trig); return CD(std::sin(a.v)); }
inline CD k_cos(CD a) { tick(&Tally::trig); return CD(std::cos(a.v)); }
inline CD k_sqrt(CD a) { tick(&Tally::sqrt_); return CD(std::sqrt(a.v)); }
inline CD k_pow(CD a, CD b) { tick(&Tally::pow_); return CD(std::pow(a.v, b.v)); }
inline CD k_abs(CD a) { return CD(std::fabs(a.v)); }
inline bool k_finite(CD a) { return std::isfinite(a.v); }

inline double k_sin(double a) { return std::sin(a); }
inline double k_cos(double a) { return std::cos(a); }
inline double k_sqrt(double a) { return std::sqrt(a); }
inline double k_pow(double a, double b) { return std::pow(a, b); }
inline double k_abs(double a) { return std::fabs(a); }
inline bool k_finite(double a) { return std::isfinite(a); }
inline float k_sin(float a) { return std::sin(a); }
inline float k_sqrt(float a) { return std::sqrt(a); }
inline float k_pow(float a, float b) { return std::pow(a, b); }
inline float k_abs(float a) { return std::fabs(a); }
inline bool k_finite(float a) { return std::isfinite(a); }

// Python's builtin max(a, b) / min(a, b) on two floats: the first argument unless the
// second compares strictly greater / smaller.
template <class X> inline X py_max(X a, X b) { return (b > a) ? b : a; }
template <class X> inline X py_min(X a, X b) { return (b < a) ? b : a; }

// The float64 type paired with a working type (the metric and the diagnostics are float64
// in the reference even in float32 mode, numba_kernel.py:165-167, 315-336).
template <class W> struct Wide { using type = double; };
template <> struct Wide<CD> { using type = CD; };

template <class X> inline double as_d(X x) { return static_cast<double>(x); }
inline double as_d(CD x) { return x.v; }

// ---------------------------------------------------------------------------------------------
// Constants (numba_backend.py:87-128).
// ---------------------------------------------------------------------------------------------
template <class D>
struct Geom {  // G_LAYOUT, numba_kernel.py:90-91
  D mass, a, a2, neg_2ma, pos_2ma, two_m, two_a2;
};

template <class W>
struct Consts {  // C_LAYOUT, numba_kernel.py:94-102, in the working dtype
  W zero, one, two, neg_half, eight, safety, fmin, fmax, exponent, rtol, atol, h_min, r_capture, r_escape,
      theta_low, theta_high, axis_sin_tol, h_initial, r_in, r_out, half_pi;
};

template <class W>
struct Tab {  // dense DP_A (7x7), DP_E (7), RK4_B, RK4_C in the working dtype
  W a[7][7];
  W e[7];
  W rk4_b[4];
  W rk4_c[4];
};

struct Run {
  double lambda_max, half_pi, h_max;
  int64_t max_steps, guard;
  bool adaptive, disk;
};

template <class W>
void make_tab(Tab<W>& t) {
  double a[7][7] = {};
  a[1][0] = 1.0 / 5.0;
  a[2][0] = 3.0 / 40.0; a[2][1] = 9.0 / 40.0;
  a[3][0] = 44.0 / 45.0; a[3][1] = -56.0 / 15.0; a[3][2] = 32.0 / 9.0;
  a[4][0] = 19372.0 / 6561.0; a[4][1] = -25360.0 / 2187.0; a[4][2] = 64448.0 / 6561.0; a[4][3] = -212.0 / 729.0;
  a[5][0] = 9017.0 / 3168.0; a[5][1] = -355.0 / 33.0; a[5][2] = 46732.0 / 5247.0; a[5][3] = 49.0 / 176.0;
  a[5][4] = -5103.0 / 18656.0;
  a[6][0] = 35.0 / 384.0; a[6][1] = 0.0; a[6][2] = 500.0 / 1113.0; a[6][3] = 125.0 / 192.0;
  a[6][4] = -2187.0 / 6784.0; a[6][5] = 11.0 / 84.0;
  const double b[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
  const double bh[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0,
                        187.0 / 2100.0, 1.0 / 40.0};
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) t.a[i][j] = W(a[i][j]);
  for (int i = 0; i < 7; ++i) t.e[i] = W(bh[i] - b[i]);  // tableaus.py:85
  const double rb[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  const double rc[4] = {0.0, 0.5, 0.5, 1.0};
  for (int i = 0; i < 4; ++i) { t.rk4_b[i] = W(rb[i]); t.rk4_c[i] = W(rc[i]); }
}

// ---------------------------------------------------------------------------------------------
// Kernel functions (numba_kernel.py).
// ---------------------------------------------------------------------------------------------
template <class D>
void inverse_metric_terms(const Geom<D>& g, D r, D th, D out[15]) {  // :111-154
  D m = g.mass;
  D a2 = g.a2;
  D s = k_sin(th);
  D c = k_cos(th);
  D s2 = s * s;
  D sin2th = k_sin(D(2.0) * th);
  D r2 = r * r;
  D sig = r2 + a2 * (c * c);
  D dlt = r2 - g.two_m * r + a2;
  D r2a2 = r2 + a2;
  D big_a = r2a2 * r2a2 - a2 * dlt * s2;
  D sd = sig * dlt;
  out[0] = -big_a / sd;
  out[1] = g.neg_2ma * r / sd;
  out[2] = dlt / sig;
  out[3] = D(1.0) / sig;
  out[4] = (dlt - a2 * s2) / (sd * s2);
  D sig_r = D(2.0) * r;
  D sig_th = (-a2) * sin2th;
  D dlt_r = D(2.0) * (r - m);
  D a_r = D(4.0) * r * r2a2 - g.two_a2 * (r - m) * s2;
  D a_th = (-a2) * dlt * sin2th;
  D sd_r = sig_r * dlt + sig * dlt_r;
  D sd_th = sig_th * dlt;
  D sd2 = sd * sd;
  D sig2 = sig * sig;
  out[5] = -(a_r * sd - big_a * sd_r) / sd2;
  out[6] = g.neg_2ma * (sd - r * sd_r) / sd2;
  out[7] = (dlt_r * sig - dlt * sig_r) / sig2;
  out[8] = -sig_r / sig2;
  out[9] = -sig_r / (sig2 * s2) + a2 * sd_r / sd2;
  out[10] = -(a_th * sd - big_a * sd_th) / sd2;
  out[11] = g.pos_2ma * r * sd_th / sd2;
  out[12] = -dlt * sig_th / sig2;
  out[13] = -sig_th / sig2;
  out[14] = -(sig_th * s2 + sig * sin2th) / (sig2 * (s2 * s2)) + a2 * sd_th / sd2;
}

template <class W>
void geodesic_rhs(const Geom<typename Wide<W>::type>& geom, const Consts<W>& k, const W* y, W* f) {  // :158-197
  using D = typename Wide<W>::type;
  D g64[15];
  inverse_metric_terms<D>(geom, D(as_d(y[R])), D(as_d(y[TH])), g64);
  W g[15];
  for (int i = 0; i < 15; ++i) g[i] = W(as_d(g64[i]));
  W zero = k.zero, two = k.two;
  W p_t = y[PT], p_r = y[PR], p_th = y[PTH], p_ph = y[PPH];
  W gphph = g[4], r_gphph = g[9], t_gphph = g[14];
  if (p_ph == zero) { gphph = zero; r_gphph = zero; t_gphph = zero; }
  f[T] = g[0] * p_t + g[1] * p_ph;
  f[R] = g[2] * p_r;
  f[TH] = g[3] * p_th;
  f[PH] = g[1] * p_t + gphph * p_ph;
  f[PT] = zero;
  W pt2 = p_t * p_t, ptpph = p_t * p_ph, pr2 = p_r * p_r, pth2 = p_th * p_th, pph2 = p_ph * p_ph;
  f[PR] = k.neg_half * (g[5] * pt2 + two * g[6] * ptpph + g[7] * pr2 + g[8] * pth2 + r_gphph * pph2);
  f[PTH] = k.neg_half * (g[10] * pt2 + two * g[11] * ptpph + g[12] * pr2 + g[13] * pth2 + t_gphph * pph2);
  f[PPH] = zero;
}

template <class W>
void dp_step(const Geom<typename Wide<W>::type>& geom, const Consts<W>& c, const Tab<W>& tb, const W* y, W h,
             W k[7][8], W* ys, W* y_new, W* err) {  // :201-238
  const auto& a = tb.a;
  const auto& e = tb.e;
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (a[1][0] * k[0][i]);
  geodesic_rhs<W>(geom, c, ys, k[1]);
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (a[2][0] * k[0][i] + a[2][1] * k[1][i]);
  geodesic_rhs<W>(geom, c, ys, k[2]);
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (a[3][0] * k[0][i] + a[3][1] * k[1][i] + a[3][2] * k[2][i]);
  geodesic_rhs<W>(geom, c, ys, k[3]);
  for (int i = 0; i < 8; ++i)
    ys[i] = y[i] + h * (a[4][0] * k[0][i] + a[4][1] * k[1][i] + a[4][2] * k[2][i] + a[4][3] * k[3][i]);
  geodesic_rhs<W>(geom, c, ys, k[4]);
  for (int i = 0; i < 8; ++i)
    ys[i] = y[i] + h * (a[5][0] * k[0][i] + a[5][1] * k[1][i] + a[5][2] * k[2][i] + a[5][3] * k[3][i] +
                        a[5][4] * k[4][i]);
  geodesic_rhs<W>(geom, c, ys, k[5]);
  for (int i = 0; i < 8; ++i)
    y_new[i] = y[i] + h * (a[6][0] * k[0][i] + a[6][2] * k[2][i] + a[6][3] * k[3][i] + a[6][4] * k[4][i] +
                           a[6][5] * k[5][i]);
  geodesic_rhs<W>(geom, c, y_new, k[6]);
  for (int i = 0; i < 8; ++i)
    err[i] = h * (e[0] * k[0][i] + e[2] * k[2][i] + e[3] * k[3][i] + e[4] * k[4][i] + e[5] * k[5][i] +
                  e[6] * k[6][i]);
}

template <class W>
void rk4_step(const Geom<typename Wide<W>::type>& geom, const Consts<W>& c, const Tab<W>& tb, const W* y, W h,
              W k[7][8], W* ys, W* y_new) {  // :242-257
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (tb.rk4_c[1] * k[0][i]);
  geodesic_rhs<W>(geom, c, ys, k[1]);
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (tb.rk4_c[2] * k[1][i]);
  geodesic_rhs<W>(geom, c, ys, k[2]);
  for (int i = 0; i < 8; ++i) ys[i] = y[i] + h * (tb.rk4_c[3] * k[2][i]);
  geodesic_rhs<W>(geom, c, ys, k[3]);
  for (int i = 0; i < 8; ++i)
    y_new[i] = y[i] + h * (tb.rk4_b[0] * k[0][i] + tb.rk4_b[1] * k[1][i] + tb.rk4_b[2] * k[2][i] +
                           tb.rk4_b[3] * k[3][i]);
  geodesic_rhs<W>(geom, c, y_new, k[6]);
}

template <class W>
W error_norm(const Consts<W>& c, const W* err, const W* y, const W* y_new) {  // :261-268
  W q[8];
  for (int i = 0; i < 8; ++i) {
    W scale = c.atol + c.rtol * py_max(k_abs(y[i]), k_abs(y_new[i]));
    W v = err[i] / scale;
    q[i] = v * v;
  }
  W total = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
  return k_sqrt(total / c.eight);
}

template <class W>
W step_factor(const Consts<W>& c, W en, bool rejected_before) {  // :272-281
  W factor;
  if (en == c.zero) {
    factor = c.fmax;
  } else {
    W raw = c.safety * k_pow(en, c.exponent);
    factor = py_min(c.fmax, py_max(c.fmin, raw));
  }
  if (rejected_before) factor = py_min(factor, c.one);
  return factor;
}

template <class W>
bool all_finite(const W* y, const W* f) {  // :285-289
  for (int i = 0; i < 8; ++i)
    if (!(k_finite(y[i]) && k_finite(f[i]))) return false;
  return true;
}

template <class W>
int classify(const Consts<W>& c, const Run& run, const W* y, const W* f, double lam, int64_t n_steps, W h,
             bool check_h) {  // :293-311
  if (!all_finite(y, f)) return FAILURE;
  if (check_h && h < c.h_min) return FAILURE;
  W r = y[R], th = y[TH];
  if (r < c.zero || th < c.theta_low || th > c.theta_high) return OUT_OF_DOMAIN;
  if (y[PPH] != c.zero && k_abs(k_sin(th)) < c.axis_sin_tol) return OUT_OF_DOMAIN;
  if (r <= c.r_capture) return CAPTURED;
  if (r >= c.r_escape && f[R] > c.zero) return ESCAPED;
  if (lam >= run.lambda_max || n_steps >= run.max_steps) return MAX_AFFINE;
  return RUNNING;
}

template <class D, class W>
D null_error(const W* y, const W* f) {  // :315-321
  D total = D(as_d(y[PT])) * D(as_d(f[T]));
  total = total + D(as_d(y[PR])) * D(as_d(f[R]));
  total = total + D(as_d(y[PTH])) * D(as_d(f[TH]));
  total = total + D(as_d(y[PPH])) * D(as_d(f[PH]));
  return k_abs(D(0.5) * total);
}

template <class D, class W>
D carter(D a2, const W* y) {  // :325-336
  D th = D(as_d(y[TH]));
  D p_th = D(as_d(y[PTH]));
  D lz = D(as_d(y[PPH]));
  D e = -D(as_d(y[PT]));
  D s = k_sin(th);
  D c = k_cos(th);
  D lz2_over_s2 = D(0.0);
  if (lz != D(0.0)) lz2_over_s2 = (lz * lz) / (s * s);
  return p_th * p_th + (c * c) * (lz2_over_s2 - a2 * e * e);
}

struct Outputs {
  double* Y;
  int64_t* state;
  int64_t* n_steps;
  int64_t* n_rejected;
  double* lam;
  double* max_null;
  double* max_e;
  double* max_lz;
  double* max_q;
  double* event_Y;
  uint8_t* event_hit;
};

struct Refs {  // per-ray conservation references computed by the caller (numba_backend.py:174-178)
  const double *e0, *lz0, *q0, *fe, *fl, *fq, *fe2;
};

// One ray, numba_kernel.py:340-463.  Phase tallies (init / attempt / accepted step) go to
// tallies[0..2] when counting.
template <class W>
void integrate_ray(int64_t n, const Geom<typename Wide<W>::type>& geom, const Consts<W>& c, const Tab<W>& tb,
                   const Run& run, const double* Y0, const Refs& refs, const Outputs& o, Tally* tallies) {
  using D = typename Wide<W>::type;
  if (tallies) g_tally = &tallies[0];
  W y[8], f[8], k[7][8], ys[8], y_new[8], y_prev[8], err[8];
  for (int i = 0; i < 8; ++i) y[i] = W(Y0[n * 8 + i]);
  D a2 = geom.a2;
  const double e0 = refs.e0[n], lz0 = refs.lz0[n], q0 = refs.q0[n];
  const double fe = refs.fe[n], fl = refs.fl[n], fq = refs.fq[n], fe2 = refs.fe2[n];
  geodesic_rhs<W>(geom, c, y, f);
  D m_null = null_error<D, W>(y, f) / D(fe2);
  D m_e = D(0.0), m_lz = D(0.0), m_q = D(0.0);
  double lam = 0.0;
  W h = c.h_initial;
  const double h_cap = run.h_max;
  if (run.adaptive && as_d(h) > h_cap) h = W(h_cap);
  int64_t n_steps = 0, n_rej = 0, attempts = 0;
  bool rejected_before = false;
  int state = classify<W>(c, run, y, f, lam, n_steps, h, false);
  while (state == RUNNING) {
    if (tallies) g_tally = &tallies[1];
    attempts += 1;
    if (attempts > run.guard) { state = FAILURE; break; }
    double remaining = run.lambda_max - lam;
    bool last = as_d(h) >= remaining;
    W h_eff = h;
    if (last) h_eff = W(remaining);
    for (int i = 0; i < 8; ++i) { k[0][i] = f[i]; y_prev[i] = y[i]; }
    if (run.adaptive)
      dp_step<W>(geom, c, tb, y, h_eff, k, ys, y_new, err);
    else
      rk4_step<W>(geom, c, tb, y, h_eff, k, ys, y_new);
    bool finite = all_finite(y_new, k[6]);
    bool accept = finite;
    W h_new = h;
    if (run.adaptive && finite) {
      W en = error_norm<W>(c, err, y, y_new);
      if (!k_finite(en)) {
        finite = false;
        accept = false;
      } else {
        accept = en <= c.one;
        W factor = step_factor<W>(c, en, rejected_before);
        if (!(accept && last)) {
          h_new = h_eff * factor;
          if (as_d(h_new) > h_cap) h_new = W(h_cap);
        }
      }
    }
    if (!finite) { state = FAILURE; break; }
    bool rejected = !accept;
    if (rejected) n_rej += 1;
    rejected_before = rejected;
    h = h_new;
    if (rejected) {
      if (h_new < c.h_min) { state = FAILURE; break; }
      continue;
    }
    if (tallies) g_tally = &tallies[2];
    for (int i = 0; i < 8; ++i) { y[i] = y_new[i]; f[i] = k[6][i]; }
    double lam_old = lam;
    lam = last ? run.lambda_max : lam + as_d(h_eff);
    n_steps += 1;
    D e = -D(as_d(y[PT]));
    D lz = D(as_d(y[PPH]));
    m_e = py_max(m_e, k_abs(e - D(e0)) / py_max(k_abs(D(e0)), D(fe)));
    m_lz = py_max(m_lz, k_abs(lz - D(lz0)) / py_max(k_abs(D(lz0)), D(fl)));
    m_q = py_max(m_q, k_abs(carter<D, W>(a2, y) - D(q0)) / py_max(k_abs(D(q0)), D(fq)));
    m_null = py_max(m_null, null_error<D, W>(y, f) / D(fe2));
    int code = classify<W>(c, run, y, f, lam, n_steps, h, true);
    if (run.disk) {  // :439-454
      double th_old = as_d(y_prev[TH]);
      double th_new = as_d(y[TH]);
      if ((th_old - run.half_pi) * (th_new - run.half_pi) < 0.0) {
        double s = (run.half_pi - th_old) / (th_new - th_old);
        for (int i = 0; i < 8; ++i) {
          W cast = W(s * as_d(y[i] - y_prev[i]));
          ys[i] = y_prev[i] + cast;
        }
        ys[TH] = W(run.half_pi);
        if (ys[R] >= c.r_in && ys[R] <= c.r_out) {
          for (int i = 0; i < 8; ++i) {
            if (o.event_Y) o.event_Y[n * 8 + i] = as_d(ys[i]);
            y[i] = ys[i];
          }
          if (o.event_hit) o.event_hit[n] = 1;
          lam = lam_old + s * as_d(h_eff);
          code = DISK_HIT;
        }
      }
    }
    state = code;
  }
  g_tally = nullptr;
  for (int i = 0; i < 8; ++i) o.Y[n * 8 + i] = as_d(y[i]);
  o.state[n] = state;
  o.n_steps[n] = n_steps;
  o.n_rejected[n] = n_rej;
  o.lam[n] = lam;
  o.max_null[n] = as_d(m_null);
  o.max_e[n] = as_d(m_e);
  o.max_lz[n] = as_d(m_lz);
  o.max_q[n] = as_d(m_q);
}

}  // namespace

// Physical and integrator parameters of one batch (IntegratorOptions, TerminationOptions,
// EventOptions of src/kerrray/geodesics/integrators.py:71-148).
struct krr_oracle_params {
  double mass, a;
  double rtol, atol, step_size, lambda_max, h_min, h_max;  // h_max = +inf for None
  int64_t max_steps, max_attempts;
  double horizon_epsilon, escape_radius;
  int32_t method;  // 0 = rk45, 1 = rk4
  int32_t dtype;   // 0 = float64, 1 = float32
  int32_t disk;
  int32_t pad;
  double r_in, r_out;
};

static void fill_geom(const krr_oracle_params* p, Geom<double>& g) {  // numba_backend.py:96-97
  const double m = p->mass, a = p->a;
  g.mass = m;
  g.a = a;
  g.a2 = a * a;
  g.neg_2ma = (-2.0 * m) * a;
  g.pos_2ma = (2.0 * m) * a;
  g.two_m = 2.0 * m;
  g.two_a2 = 2.0 * (a * a);
}

template <class W>
static void fill_consts(const krr_oracle_params* p, Consts<W>& c) {  // numba_backend.py:100-108
  const double r_plus = p->mass + std::sqrt(p->mass * p->mass - p->a * p->a);  // geometry/horizons.py:33-37
  c.zero = W(0.0); c.one = W(1.0); c.two = W(2.0); c.neg_half = W(-0.5); c.eight = W(8.0);
  c.safety = W(0.9); c.fmin = W(0.2); c.fmax = W(5.0); c.exponent = W(-1.0 / 5.0);
  c.rtol = W(p->rtol); c.atol = W(p->atol); c.h_min = W(p->h_min);
  c.r_capture = W(r_plus + p->horizon_epsilon);
  c.r_escape = W(p->escape_radius);
  c.theta_low = W(-1e-9);
  c.theta_high = W(M_PI + 1e-9);
  c.axis_sin_tol = W(1e-12);
  c.h_initial = W(p->step_size);
  c.r_in = W(p->disk ? p->r_in : 0.0);
  c.r_out = W(p->disk ? p->r_out : 0.0);
  c.half_pi = W(0.5 * M_PI);
}

static Run make_run(const krr_oracle_params* p) {
  Run run;
  run.lambda_max = p->lambda_max;
  run.half_pi = 0.5 * M_PI;
  run.h_max = p->h_max;
  run.max_steps = p->max_steps;
  run.guard = p->max_attempts;
  run.adaptive = p->method == 0;
  run.disk = p->disk != 0;
  return run;
}

template <class W>
static void run_batch(const krr_oracle_params* p, const double* Y0, int64_t n, const Refs& refs, const Outputs& o,
                      int threads) {
  Geom<double> g;
  fill_geom(p, g);
  Consts<W> c;
  fill_consts<W>(p, c);
  Tab<W> tb;
  make_tab<W>(tb);
  Run run = make_run(p);
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads)
#endif
  for (int64_t i = 0; i < n; ++i) integrate_ray<W>(i, g, c, tb, run, Y0, refs, o, nullptr);
}

extern "C" {

// Integrate n rays (numba_kernel.py:467-474).  All pointers are host arrays; e0 .. fe2 are the
// per-ray conservation references of numba_backend.py:174-178.  Returns 0, or 1 on an invalid
// argument.  threads <= 0 uses every OpenMP thread.
int krr_oracle_integrate(const krr_oracle_params* p, const double* Y0, int64_t n, const double* e0,
                         const double* lz0, const double* q0, const double* fe, const double* fl, const double* fq,
                         const double* fe2, double* Y, int64_t* state, int64_t* n_steps, int64_t* n_rejected,
                         double* lam, double* max_null, double* max_e, double* max_lz, double* max_q,
                         double* event_Y, uint8_t* event_hit, int threads) {
  if (!p || n < 0 || (n > 0 && (!Y0 || !Y || !state || !n_steps || !n_rejected || !lam))) return 1;
  Refs refs{e0, lz0, q0, fe, fl, fq, fe2};
  Outputs o{Y, state, n_steps, n_rejected, lam, max_null, max_e, max_lz, max_q, event_Y, event_hit};
  if (p->dtype == 1)
    run_batch<float>(p, Y0, n, refs, o, threads);
  else
    run_batch<double>(p, Y0, n, refs, o, threads);
  return 0;
}

// Inverse metric terms at (r, theta) (numba_kernel.py:111-154), for the metric pin test.
void krr_oracle_metric_terms(double mass, double a, double r, double th, double* out15) {
  krr_oracle_params p{};
  p.mass = mass;
  p.a = a;
  Geom<double> g;
  fill_geom(&p, g);
  inverse_metric_terms<double>(g, r, th, out15);
}

// Right-hand side of one float64 state (numba_kernel.py:158-197).
void krr_oracle_rhs(double mass, double a, const double* y8, double* f8) {
  krr_oracle_params p{};
  p.mass = mass;
  p.a = a;
  p.escape_radius = 1000.0;
  Geom<double> g;
  fill_geom(&p, g);
  Consts<double> c;
  fill_consts<double>(&p, c);
  geodesic_rhs<double>(g, c, y8, f8);
}

// Integrate n float64 rays single-threaded with the counting scalar and return the operation
// tallies by phase: counts[0..5] = init (add, mul, div, sqrt, trig, pow), counts[6..11] = all
// step attempts, counts[12..17] = the accepted-step diagnostics and classification.  The
// integer outputs (state, n_steps, n_rejected) are written like krr_oracle_integrate.
int krr_oracle_count_flops(const krr_oracle_params* p, const double* Y0, int64_t n, const double* e0,
                           const double* lz0, const double* q0, const double* fe, const double* fl,
                           const double* fq, const double* fe2, int64_t* state, int64_t* n_steps,
                           int64_t* n_rejected, int64_t* counts18) {
  if (!p || n < 0 || p->dtype != 0) return 1;
  Geom<CD> g;
  Geom<double> gd;
  fill_geom(p, gd);
  g.mass = gd.mass; g.a = gd.a; g.a2 = gd.a2; g.neg_2ma = gd.neg_2ma; g.pos_2ma = gd.pos_2ma;
  g.two_m = gd.two_m; g.two_a2 = gd.two_a2;
  Consts<double> cd;
  fill_consts<double>(p, cd);
  Consts<CD> c;
  const double* src = &cd.zero;
  CD* dst = &c.zero;
  for (size_t i = 0; i < sizeof(Consts<double>) / sizeof(double); ++i) dst[i] = CD(src[i]);
  Tab<CD> tb;
  make_tab<CD>(tb);
  Run run = make_run(p);
  Refs refs{e0, lz0, q0, fe, fl, fq, fe2};
  std::vector<double> yb(static_cast<size_t>(n) * 8), lam(n), m0(n), m1(n), m2(n), m3(n);
  Outputs o{yb.data(), state, n_steps, n_rejected, lam.data(), m0.data(), m1.data(), m2.data(), m3.data(),
            nullptr, nullptr};
  Tally tallies[3];
  for (int64_t i = 0; i < n; ++i) integrate_ray<CD>(i, g, c, tb, run, Y0, refs, o, tallies);
  for (int ph = 0; ph < 3; ++ph) {
    counts18[ph * 6 + 0] = tallies[ph].add;
    counts18[ph * 6 + 1] = tallies[ph].mul;
    counts18[ph * 6 + 2] = tallies[ph].div;
    counts18[ph * 6 + 3] = tallies[ph].sqrt_;
    counts18[ph * 6 + 4] = tallies[ph].trig;
    counts18[ph * 6 + 5] = tallies[ph].pow_;
  }
  return 0;
}

}  // extern "C"
