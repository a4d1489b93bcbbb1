// Forward-mode dual numbers and the metric/camera written once for any scalar type, for the
// derivatives the adjoint needs: the (r, theta, a) derivatives of the 15 inverse-metric terms
// inside the right-hand side's vector-Jacobian product, and the (alpha, beta, a, theta_o)
// derivatives of a camera ray's initial state.
//
// The closed forms are those of geometry/metric.py (inverse metric and its r/theta
// derivatives, :166-313; covariant metric, :147-163) and raytracing/camera.py (:225-381).
#pragma once

#include <cuda_runtime.h>

namespace krr {

template <int N>
struct Dual {
  double v;
  double d[N];
  __device__ Dual() : v(0.0) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  __device__ Dual(double x) : v(x) {  // NOLINT: a constant
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  __device__ static Dual var(double x, int k) {
    Dual r(x);
    r.d[k] = 1.0;
    return r;
  }
};

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = fma(a.d[i], b.v, a.v * b.d[i]);
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double s, const Dual<N>& a) {
  Dual<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double s, const Dual<N>& a) {
  Dual<N> r = a;
  r.v = s + a.v;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double s, const Dual<N>& a) {
  return s + (-a);
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v = a.v - s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double s) {
  return s + a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double s) {
  return s * a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double s) {
  return (1.0 / s) * a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double s, const Dual<N>& b) {
  return Dual<N>(s) / b;
}
template <int N>
__device__ __forceinline__ void dsincos(const Dual<N>& a, Dual<N>& s, Dual<N>& c) {
  double sv, cv;
  sincos(a.v, &sv, &cv);
  s.v = sv;
  c.v = cv;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    s.d[i] = cv * a.d[i];
    c.d[i] = -sv * a.d[i];
  }
}
template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = sqrt(a.v);
  const double h = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = h * a.d[i];
  return r;
}
__device__ __forceinline__ void dsincos(double a, double& s, double& c) { sincos(a, &s, &c); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dval(double a) { return a; }
template <int N>
__device__ __forceinline__ double dval(const Dual<N>& a) { return a.v; }

// The 15 inverse-metric terms (g^tt, g^tph, g^rr, g^thth, g^phph, then d_r and d_theta of the five)
// at (r, theta) for spin parameter a and mass m, in any scalar type.
template <class T>
__device__ __forceinline__ void metric_terms(T r, T th, T a, double m, T g[15]) {
  T s, c;
  dsincos(th, s, c);
  const T a2 = a * a;
  const T s2 = s * s;
  const T sin2th = 2.0 * (s * c);
  const T r2 = r * r;
  const T sig = r2 + a2 * (c * c);
  const T dlt = r2 - (2.0 * m) * r + a2;
  const T r2a2 = r2 + a2;
  const T big_a = r2a2 * r2a2 - a2 * dlt * s2;
  const T sd = sig * dlt;
  const T two_ma = (2.0 * m) * a;
  g[0] = -big_a / sd;
  g[1] = -(two_ma * r) / sd;
  g[2] = dlt / sig;
  g[3] = 1.0 / sig;
  g[4] = (dlt - a2 * s2) / (sd * s2);
  const T sig_r = 2.0 * r;
  const T sig_th = -(a2 * sin2th);
  const T dlt_r = 2.0 * (r - m);
  const T a_r = (4.0 * r) * r2a2 - (2.0 * a2) * (r - m) * s2;
  const T a_th = -(a2 * dlt * sin2th);
  const T sd_r = sig_r * dlt + sig * dlt_r;
  const T sd_th = sig_th * dlt;
  const T sd2 = sd * sd;
  const T sig2 = sig * sig;
  g[5] = -(a_r * sd - big_a * sd_r) / sd2;
  g[6] = -(two_ma * (sd - r * sd_r)) / sd2;
  g[7] = (dlt_r * sig - dlt * sig_r) / sig2;
  g[8] = -sig_r / sig2;
  g[9] = -sig_r / (sig2 * s2) + a2 * sd_r / sd2;
  g[10] = -(a_th * sd - big_a * sd_th) / sd2;
  g[11] = two_ma * r * sd_th / sd2;
  g[12] = -(dlt * sig_th) / sig2;
  g[13] = -sig_th / sig2;
  g[14] = -(sig_th * s2 + sig * sin2th) / (sig2 * (s2 * s2)) + a2 * sd_th / sd2;
}

// Backward null state of image point (alpha, beta) for an observer at (r_o, theta_o, phi_o) in
// spacetime (m, a), in any scalar type (the camera of camera.py:298-381 with its frame).
template <class T>
__device__ __forceinline__ void camera_state_t(T alpha, T beta, T a, T th_o, double r_o, double ph_o, double m,
                                               T y0[8]) {
  T s, c;
  dsincos(th_o, s, c);
  const T s2 = s * s;
  const T a2 = a * a;
  const T rr = T(r_o);
  const T sig = rr * rr + a2 * (c * c);
  const T dlt = rr * rr - (2.0 * m) * rr + a2;
  const T g_tt = -(1.0 - (2.0 * m) * rr / sig);
  const T g_tphi = -((2.0 * m) * a * rr * s2) / sig;
  const T g_rr = sig / dlt;
  const T g_thth = sig;
  const T g_phph = (rr * rr + a2 + (2.0 * m) * a2 * rr * s2 / sig) * s2;
  const T omega = -g_tphi / g_phph;
  const T lapse = dsqrt(-(g_tt - g_tphi * g_tphi / g_phph));
  const T e00 = 1.0 / lapse, e03 = omega / lapse;
  const T e11 = 1.0 / dsqrt(g_rr), e22 = 1.0 / dsqrt(g_thth), e33 = 1.0 / dsqrt(g_phph);
  const T r2a2 = rr * rr + a2;
  const T big_a = r2a2 * r2a2 - a2 * dlt * s2;
  const T sd = sig * dlt;
  const T gi_tt = -big_a / sd, gi_tphi = -((2.0 * m) * a * rr) / sd, gi_rr = dlt / sig, gi_thth = 1.0 / sig;
  const T gi_phph = (dlt - a2 * s2) / (sd * s2);
  const T rho2 = (alpha * alpha + beta * beta) / (r_o * r_o);
  const T p1 = dsqrt(1.0 - rho2), p2 = beta / r_o, p3 = -alpha / r_o;
  const T u0 = e00, u1 = p1 * e11, u2 = p2 * e22, u3 = e03 + p3 * e33;
  T pt = -(u0 * g_tt + u3 * g_tphi);
  const T pr = -(u1 * g_rr), pth = -(u2 * g_thth);
  const T pph = -(u0 * g_tphi + u3 * g_phph);
  // Re-solve p_t from the null quadratic, the root nearest the projected value.
  const T qb = 2.0 * gi_tphi * pph;
  const T qc = gi_rr * pr * pr + gi_thth * pth * pth + gi_phph * pph * pph;
  T disc = qb * qb - 4.0 * gi_tt * qc;
  if (dval(disc) < 0.0) disc = T(0.0);
  const T sq = dsqrt(disc);
  const T q = (dval(qb) >= 0.0) ? -0.5 * (qb + sq) : -0.5 * (qb - sq);
  const T root1 = q / gi_tt;
  const T root2 = (dval(q) != 0.0) ? qc / q : root1;
  pt = (fabs(dval(root1) - dval(pt)) <= fabs(dval(root2) - dval(pt))) ? root1 : root2;
  y0[0] = T(0.0);
  y0[1] = rr;
  y0[2] = th_o;
  y0[3] = T(ph_o);
  y0[4] = pt;
  y0[5] = pr;
  y0[6] = pth;
  y0[7] = pph;
}

}  // namespace krr
