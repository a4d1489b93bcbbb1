// Analytic capture/escape of a photon from its constants of motion, with a margin that says
// how far the photon is from the critical (photon-orbit) boundary.
//
// A Kerr null geodesic with E = -p_t, L = p_phi and Carter constant Q moves radially in the
// potential (Carter 1968, Phys. Rev. 174, 1559; Bardeen 1973)
//
//   R(r) / E^2 = (r^2 + a^2 - a lam)^2 - Delta (eta + (lam - a)^2)
//              = r^4 + (a^2 - lam^2 - eta) r^2 + 2 M (eta + (lam - a)^2) r - a^2 eta,
//
// lam = L / E, eta = Q / E^2, with (dr/dlambda)^2 Sigma^2 = R.  A photon moving inward from r0
// turns around (and escapes) exactly when R has a root between the capture radius and r0, i.e.
// when the minimum of R over [r_capture, r0] is negative; otherwise it reaches the capture
// radius.  The minimum sits at r_capture or at a local minimum of R, a root of the depressed
// cubic R'(r) = 4 r^3 + 2 c2 r + c1.
//
// The numerical integration classifies a photon the same way unless its error moves the photon
// across the boundary.  A displacement db of the image point moves (lam, eta) by at most about
// (db, 2 b db) (b the impact parameter), so |R_min| / (|dR/dlam| + 2 b |dR/deta|) is a
// first-order distance to the boundary in the image plane.  Photons closer than a band
// tau_b (of the order of 1e-3 M at rtol 1e-6, a hundred times the integration's error in b)
// are "critical": the mixed-precision pipeline traces them in reference-order FP64 from the
// start; the rest are checked against their analytic class afterwards.
#pragma once

#include <cmath>

#include "krr_device.cuh"

namespace krr {

// RISK_NEAR: an escaping photon within the near-edge band (near_band) of the boundary; its
// terminal state, not its class, needs FP64 (the mixed pipeline traces it in fast FP64).
enum : int { RISK_ESCAPE = 0, RISK_CAPTURE = 1, RISK_CRITICAL = 2, RISK_RECHECK = 3, RISK_NEAR = 4 };

#if defined(__CUDACC__)
#define KRR_HD __host__ __device__
#else
#define KRR_HD
#endif

// R(r) / E^2 = r^4 + c2 r^2 + c1 r + c0.
struct RadialPoly {
  double c2, c1, c0;
};

KRR_HD inline double radial_value(const RadialPoly& R, double r) {
  const double r2 = r * r;
  return fma(r2, r2 + R.c2, fma(R.c1, r, R.c0));
}
KRR_HD inline double radial_d1(const RadialPoly& R, double r) { return fma(4.0 * r * r, r, fma(2.0 * R.c2, r, R.c1)); }
KRR_HD inline double radial_d2(const RadialPoly& R, double r) { return fma(12.0 * r, r, 2.0 * R.c2); }

// Local minima of R: the largest real root of R' = 4 (t^3 + p t + q), p = c2 / 2, q = c1 / 4,
// and, when the cubic has three real roots, the smallest (the middle one is a maximum).
// Three roots: t_k = m cos(phi - 2 pi k / 3), m = 2 sqrt(-p / 3), cos(3 phi) = 3 q / (p m)
// (Viete); one root: Cardano.  Each root is polished by two Newton steps on R'.
KRR_HD inline int radial_minima(const RadialPoly& R, double out[2]) {
  const double p = 0.5 * R.c2, q = 0.25 * R.c1;
  int n = 1;
  if (p < 0.0 && 4.0 * p * p * p + 27.0 * q * q < 0.0) {
    const double m = 2.0 * sqrt(-p / 3.0);
    const double c3 = fmin(1.0, fmax(-1.0, 3.0 * q / (p * m)));
    const double phi = acos(c3) / 3.0;
    out[0] = m * cos(phi);
    out[1] = m * cos(phi + 2.0 * PI / 3.0);
    n = 2;
  } else {
    const double sq = sqrt(fmax(0.25 * q * q + p * p * p / 27.0, 0.0));
    out[0] = cbrt(-0.5 * q + sq) + cbrt(-0.5 * q - sq);
  }
  for (int k = 0; k < n; ++k) {
    for (int it = 0; it < 2; ++it) {
      const double d2 = radial_d2(R, out[k]);
      if (d2 > 0.0) out[k] -= radial_d1(R, out[k]) / d2;
    }
  }
  return n;
}

// RISK_ESCAPE / RISK_CAPTURE for a photon whose analytic class holds with a margin of tau_b
// (M) in the image plane, RISK_CRITICAL otherwise.  Only photons moving inward (p_r < 0) from
// outside the capture radius, with |L| not negligible against their impact parameter (an
// axis-crossing ray ends OUT_OF_DOMAIN), are classified; anything else, and any non-finite
// intermediate, is critical.
// With tau_near > tau_b, an escaping photon within tau_near of the boundary is RISK_NEAR.
KRR_HD inline int radial_risk(double mass, double a, double r_capture, const double y0[8], double tau_b,
                              double tau_near = 0.0) {
  const double r0 = y0[1], th = y0[2], pt = y0[4], pr = y0[5], pth = y0[6], pph = y0[7];
  if (!(pr < 0.0) || !(r0 > r_capture)) return RISK_CRITICAL;
  const double e = -pt;
  if (!(e != 0.0)) return RISK_CRITICAL;
  const double s = sin(th), c = cos(th);
  const double lz2_over_s2 = (pph != 0.0) ? (pph * pph) / (s * s) : 0.0;
  const double q = pth * pth + (c * c) * (lz2_over_s2 - a * a * e * e);
  const double lam = pph / e;
  const double eta = q / (e * e);
  const double a2 = a * a;
  const double b = sqrt(fmax(eta + lam * lam, 0.0));
  if (!(fabs(lam) > 1e-6 * b)) return RISK_CRITICAL;
  RadialPoly R;
  R.c2 = a2 - lam * lam - eta;
  R.c1 = 2.0 * mass * (eta + (lam - a) * (lam - a));
  R.c0 = -a2 * eta;
  double rm = r_capture;
  double vmin = radial_value(R, r_capture);
  double mins[2];
  const int n = radial_minima(R, mins);
  for (int k = 0; k < n; ++k) {
    if (mins[k] > r_capture && mins[k] < r0) {
      const double v = radial_value(R, mins[k]);
      if (v < vmin) {
        vmin = v;
        rm = mins[k];
      }
    }
  }
  const double dlt = fma(rm, rm - 2.0 * mass, a2);
  const double dr_deta = -dlt;
  const double dr_dlam = -2.0 * a * (rm * rm + a2 - a * lam) - 2.0 * dlt * (lam - a);
  const double sens = fabs(dr_dlam) + 2.0 * b * fabs(dr_deta);
  if (!(fabs(vmin) > tau_b * sens)) return RISK_CRITICAL;
  if (vmin < 0.0 && !(fabs(vmin) > tau_near * sens)) return RISK_NEAR;
  return vmin < 0.0 ? RISK_ESCAPE : RISK_CAPTURE;
}

// The band of the mixed pipeline (M): a hundred times the integration's error in the impact
// parameter at rtol 1e-6 and above, scaled with rtol beyond.
KRR_HD inline double risk_band(double mass, double rtol) { return mass * fmax(2e-3, 2e3 * rtol); }

// The near-edge band of the mixed pipeline (M): escaping photons this close to the boundary
// pass near the unstable photon orbit, where -dH/dr is a small difference of large terms and
// the orbit magnifies the FP32 stages' round-off in the exit direction beyond 10 rtol (at
// rtol 1e-6 on an a* = 0.99, i = 85 deg image, within 0.3 M but one ray, which lay at 0.34 M;
// with 0.35 M none of the 1024^2 or 2048^2 image's escaped rays is beyond the oracle's bar).
KRR_HD inline double near_band(double mass) { return 0.35 * mass; }

}  // namespace krr
