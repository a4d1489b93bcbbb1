// Camera ray initialisation at a finite observer distance, per pixel on the device.
//
// Follows src/kerrray/raytracing/camera.py:206-381: pixel centres alpha_j = fov(2j+1-n)/n,
// beta_i = -fov(2i+1-n)/n (row-major, row 0 on top); local momentum p^(a) = (1, sqrt(1-rho^2),
// beta/r_o, -alpha/r_o) in the ZAMO frame; p^mu = p^(a) e_(a)^mu; p_mu = g_mu_nu p^nu; null
// check to 1e-10; reversal for backward tracing; p_t re-solved from the null quadratic with
// the cancellation-free root nearest the projected value.  The per-image frame constants (the
// five non-zero tetrad entries and the covariant and contravariant metric at the observer)
// are evaluated once on the host; each pixel costs ~40 FP64 operations and two square roots.
// Every operation uses an explicitly rounded intrinsic so that no translation unit contracts
// it into an FMA: the states are identical whichever kernel builds them.
#pragma once

#include "krr_device.cuh"

namespace krr {

struct Frame {
  double r_o, th_o, ph_o;
  double e00, e03, e11, e22, e33;                    // rows e_(a)^mu of the ZAMO tetrad
  double g_tt, g_tphi, g_rr, g_thth, g_phph;         // g_mu_nu at the observer
  double gi_tt, gi_tphi, gi_rr, gi_thth, gi_phph;    // g^mu_nu at the observer
};

// One image of a batched launch: its physics and integrator parameters, its observer frame,
// its pixel grid and its range of global photon indices.
struct Image {
  Params P;
  Frame F;
  double fov;
  long long res;     // pixels per side
  long long offset;  // first global photon index of this image
  long long count;   // photons: its pixels first .. first + count - 1 (row-major)
  long long first;   // pixel of the image's first photon (0 unless the image is a pixel range)
};

// (alpha, beta) of pixel p of an n x n image with half-width fov (camera.py:219-222).
__device__ __forceinline__ void pixel_alpha_beta(double fov, long long n, long long p, double& alpha,
                                                 double& beta) {
  const long long i = p / n, j = p - (p / n) * n;
  const double nd = (double)n;
  alpha = __ddiv_rn(__dmul_rn(fov, __dsub_rn(__dadd_rn(__dmul_rn(2.0, (double)j), 1.0), nd)), nd);
  beta = -__ddiv_rn(__dmul_rn(fov, __dsub_rn(__dadd_rn(__dmul_rn(2.0, (double)i), 1.0), nd)), nd);
}

// Backward null state for image-plane point (alpha, beta).  Returns 0, or 1 when the tetrad
// projection is not null to 1e-10 or no null momentum exists (the reference raises then).
__device__ __forceinline__ int camera_state(const Frame& F, double alpha, double beta, double y0[8]) {
  const double r_o = F.r_o;
  const double rho2 = __ddiv_rn(__dadd_rn(__dmul_rn(alpha, alpha), __dmul_rn(beta, beta)), __dmul_rn(r_o, r_o));
  const double p1 = __dsqrt_rn(__dsub_rn(1.0, rho2));
  const double p2 = __ddiv_rn(beta, r_o);
  const double p3 = __ddiv_rn(-alpha, r_o);
  // p^mu = sum_a p^(a) e_(a)^mu with p^(t) = 1.
  const double u0 = F.e00;
  const double u1 = __dmul_rn(p1, F.e11);
  const double u2 = __dmul_rn(p2, F.e22);
  const double u3 = __dadd_rn(F.e03, __dmul_rn(p3, F.e33));
  // p_mu = g_mu_nu p^nu
  double pt = __dadd_rn(__dmul_rn(u0, F.g_tt), __dmul_rn(u3, F.g_tphi));
  double pr = __dmul_rn(u1, F.g_rr);
  double pth = __dmul_rn(u2, F.g_thth);
  double pph = __dadd_rn(__dmul_rn(u0, F.g_tphi), __dmul_rn(u3, F.g_phph));
  int err = 0;
  const double residual = __dadd_rn(
      __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(F.gi_tt, __dmul_rn(pt, pt)),
                                    __dmul_rn(__dmul_rn(__dmul_rn(2.0, F.gi_tphi), pt), pph)),
                          __dmul_rn(F.gi_rr, __dmul_rn(pr, pr))),
                __dmul_rn(F.gi_thth, __dmul_rn(pth, pth))),
      __dmul_rn(F.gi_phph, __dmul_rn(pph, pph)));
  if (!(fabs(residual) < 1e-10)) err = 1;
  pt = -pt;
  pr = -pr;
  pth = -pth;
  pph = -pph;
  // _null_pt (camera.py:265-295)
  const double qa = F.gi_tt;
  const double qb = __dmul_rn(__dmul_rn(2.0, F.gi_tphi), pph);
  const double qc = __dadd_rn(__dadd_rn(__dmul_rn(F.gi_rr, __dmul_rn(pr, pr)), __dmul_rn(F.gi_thth, __dmul_rn(pth, pth))),
                              __dmul_rn(F.gi_phph, __dmul_rn(pph, pph)));
  if (!(qa < 0.0)) err = 1;
  const double four_ac = __dmul_rn(__dmul_rn(4.0, qa), qc);
  const double disc = __dsub_rn(__dmul_rn(qb, qb), four_ac);
  if (disc < -1e-10 * __dadd_rn(__dmul_rn(qb, qb), fabs(four_ac))) err = 1;
  const double sq = __dsqrt_rn(disc > 0.0 ? disc : 0.0);
  const double q = __dmul_rn(-0.5, __dadd_rn(qb, copysign(sq, qb)));
  const double root1 = __ddiv_rn(q, qa);
  const double root2 = (q != 0.0) ? __ddiv_rn(qc, q) : root1;
  pt = (fabs(__dsub_rn(root1, pt)) <= fabs(__dsub_rn(root2, pt))) ? root1 : root2;
  y0[0] = 0.0;
  y0[1] = r_o;
  y0[2] = F.th_o;
  y0[3] = F.ph_o;
  y0[4] = pt;
  y0[5] = pr;
  y0[6] = pth;
  y0[7] = pph;
  return err;
}

__device__ __forceinline__ int camera_pixel_state(const Image& im, long long p, double y0[8]) {
  double alpha, beta;
  pixel_alpha_beta(im.fov, im.res, p, alpha, beta);
  return camera_state(im.F, alpha, beta, y0);
}

}  // namespace krr
