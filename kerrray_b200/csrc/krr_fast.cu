// Fast kernels: FP64 (Fast64) and FP32 stages with FP64 accumulation (Mixed).  Their FMAs are
// written out in the source; the translation unit is compiled with -fmad=false so the compiler
// fuses nothing else and every launch variant (register cap) computes identical results.
#include <math_constants.h>

#include <algorithm>

#include "krr_launch.h"

namespace krr {

cudaError_t fast_plain(bool mixed, bool rk4, const PlainArgs& a, int block, cudaStream_t s) {
  if (mixed) {
    if (rk4) return cudaErrorNotSupported;
    return run_plain<Mixed, false>(a, block, s);
  }
  return rk4 ? run_plain<Fast64, true>(a, block, s) : run_plain<Fast64, false>(a, block, s);
}

// Launch shapes the autotuner chooses from: (threads per block, minimum resident blocks per SM).
// The minimum caps the registers at 65536 / (block * min_blocks): unbounded, 170, 128 and 102
// for FP64; unbounded, 128, 102 and 85 for the mixed mode.
const Variant* fast_variants(bool mixed, bool rk4, int* count) {
  static const Variant f64[] = {
      make_variant<Fast64, false, 128, 1>(), make_variant<Fast64, false, 128, 3>(),
      make_variant<Fast64, false, 128, 4>(), make_variant<Fast64, false, 128, 5>(),
      make_variant<Fast64, false, 256, 2>(), make_variant<Fast64, false, 64, 8>(),
  };
  static const Variant f64rk4[] = {make_variant<Fast64, true, 128, 1>()};
  static const Variant mix[] = {
      make_variant<Mixed, false, 128, 1>(), make_variant<Mixed, false, 128, 4>(),
      make_variant<Mixed, false, 128, 5>(), make_variant<Mixed, false, 128, 6>(),
      make_variant<Mixed, false, 256, 2>(), make_variant<Mixed, false, 64, 10>(),
  };
  if (mixed) {
    if (rk4) {
      *count = 0;
      return nullptr;
    }
    *count = (int)(sizeof(mix) / sizeof(mix[0]));
    return mix;
  }
  if (rk4) {
    *count = 1;
    return f64rk4;
  }
  *count = (int)(sizeof(f64) / sizeof(f64[0]));
  return f64;
}

const Variant* near_wide_variant() {
  static const Variant v = make_variant<Fast64, false, 384, 1>();
  return &v;
}

// The mixed re-trace of the few rays an FP32 overflow ended early (MixedSat: an overflowing
// trial step is a rejection, as in FP64).
const Variant* mixed_sat_variant() {
  static const Variant v = make_variant<MixedSat, false, 128, 4>();
  return &v;
}

// Where an escaped ray crosses r = r_s: from its final state (the first accepted state at or
// beyond the escape radius, which overshoots the surface by up to a step), flow back along the
// same Hamiltonian in FP64 (classical RK4, 32 substeps of the FP64 separated right-hand side)
// over the affine offset dl that Newton's method drives to r(dl) = r_s (dr/dl = f_r), three
// iterations from the linear estimate.  Gives theta and phi on the surface, the quantities two
// integrations of the same ray can be compared on whatever steps they took.
__device__ void flow_rk4(const Params& P, double y[8], double dl, int n) {
  const double hh = dl / n;
  auto f8 = [&](const double z[8], double out[8]) {
    double f[NV];
    Trig tr;
    Fast64::rhs(P, z[1], z[2], z[4], z[5], z[6], z[7], f, tr);
    out[0] = f[CT];
    out[1] = f[CR];
    out[2] = f[CTH];
    out[3] = f[CPH];
    out[4] = 0.0;
    out[5] = f[CPR];
    out[6] = f[CPTH];
    out[7] = 0.0;
  };
  for (int k = 0; k < n; ++k) {
    double k1[8], k2[8], k3[8], k4[8], z[8];
    f8(y, k1);
    for (int i = 0; i < 8; ++i) z[i] = fma(0.5 * hh, k1[i], y[i]);
    f8(z, k2);
    for (int i = 0; i < 8; ++i) z[i] = fma(0.5 * hh, k2[i], y[i]);
    f8(z, k3);
    for (int i = 0; i < 8; ++i) z[i] = fma(hh, k3[i], y[i]);
    f8(z, k4);
    for (int i = 0; i < 8; ++i) y[i] = fma(hh / 6.0, k1[i] + 2.0 * (k2[i] + k3[i]) + k4[i], y[i]);
  }
}

__global__ void k_escape_directions(Params P, double r_s, const double* __restrict__ Y,
                                    const long long* __restrict__ state, long long n, double* __restrict__ theta,
                                    double* __restrict__ phi) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double th = CUDART_NAN, ph = CUDART_NAN;
  if (state[i] == ESCAPED) {
    double y0[8], y[8], f[NV];
    Trig tr;
    for (int c = 0; c < 8; ++c) y0[c] = Y[i * 8 + c];
    Fast64::rhs(P, y0[1], y0[2], y0[4], y0[5], y0[6], y0[7], f, tr);
    double dl = -(y0[1] - r_s) / f[CR];
    for (int it = 0; it < 3; ++it) {
      for (int c = 0; c < 8; ++c) y[c] = y0[c];
      flow_rk4(P, y, dl, 32);
      Fast64::rhs(P, y[1], y[2], y[4], y[5], y[6], y[7], f, tr);
      dl -= (y[1] - r_s) / f[CR];
    }
    for (int c = 0; c < 8; ++c) y[c] = y0[c];
    flow_rk4(P, y, dl, 32);
    th = y[2];
    ph = y[3];
  }
  theta[i] = th;
  phi[i] = ph;
}

cudaError_t escape_directions(const Params& P, double r_s, const double* Y, const long long* state, long long n,
                              double* theta, double* phi, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int block = 128;
  k_escape_directions<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(P, r_s, Y, state, n, theta, phi);
  return cudaGetLastError();
}

// The step kernels' own sines and cosines at given angles, for accuracy checks: which 0 is
// sincos_reduced(theta) (FP32, the mixed mode's accepted states); 1 is sincos_shift_x2 from the
// FP32-rounded sine and cosine of theta by (float)delta (the mixed stages); 2 is sincos_shift from
// the FP64 sine and cosine of theta by delta (the fast64 stages).  NaN where a shift declines.
__global__ void k_trig_eval(int which, const double* __restrict__ theta, const double* __restrict__ delta, long long n,
                            double* __restrict__ s_out, double* __restrict__ c_out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double th = theta[i];
  double s = CUDART_NAN, c = CUDART_NAN;
  if (which == 0) {
    float fs, fc;
    sincos_reduced(th, fs, fc);
    s = fs;
    c = fc;
  } else {
    double s0, c0;
    sincos(th, &s0, &c0);
    if (which == 1) {
      float fs, fc;
      if (sincos_shift_x2((float)s0, (float)c0, (float)delta[i], fs, fc)) {
        s = fs;
        c = fc;
      }
    } else {
      double ds, dc;
      if (sincos_shift(s0, c0, delta[i], ds, dc)) {
        s = ds;
        c = dc;
      }
    }
  }
  s_out[i] = s;
  c_out[i] = c;
}

cudaError_t trig_eval(int which, const double* theta, const double* delta, long long n, double* s_out, double* c_out,
                      cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int block = 256;
  k_trig_eval<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(which, theta, delta, n, s_out, c_out);
  return cudaGetLastError();
}

// Accretion-disk shading of the disk-plane crossings (raytracing/renderer.py:render_disk step
// 3): the redshift factor g = nu_obs / nu_em of each crossing state for a circular equatorial
// Keplerian emitter (physics/redshift.py:redshift_factor, BPT 1972 eq. 2.16 for Omega, u^t from
// the normalisation at theta = pi/2) and I_obs = g^n (r / r_in)^-p on r_in <= r <= r_out
// (physics/accretion.py:observed_intensity).  g = (-p_t) / (-p_mu u^mu) is the same for the
// stored (reversed) momentum.  Rows without a hit: g = r_hit = NaN, I = 0; a hit that is not
// equatorial (to 1e-6), lies where no circular orbit exists, or gives g <= 0 gets g = NaN (the
// caller raises, as the reference does).
__global__ void k_disk_shading(double m, double a, int prograde, double r_in, double r_out, double p_index, int n_pow,
                               const double* __restrict__ Y, const unsigned char* __restrict__ hit, long long n,
                               double* __restrict__ g_out, double* __restrict__ i_out, double* __restrict__ r_hit) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double g = CUDART_NAN, inten = 0.0, rh = CUDART_NAN;
  if (hit[i]) {
    const double* y = Y + 8 * i;
    const double r = y[1], th = y[2], pt = y[4], pph = y[7];
    rh = r;
    const double s = prograde ? 1.0 : -1.0;
    const double sa = (a < 0.0) ? -1.0 : 1.0;
    const double sqm = sqrt(m);
    const double om = s * sa * sqm / (r * sqrt(r) + s * fabs(a) * sqm);
    const double g_tt = -(1.0 - 2.0 * m / r);
    const double g_tph = -2.0 * m * a / r;
    const double g_phph = r * r + a * a + 2.0 * m * a * a / r;
    const double rad = -(g_tt + 2.0 * om * g_tph + om * om * g_phph);
    if (fabs(th - 0.5 * CUDART_PI) <= 1e-6 && isfinite(rad) && rad > 0.0) {
      const double ut = 1.0 / sqrt(rad);
      const double gg = pt / (pt * ut + pph * (om * ut));
      if (isfinite(gg) && gg > 0.0) {
        g = gg;
        double gn = gg * gg * gg;
        if (n_pow == 4) gn *= gg;
        if (r >= r_in && r <= r_out) inten = pow(r / r_in, -p_index) * gn;
      }
    }
  }
  g_out[i] = g;
  i_out[i] = inten;
  r_hit[i] = rh;
}

cudaError_t disk_shading(double m, double a, int prograde, double r_in, double r_out, double p_index, int n_pow,
                         const double* Y, const unsigned char* hit, long long n, double* g, double* inten, double* r_hit,
                         cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int block = 256;
  k_disk_shading<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(m, a, prograde, r_in, r_out, p_index, n_pow, Y,
                                                                       hit, n, g, inten, r_hit);
  return cudaGetLastError();
}

// Count of the non-finite values among n doubles (added to *count).
__global__ void k_count_nonfinite(const double* __restrict__ x, long long n, unsigned long long* count) {
  unsigned long long mine = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) mine += !isfinite(x[i]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, off);
  if ((threadIdx.x & 31u) == 0 && mine) atomicAdd(count, mine);
}

cudaError_t count_nonfinite(const double* x, long long n, unsigned long long* count, int sms, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n + 255) / 256, (long long)std::max(sms, 1) * 8);
  k_count_nonfinite<<<(unsigned)blocks, 256, 0, s>>>(x, n, count);
  return cudaGetLastError();
}

// The fast64 bisection at three blocks per SM (168 registers, spilling 44 B) only for a study
// large enough to keep those lanes at most 3/4 of its items (run_bisect's rule); below that at
// two blocks per SM, whose register budget holds the whole kernel (186-188 registers, no spills:
// 2.5 % faster on the 51,840-item edge study).  On a study of 155,520 items the build for three
// at three blocks per SM takes 283-288 ms, the build for two at two 310-318 ms.
cudaError_t fast_bisect(bool mixed, const EdgeArgs& a, cudaStream_t s) {
  if (mixed) return run_bisect<Mixed, 128, 1>(a, s);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (4LL * sms * 3 * 128 <= 3LL * a.n_items) return run_bisect<Fast64, 128, 3>(a, s);
  return run_bisect<Fast64, 128, 2>(a, s);
}

}  // namespace krr
