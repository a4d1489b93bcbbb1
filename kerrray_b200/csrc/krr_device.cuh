// Device code of the per-ray hot path: Kerr Boyer-Lindquist Hamiltonian right-hand side,
// adaptive Dormand-Prince 5(4) step with the Hairer-Norsett-Wanner error norm and step
// controller, termination classification and the conservation diagnostics.
//
// Semantics follow KerrRay's scalar ray kernel (src/kerrray/raytracing/backends/
// numba_kernel.py:111-463): same state layout [t, r, theta, phi, p_t, p_r, p_theta, p_phi]
// (geodesics/state.py:35), same tableau (geodesics/tableaus.py:59-91), same controller
// constants and the same classification priority (photons/classification.py:72-130).
//
// One photon lives in one thread's registers.  p_t and p_phi are exact constants of the
// motion in this formulation (their right-hand sides are identically zero, so the reference's
// stage sums leave them bit-unchanged) and are carried as scalars; the other six components
// are integrated.  Three arithmetic modes share the step/controller/classification code:
//
//   RefMode<double>  reference operation order in FP64 (compile the translation unit with
//                    -fmad=false so that products and sums round separately as in the
//                    reference's fastmath=False build);
//   RefMode<float>   the reference's float32 working-precision mode (metric in FP64, cast);
//   Fast64           FP64 with explicit FMAs, sincos, three reciprocals instead of the
//                    seventeen divisions, and a single-precision step-factor power;
//   Mixed            FP32 stages (metric, right-hand side, stage sums, error estimate) with the
//                    state accumulation y + h*sum(b_i k_i), Delta = r^2 - 2Mr + a^2 and the error
//                    norm in FP64.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace krr {

enum : int { RUNNING = 0, ESCAPED = 1, CAPTURED = 2, MAX_AFFINE = 3, FAILURE = 4, OUT_OF_DOMAIN = 5, DISK_HIT = 6 };

// Integrated components (indices into the 6-vectors) and their positions in the 8-state.
enum : int { CT = 0, CR = 1, CTH = 2, CPH = 3, CPR = 4, CPTH = 5, NV = 6 };

// ------------------------------------------------------------------------------------------
// Dormand-Prince 5(4) (Dormand & Prince 1980; Hairer, Norsett & Wanner 1993, Table 5.2).
// ------------------------------------------------------------------------------------------
namespace dp {
constexpr double A10 = 1.0 / 5.0;
constexpr double A20 = 3.0 / 40.0, A21 = 9.0 / 40.0;
constexpr double A30 = 44.0 / 45.0, A31 = -56.0 / 15.0, A32 = 32.0 / 9.0;
constexpr double A40 = 19372.0 / 6561.0, A41 = -25360.0 / 2187.0, A42 = 64448.0 / 6561.0, A43 = -212.0 / 729.0;
constexpr double A50 = 9017.0 / 3168.0, A51 = -355.0 / 33.0, A52 = 46732.0 / 5247.0, A53 = 49.0 / 176.0,
                 A54 = -5103.0 / 18656.0;
constexpr double B0 = 35.0 / 384.0, B2 = 500.0 / 1113.0, B3 = 125.0 / 192.0, B4 = -2187.0 / 6784.0, B5 = 11.0 / 84.0;
// Error weights E = b_hat - b (tableaus.py:85), evaluated in double like the reference.
constexpr double E0 = 5179.0 / 57600.0 - 35.0 / 384.0;
constexpr double E2 = 7571.0 / 16695.0 - 500.0 / 1113.0;
constexpr double E3 = 393.0 / 640.0 - 125.0 / 192.0;
constexpr double E4 = -92097.0 / 339200.0 - (-2187.0 / 6784.0);
constexpr double E5 = 187.0 / 2100.0 - 11.0 / 84.0;
constexpr double E6 = 1.0 / 40.0 - 0.0;
// Classical RK4 (Hairer, Norsett & Wanner 1993, Table 1.2).
constexpr double RK4_B0 = 1.0 / 6.0, RK4_B1 = 1.0 / 3.0, RK4_B2 = 1.0 / 3.0, RK4_B3 = 1.0 / 6.0;
}  // namespace dp

// Controller constants (tableaus.py:88-91).
constexpr double SAFETY = 0.9, FACTOR_MIN = 0.2, FACTOR_MAX = 5.0, ERROR_EXPONENT = -1.0 / 5.0;
// Classification tolerances (classification.py:53,56).
constexpr double THETA_TOL = 1e-9, AXIS_SIN_TOL = 1e-12;
constexpr double PI = 3.141592653589793;

// ------------------------------------------------------------------------------------------
// Parameters of one batch (or one image): geometry constants packed like numba_backend.py:96-97
// plus the integrator, termination and event options.
// ------------------------------------------------------------------------------------------
struct Params {
  double mass, a, a2, neg_2ma, pos_2ma, two_m, two_a2;
  double rtol, atol, h0, h_min, h_max, lambda_max;
  double r_capture, r_escape, r_in, r_out;
  double r_plus;  // outer horizon M + sqrt(M^2 - a^2)
  long long max_steps, guard;
  int rk4;   // 0: Dormand-Prince 5(4), 1: fixed-step RK4
  int disk;  // disk-plane event enabled
  // FP32 copies for the mixed mode's stages (rounded once on the host).
  float f_mass, f_a, f_a2;
  float f_rpm;  // r_plus - r_minus = 2 sqrt(M^2 - a^2)
};

// Per-ray conservation references (numba_backend.py:174-178).  E and L_z are exact constants
// of the integration here, so only Q0 and the two denominators of the drifts are kept:
// max(|Q0|, E0^2 M^2) for the Carter constant and E0^2 for the null error.  The reference
// modes divide by them; the fast modes keep their reciprocals and multiply.
template <class D>
struct Refs {
  double q0;
  D q_den, e_den;
};

// x / den in the reference modes, x * den (den holding the reciprocal) in the fast modes.
template <class M>
__device__ __forceinline__ double drift(double x, double den) {
  if constexpr (M::kFused) return x * den;
  else return x / den;
}

// ------------------------------------------------------------------------------------------
// Arithmetic modes.
// ------------------------------------------------------------------------------------------
template <class X>
__device__ __forceinline__ X py_max(X a, X b) { return (b > a) ? b : a; }  // Python max(a, b)
template <class X>
__device__ __forceinline__ X py_min(X a, X b) { return (b < a) ? b : a; }  // Python min(a, b)

__device__ __forceinline__ bool finite_(double x) { return isfinite(x); }
__device__ __forceinline__ bool finite_(float x) { return isfinite(x); }

// a*x + acc: one fused operation in the fast modes, two roundings (the reference's order) in
// the reference modes.  Contraction is never left to the compiler, so every launch variant of
// a mode computes the same bits.
__device__ __forceinline__ double fused(double a, double x, double acc) { return fma(a, x, acc); }
__device__ __forceinline__ float fused(float a, float x, float acc) { return fmaf(a, x, acc); }

template <class M, class X>
__device__ __forceinline__ X madd(X acc, X a, X x) {
  if constexpr (M::kFused) return fused(a, x, acc);
  else return acc + a * x;
}

// y + h * acc, the state update of a stage.  The mixed mode forms h * acc exactly in FP64 (a
// product of two floats) and rounds once when adding it to the FP64 state.
template <class M>
__device__ __forceinline__ typename M::S upd(typename M::S y, typename M::K h, typename M::K acc) {
  using S = typename M::S;
  if constexpr (!M::kFused) return y + (S)(h * acc);
  else return fused((S)h, (S)acc, y);
}

// Sine and cosine of the last right-hand-side evaluation, reused by classification and the
// Carter constant (same function, same argument, so the same values the reference recomputes).
struct Trig {
  double s, c;
};

// Reference operation order (numba_kernel.py:111-197).  W is the working type; the metric is
// always FP64 and cast to W before it meets the momenta.
template <class W>
struct RefMode {
  using S = W;       // state type
  using K = W;       // stage type
  using N = W;       // error-norm type
  using D = double;  // diagnostics (running maxima and their denominators)
  static constexpr bool kSaturate = false;
  static constexpr bool kMixed = false;
  static constexpr bool kFused = false;

  __device__ static Trig accept_trig(double, const Trig& tr) { return tr; }

  struct Shadow {};

  __device__ static void init_rhs(const Params& P, const S y[NV], S pt, S pph, Shadow&, K f[NV], Trig& tr) {
    rhs(P, y[CR], y[CTH], pt, y[CPR], y[CPTH], pph, f, tr);
  }
  __device__ static void accepted(const Params&, const S[NV], Shadow&, const Trig&) {}

  // Right-hand side at the stage input y + h*acc (on LAST also returned in yn: the new state);
  // IDX is the stage's number (1..6).
  template <bool LAST, int IDX, class R>
  __device__ static void stage(const Params& P, const R& ry, K h, const K acc[NV], K f[NV], Trig& tr, S yn[NV]) {
    S ys[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) ys[i] = upd<RefMode<W>>(ry.y[i], h, acc[i]);
    if constexpr (LAST) {
#pragma unroll
      for (int i = 0; i < NV; ++i) yn[i] = ys[i];
    }
    rhs(P, ys[CR], ys[CTH], ry.pt, ys[CPR], ys[CPTH], ry.pph, f, tr);
  }

  __device__ static void metric(const Params& P, double r, double th, double g[15], Trig& tr) {
    const double m = P.mass, a2 = P.a2;
    const double s = sin(th);
    const double c = cos(th);
    tr.s = s;
    tr.c = c;
    const double s2 = s * s;
    const double sin2th = sin(2.0 * th);
    const double r2 = r * r;
    const double sig = r2 + a2 * (c * c);
    const double dlt = r2 - P.two_m * r + a2;
    const double r2a2 = r2 + a2;
    const double big_a = r2a2 * r2a2 - a2 * dlt * s2;
    const double sd = sig * dlt;
    g[0] = -big_a / sd;
    g[1] = P.neg_2ma * r / sd;
    g[2] = dlt / sig;
    g[3] = 1.0 / sig;
    g[4] = (dlt - a2 * s2) / (sd * s2);
    const double sig_r = 2.0 * r;
    const double sig_th = (-a2) * sin2th;
    const double dlt_r = 2.0 * (r - m);
    const double a_r = 4.0 * r * r2a2 - P.two_a2 * (r - m) * s2;
    const double a_th = (-a2) * dlt * sin2th;
    const double sd_r = sig_r * dlt + sig * dlt_r;
    const double sd_th = sig_th * dlt;
    const double sd2 = sd * sd;
    const double sig2 = sig * sig;
    g[5] = -(a_r * sd - big_a * sd_r) / sd2;
    g[6] = P.neg_2ma * (sd - r * sd_r) / sd2;
    g[7] = (dlt_r * sig - dlt * sig_r) / sig2;
    g[8] = -sig_r / sig2;
    g[9] = -sig_r / (sig2 * s2) + a2 * sd_r / sd2;
    g[10] = -(a_th * sd - big_a * sd_th) / sd2;
    g[11] = P.pos_2ma * r * sd_th / sd2;
    g[12] = -dlt * sig_th / sig2;
    g[13] = -sig_th / sig2;
    g[14] = -(sig_th * s2 + sig * sin2th) / (sig2 * (s2 * s2)) + a2 * sd_th / sd2;
  }

  // f (6 integrated components) at state (r, th, pr, pth) with constants (pt, pph).
  __device__ static void rhs(const Params& P, S r, S th, S pt, S pr, S pth, S pph, K f[NV], Trig& tr) {
    double g64[15];
    metric(P, (double)r, (double)th, g64, tr);
    W g[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) g[i] = (W)g64[i];
    const W zero = (W)0.0, two = (W)2.0, neg_half = (W)-0.5;
    W gphph = g[4], r_gphph = g[9], t_gphph = g[14];
    if (pph == zero) {  // polar-axis guard, numba_kernel.py:177-180
      gphph = zero;
      r_gphph = zero;
      t_gphph = zero;
    }
    f[CT] = g[0] * pt + g[1] * pph;
    f[CR] = g[2] * pr;
    f[CTH] = g[3] * pth;
    f[CPH] = g[1] * pt + gphph * pph;
    const W pt2 = pt * pt, ptpph = pt * pph, pr2 = pr * pr, pth2 = pth * pth, pph2 = pph * pph;
    f[CPR] = neg_half * (g[5] * pt2 + two * g[6] * ptpph + g[7] * pr2 + g[8] * pth2 + r_gphph * pph2);
    f[CPTH] = neg_half * (g[10] * pt2 + two * g[11] * ptpph + g[12] * pr2 + g[13] * pth2 + t_gphph * pph2);
  }
};

// ------------------------------------------------------------------------------------------
// The fast modes' right-hand side: the same Hamiltonian in Carter's separated form,
//
//   2 Sigma H = Delta p_r^2 + p_theta^2 - K^2 / Delta + v^2,
//   K = (r^2 + a^2) E - a L,   v = L / sin(theta) - a E sin(theta),   E = -p_t,   L = p_phi,
//
// which is an algebraic identity of g^{mu nu} p_mu p_nu for the Boyer-Lindquist inverse metric
// (Carter 1968, Phys. Rev. 174, 1559).  Hamilton's equations of this form are therefore the
// reference's right-hand side (numba_kernel.py:158-197) on and off the null shell; only the
// rounding differs.  They take about 50 operations and three reciprocals, where the fifteen
// metric terms and their derivatives take about 95 operations and seventeen divisions.  For
// L = 0 the 1/sin terms vanish identically, as the reference's polar-axis guard makes them.
// ------------------------------------------------------------------------------------------

// 1/x by Newton-Raphson on the hardware's approximate FP64 reciprocal: r <- r + r (1 - x r)
// converges quadratically (steps = 1: about 46 correct bits; steps = 2: a rounding error).
// A zero, infinite or subnormal x gives NaN, where a division gives an infinity: either way the
// step is non-finite and the ray a NUMERICAL_FAILURE.
template <int STEPS = 2>
__device__ __forceinline__ double rcp_newton(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
#pragma unroll
  for (int i = 0; i < STEPS; ++i) r = fma(r, fma(-x, r, 1.0), r);
  return r;
}
// The fast modes' FP64 reciprocal: one Newton step, relative error below 2^-40 (1e-12), four
// orders under the tightest tolerance these modes serve (rtol 1e-10 of the edge study; below
// about 1e-11 the reference precision is the one to use).  The second step cost 4 % of the
// FP64-bound sweep and changed no terminal state of its 12.4M photons.
__device__ __forceinline__ double rcp_fast(double x) { return rcp_newton<1>(x); }
// FP32: the hardware reciprocal alone (relative error within 2^-23; subnormals flush to zero).
// __fdividef(1, x) gives the same values in this kernel's range but adds the handling of
// subnormal quotients around it: about 9 % of the mixed kernel's time.
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// sin and cos of theta0 + d from s0 = sin(theta0), c0 = cos(theta0) by the angle-addition
// formulas, with sin d and cos d from their Taylor series: through d^9 and d^10 in FP64
// (|d| <= 1/10: truncation below 3e-19); the FP32 form (sincos_shift_x2) goes through d^7 and
// d^6 (|d| <= 1/4: below 4e-10).  The stages of one step move theta by such small amounts, so
// this replaces a full sincos (argument reduction and two polynomials) by about a dozen fused
// operations.  Returns false, computing nothing, when |d| exceeds the range.
__device__ __forceinline__ bool sincos_shift(double s0, double c0, double d, double& s, double& c) {
  if (!(fabs(d) <= 0.1)) return false;
  const double d2 = d * d;
  const double sd = d * fma(d2, fma(d2, fma(d2, fma(d2, 1.0 / 362880.0, -1.0 / 5040.0), 1.0 / 120.0), -1.0 / 6.0), 1.0);
  const double cd =
      fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, -1.0 / 3628800.0, 1.0 / 40320.0), -1.0 / 720.0), 1.0 / 24.0), -0.5), 1.0);
  s = fma(s0, cd, c0 * sd);
  c = fma(c0, cd, -(s0 * sd));
  return true;
}

// Per-ray constants of the separated form.
template <class T>
struct Motion {
  T e, l;    // E = -p_t, L = p_phi
  T ae, al;  // a E, a L
  T m2e;     // -2 E
  __device__ void set(T pt, T pph, T a) {
    e = -pt;
    l = pph;
    ae = a * e;
    al = a * l;
    m2e = T(-2) * e;
  }
};

// f (six integrated components) at (r, theta, p_r, p_theta) with Delta supplied by the mode.
// With T_DEVIATION, f[CT] holds dt/dlambda - E = 2 M r K / (Delta Sigma) instead of dt/dlambda:
// the identity Sigma dt/dlambda = a sin v + (r^2 + a^2) K / Delta = E Sigma + 2 M r K / Delta.
// Far from the hole dt/dlambda is E to within 2M/r; an FP32 stage value of it carries rounding
// noise of 6e-8 E, which the Dormand-Prince error estimate (sum_j E_j k_j, a difference of
// nearly equal stages) reads as an error of t -- whose scale atol + rtol |t| is small near the
// observer, where t starts at 0 -- and the controller then takes another step sequence than
// FP64 would.  The deviation rounds relative to its own, small size instead.
//
// With T_DEVIATION and r_deviation (a runtime choice), f[CR] holds dr/dlambda - p_r =
// p_r (a^2 sin^2 - 2 M r) / Sigma (as Delta = Sigma - 2 M r + a^2 sin^2): far from the hole dr/dlambda
// is p_r to within 2M/r, and a step's stages then differ from p_r by small amounts that FP32
// keeps to its relative precision (the r error estimate's rounding noise otherwise steers the
// controller on long steps, whose r scale rtol r is comparable with 6e-8 h |p_r| / r).  Near the
// hole, where that difference is most of dr/dlambda, f[CR] is dr/dlambda itself.
template <class T, bool T_DEVIATION = false>
__device__ __forceinline__ void rhs_separated(T dlt, T r, T s, T c, T pr, T pth, const Motion<T>& mo, T a, T a2,
                                              T m, T f[NV], bool r_deviation = false) {
  const T r2a2 = fused(r, r, a2);                          // r^2 + a^2
  const T as = a * s;
  const T a2s = a * as;                                    // a^2 sin
  const T k = fused(r2a2, mo.e, -mo.al);                    // K
  const T isig = rcp_fast(fused(-a2s, s, r2a2));           // 1 / Sigma, Sigma = r^2 + a^2 - a^2 sin^2
  const T kd = k * rcp_fast(dlt);                          // K / Delta
  const T is = (mo.l != T(0)) ? rcp_fast(s) : T(0);        // 1 / sin (unused for L = 0)
  const T lis = mo.l * is;                                 // L / sin
  const T v = fused(-mo.ae, s, lis);                       // L / sin - a E sin
  const T rm = r - m;
  const T pr2 = pr * pr;
  const T bs = fused(v, v, fused(-k, kd, fused(dlt, pr2, pth * pth))) * isig;  // 2 H = B / Sigma
  if constexpr (T_DEVIATION) f[CT] = ((m + m) * r) * kd * isig;  // -dH/dE - E
  else f[CT] = isig * fused(as, v, kd * r2a2);                      // -dH/dE
  if constexpr (T_DEVIATION) f[CR] = pr * (r_deviation ? fused(a2s, s, -(m + m) * r) : dlt) * isig;
  else f[CR] = dlt * pr * isig;                            // dH/dp_r
  f[CTH] = pth * isig;                                     // dH/dp_theta
  f[CPH] = isig * fused(a, kd, fused(lis, is, -mo.ae));    // dH/dL = (a K / Delta + L / sin^2 - a E) / Sigma
  // -dH/dr = (r B / Sigma - (r - M) p_r^2 - (K / Delta)((K / Delta)(r - M) - 2 E r)) / Sigma
  f[CPR] = isig * fused(r, bs, -fused(rm, pr2, kd * fused(kd, rm, mo.m2e * r)));
  // -dH/dtheta = cos (v (L / sin^2 + a E) - a^2 sin B / Sigma) / Sigma
  f[CPTH] = (isig * c) * fused(v, fused(lis, is, mo.ae), -a2s * bs);
}

// rhs_separated<float, true>, the mixed mode's right-hand side, with its six numerators
// multiplied by 1 / Sigma as three packed pairs in the pairing of the mixed stage sums:
// out[0] = (f_r, f_theta), out[1] = (f_pr, f_ptheta), out[2] = (f_t, f_phi), f_t (and, far,
// f_r) as deviations.  Every value is the same operation on the same operands as in
// rhs_separated (f_ptheta = F * (1/Sigma * cos) as there), so the results are its results bit
// for bit, in three packed multiplies where it takes six, and with 2 M r formed once.
__device__ __forceinline__ void rhs_separated_pairs(float dlt, float r, float s, float c, float pr, float pth,
                                                    const Motion<float>& mo, float a, float a2, float m,
                                                    float2 out[3], bool far) {
  const float r2a2 = fmaf(r, r, a2);
  const float as = a * s;
  const float a2s = a * as;
  const float k = fmaf(r2a2, mo.e, -mo.al);
  const float isig = rcp_fast(fmaf(-a2s, s, r2a2));
  const float kd = k * rcp_fast(dlt);
  const float is = (mo.l != 0.0f) ? rcp_fast(s) : 0.0f;
  const float lis = mo.l * is;
  const float v = fmaf(-mo.ae, s, lis);
  const float rm = r - m;
  const float pr2 = pr * pr;
  const float bs = fmaf(v, v, fmaf(-k, kd, fmaf(dlt, pr2, pth * pth))) * isig;
  const float tmr = (m + m) * r;
  out[0] = __fmul2_rn(make_float2(pr * (far ? fmaf(a2s, s, -tmr) : dlt), pth), make_float2(isig, isig));
  out[1] = __fmul2_rn(make_float2(fmaf(r, bs, -fmaf(rm, pr2, kd * fmaf(kd, rm, mo.m2e * r))),
                                  fmaf(v, fmaf(lis, is, mo.ae), -a2s * bs)),
                      make_float2(isig, isig * c));
  out[2] = __fmul2_rn(make_float2(tmr * kd, fmaf(a, kd, fmaf(lis, is, -mo.ae))), make_float2(isig, isig));
}

// The FP32 sincos_shift on packed pairs (fma/mul.rn.f32x2, sm_100): the sine and cosine
// polynomials and the two rotation products advance together, every value the same operation
// on the same operands as in the scalar form.  (The right-hand side stays scalar: packing its
// operands ties registers into pairs, and the moves cost more than the instructions saved.)
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ bool sincos_shift_x2(float s0, float c0, float d, float& s, float& c) {
  if (!(fabsf(d) <= 0.25f)) return false;
  const float d2 = d * d;
  const float2 dd = f2(d2, d2);
  float2 p = __ffma2_rn(dd, f2(-1.0f / 5040.0f, -1.0f / 720.0f), f2(1.0f / 120.0f, 1.0f / 24.0f));
  p = __ffma2_rn(dd, p, f2(-1.0f / 6.0f, -0.5f));
  p = __ffma2_rn(dd, p, f2(1.0f, 1.0f));  // (sin d / d, cos d)
  const float sd = d * p.x;
  const float2 t = __fmul2_rn(f2(c0, -s0), f2(sd, sd));
  const float2 r = __ffma2_rn(f2(s0, c0), f2(p.y, p.y), t);
  s = r.x;
  c = r.y;
  return true;
}

// sin and cos of an FP64 angle to FP32 accuracy (the mixed mode's accepted states and its rare
// stage fallback), in about twenty instructions and no slow path:
// - Cody and Waite's reduction by the nearest multiple k of pi/2, in FP64 with pi/2 split in two
//   (x = th - k pi/2, |x| <= pi/4, for |th| < 2^51).  Next to the axis (th near 0 or pi) x keeps
//   its relative accuracy.  k is rounded to nearest by adding 1.5 * 2^52, whose low word is then
//   k mod 2^32;
// - the Taylor series of sin(x)/x through x^8 and of cos x through x^10, in x^2, on packed pairs
//   (truncation below 3e-9 and 1.2e-10 of the value for |x| <= pi/4);
// - k mod 4 picks the pair and its signs.
__device__ __forceinline__ void sincos_reduced(double th, float& s, float& c) {
  constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
  constexpr double kPio2Hi = 1.5707963267948966, kPio2Lo = 6.123233995736766e-17;
  const double t = fma(th, 2.0 / PI, kRound);
  const int q = __double2loint(t);
  const double k = t - kRound;
  const float x = (float)fma(-k, kPio2Lo, fma(-k, kPio2Hi, th));
  const float x2 = x * x;
  const float2 dd = f2(x2, x2);
  float2 p = __ffma2_rn(dd, f2(0.0f, -1.0f / 3628800.0f), f2(1.0f / 362880.0f, 1.0f / 40320.0f));
  p = __ffma2_rn(dd, p, f2(-1.0f / 5040.0f, -1.0f / 720.0f));
  p = __ffma2_rn(dd, p, f2(1.0f / 120.0f, 1.0f / 24.0f));
  p = __ffma2_rn(dd, p, f2(-1.0f / 6.0f, -0.5f));
  p = __ffma2_rn(dd, p, f2(1.0f, 1.0f));  // (sin x / x, cos x)
  const float sx = x * p.x, cx = p.y;
  const float u = (q & 1) ? cx : sx;
  const float v = (q & 1) ? sx : cx;
  s = (q & 2) ? -u : u;
  c = ((q + 1) & 2) ? -v : v;
}

// FP64 with explicit FMAs, sincos and Newton reciprocals on the separated form.
struct Fast64 {
  using S = double;
  using K = double;
  using N = double;
  using D = float;  // the drift maxima: FP64 values, kept to single precision
  static constexpr bool kSaturate = false;
  static constexpr bool kMixed = false;
  static constexpr bool kFused = true;

  __device__ static Trig accept_trig(double, const Trig& tr) { return tr; }

  // kTape: the shadow records each inner stage input (Fast64 derivatives with a shadow that
  // has record(): the adjoint's forward pass).
  struct Shadow {
    static constexpr bool kTape = false;
  };

  __device__ static void init_rhs(const Params& P, const S y[NV], S pt, S pph, Shadow&, K f[NV], Trig& tr) {
    rhs(P, y[CR], y[CTH], pt, y[CPR], y[CPTH], pph, f, tr);
  }
  __device__ static void accepted(const Params&, const S[NV], Shadow&, const Trig&) {}

  // Right-hand side at the stage input y + h*acc (on LAST also returned in yn: the new state);
  // IDX is the stage's number (1..6).  Stages 1..5 take sin and cos of their theta from the
  // accepted state's (ry.tr, exact) by a small-angle shift; the last stage evaluates them
  // exactly at the candidate, whose trig then serves the classification, the diagnostics and
  // the next step.  With a recording shadow, stages 1..5 hand (r, p_r, p_theta, sin, cos) of
  // their input to it.
  template <bool LAST, int IDX, class R>
  __device__ static void stage(const Params& P, const R& ry, K h, const K acc[NV], K f[NV], Trig& tr, S yn[NV]) {
    S ys[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) ys[i] = upd<Fast64>(ry.y[i], h, acc[i]);
    double s, c;
    if constexpr (LAST) {
#pragma unroll
      for (int i = 0; i < NV; ++i) yn[i] = ys[i];
      sincos(ys[CTH], &s, &c);
    } else {
      if (!sincos_shift(ry.tr.s, ry.tr.c, ys[CTH] - ry.y[CTH], s, c)) sincos(ys[CTH], &s, &c);
    }
    tr.s = s;
    tr.c = c;
    if constexpr (decltype(ry.sh)::kTape && !LAST) ry.sh.record(IDX, ys[CR], ys[CPR], ys[CPTH], s, c);
    rhs_sc(P, ys[CR], s, c, ry.pt, ys[CPR], ys[CPTH], ry.pph, f);
  }

  __device__ static void rhs(const Params& P, double r, double th, double pt, double pr, double pth, double pph,
                             double f[NV], Trig& tr) {
    double s, c;
    sincos(th, &s, &c);
    tr.s = s;
    tr.c = c;
    rhs_sc(P, r, s, c, pt, pr, pth, pph, f);
  }

  __device__ static void rhs_sc(const Params& P, double r, double s, double c, double pt, double pr, double pth,
                                double pph, double f[NV]) {
    Motion<double> mo;
    mo.set(pt, pph, P.a);
    rhs_separated<double>(fma(r, r - P.two_m, P.a2), r, s, c, pr, pth, mo, P.a, P.a2, P.mass, f);
  }
};

// FP32 stages from an FP32 shadow of the FP64 state; FP64 state accumulation, error norm,
// classification and diagnostics.  Delta is formed as (r - r_plus)(r - r_minus): r - r_plus is
// taken from the FP64 state once per accepted step and carried in FP32, so Delta keeps its
// relative accuracy down to the capture margin (the quadratic r^2 - 2Mr + a^2 cancels there).
struct Mixed {
  using S = double;
  using K = float;
  using N = double;
  using D = float;
  static constexpr bool kMixed = true;
  // A trial step through the singular region can overflow the FP32 stages where FP64 stays
  // finite (values of 1e13..1e40 near r_+), and FP64 then rejects it with the smallest step
  // factor because its error norm is huge.  This mode ends such a ray as a NUMERICAL_FAILURE
  // like the reference does on a non-finite step (a handful of rays per million; the
  // pipelines trace them again); MixedSat below rejects instead.
  static constexpr bool kSaturate = false;
  static constexpr bool kFused = true;

  // FP32 copy of what the stages read: (r, r - r_plus), (p_r, p_theta) as packed pairs, theta
  // with its sine and cosine, and the ray's constants of motion.
  struct Shadow {
    float2 rd, pp;
    float ep, psgn, s0, c0;  // theta's distance from the nearer pole (+1: theta, -1: pi - theta)
    Motion<float> mo;
    bool far;  // r > FAR_R M: the r stages hold dr/dlambda - p_r (rhs_separated)
  };

  // Radius (in M) beyond which a step carries dr/dlambda as its deviation from the step's p_r.
  static constexpr double FAR_R = 32.0;

  // The accepted state's sine and cosine: the mixed mode needs them only in FP32 (the shadow,
  // the diagnostics), from theta in FP64 (sincos_reduced); the axis test works on theta itself.
  __device__ static Trig accept_trig(double th, const Trig&) {
    float s, c;
    sincos_reduced(th, s, c);
    Trig t;
    t.s = (double)s;
    t.c = (double)c;
    return t;
  }

  // tr: the accepted state's FP64 sine and cosine (accept_trig).
  __device__ static void accepted(const Params& P, const S y[NV], Shadow& sh, const Trig& tr) {
    sh.rd = make_float2((float)y[CR], (float)(y[CR] - P.r_plus));
    sh.pp = make_float2((float)y[CPR], (float)y[CPTH]);
    const bool south = y[CTH] > 0.5 * PI;
    sh.ep = (float)(south ? PI - y[CTH] : y[CTH]);  // in FP64: FP32 keeps it to its relative precision
    sh.psgn = south ? -1.0f : 1.0f;
    sh.s0 = (float)tr.s;
    sh.c0 = (float)tr.c;
    sh.far = y[CR] > FAR_R * P.mass;
  }

  // After an accepted step: the FSAL value of r in the form of the new state's region (the step
  // computed it in the form of the old one; they differ only when the step crossed FAR_R).
  __device__ static void rebase_fsal(bool far_old, const Shadow& sh, K f[NV]) {
    if (far_old && !sh.far) f[CR] = sh.pp.x + f[CR];
    else if (!far_old && sh.far) f[CR] = f[CR] - sh.pp.x;
  }

  __device__ static void init_rhs(const Params& P, const S y[NV], S pt, S pph, Shadow& sh, K f[NV], Trig& tr) {
    sh.mo.set((float)pt, (float)pph, (float)P.a);
    tr = accept_trig(y[CTH], tr);
    accepted(P, y, sh, tr);
    float2 o[3];
    rhs_f(P, sh.rd.y, sh.rd.x, sh.s0, sh.c0, sh.pp.x, sh.pp.y, sh.mo, o, sh.far);
    f[CR] = o[0].x;
    f[CTH] = o[0].y;
    f[CPR] = o[1].x;
    f[CPTH] = o[1].y;
    f[CT] = o[2].x;
    f[CPH] = o[2].y;
  }

  // The right-hand side at the stage input shadow + h * acc, from the pairs (r, theta) and
  // (p_r, p_theta) of acc; k receives f as the pairs (r, theta), (p_r, p_theta), (t, phi).
  // Every stage's sine and cosine come from the accepted state's by a small-angle shift; near
  // the axis (|sin| < 1/50, where the shift's sum would cancel) or for a large shift,
  // sincos_reduced of the stage's angle from the nearer pole.
  // node: the stage's c_s (sum of its tableau row).  Far from the hole (sh.far) acc[0].x sums the
  // stages' deviations of dr/dlambda from the step's p_r, so the r input adds c_s p_r, and the
  // stage returns its own deviation from that p_r: h sum_j a_sj k_pr,j (its p_r offset) plus
  // rhs_f's.  dev_r (nullable) receives rhs_f's value alone: the FSAL value of the candidate.
  __device__ static void stage(const Params& P, const Shadow& sh, float h, float node, const float2 acc[2],
                               float2 k[3], float* dev_r = nullptr) {
    const float2 hh = make_float2(h, h);
    const float ar = sh.far ? fmaf(node, sh.pp.x, acc[0].x) : acc[0].x;
    const float2 rd = __ffma2_rn(hh, make_float2(ar, ar), sh.rd);  // (r, r - r_plus)
    const float2 pp = __ffma2_rn(hh, acc[1], sh.pp);              // (p_r, p_theta)
    const float dth = h * acc[0].y;
    float s, c;
    if (!(fabsf(sh.s0) >= 0.02f && sincos_shift_x2(sh.s0, sh.c0, dth, s, c))) {
      // Near the axis (or for a long shift): the sine and cosine of the stage's angle from the
      // nearer pole, which FP32 holds to its relative precision (theta itself, next to pi, only
      // to 2.4e-7 absolute: a relative 1e-4 of sin theta at 2e-3 from the axis, which the L/sin
      // and L/sin^2 terms then carried into the stages).
      sincos_reduced((double)fmaf(sh.psgn, dth, sh.ep), s, c);
      c *= sh.psgn;
    }
    float2 o[3];
    rhs_f(P, rd.y, rd.x, s, c, pp.x, pp.y, sh.mo, o, sh.far);
    if (dev_r) *dev_r = o[0].x;
    k[0] = make_float2(sh.far ? fmaf(h, acc[1].x, o[0].x) : o[0].x, o[0].y);
    k[1] = o[1];
    k[2] = o[2];
  }

  // The right-hand side in FP32 at (r - r_plus = d, r, sin, cos, p_r, p_theta), its t component
  // as the deviation dt/dlambda - E and, with far, its r component as dr/dlambda - p_r
  // (rhs_separated): every stage, the FSAL values and the stage sums of t (and of r, far from the
  // hole) hold deviations, and the step adds h E to t (and h p_r to r) in FP64.  The result comes
  // as the stage sums' pairs (rhs_separated_pairs): (r, theta), (p_r, p_theta), (t, phi).
  __device__ static void rhs_f(const Params& P, float d, float rf, float s, float c, float pr, float pth,
                               const Motion<float>& mo, float2 out[3], bool far) {
    rhs_separated_pairs(d * (d + P.f_rpm), rf, s, c, pr, pth, mo, P.f_a, P.f_a2, P.f_mass, out, far);
  }
};

// The mixed mode with an infinite or NaN error norm taken as a rejection with the smallest step
// factor (en^2 = inf or NaN: accept fails, the factor clamps to 1/5), which is what FP64 does
// with the same trial step's huge but finite norm; a ray singular in FP64 as well keeps
// shrinking its step below h_min and still ends as a NUMERICAL_FAILURE.  Used for the few rays
// the mixed trace lost to an FP32 overflow (as the main kernel it costs about 5 % of its time:
// code generation, the attempt counts being the same).
struct MixedSat : Mixed {
  static constexpr bool kSaturate = true;
};
// ------------------------------------------------------------------------------------------
// The state of one ray between step attempts.
// ------------------------------------------------------------------------------------------
template <class M>
struct Ray {
  using S = typename M::S;
  using K = typename M::K;
  S y[NV];   // t, r, theta, phi, p_r, p_theta
  S pt, pph; // constants of the motion
  K f[NV];   // FSAL right-hand side at y
  S h;       // proposed step (working type, like the reference's h)
  S h_taken; // step of the last accepted attempt
  double lam;
  typename M::D m_null, m_q;
  Refs<typename M::D> ref;
  Trig tr;   // sin/cos of theta at y
  typename M::Shadow sh;
  long long attempts;
  int n_steps, n_rej;
  int state;
  bool rejected_before;
};

template <class M>
__device__ __forceinline__ bool all_finite(const typename M::S y[NV], typename M::S pt, typename M::S pph,
                                           const typename M::K f[NV]) {
  bool ok = finite_(pt) && finite_(pph);
#pragma unroll
  for (int i = 0; i < NV; ++i) ok = ok && finite_(y[i]) && finite_(f[i]);
  return ok;
}

// |sin(theta)| < 1e-12 (classification.py:56): from the sine in the reference and fast64 modes;
// in the mixed mode, whose sine is FP32, as min(|theta|, |pi - theta|) < 1e-12 in FP64 (sin x = x
// to a relative 1e-24 there; theta lies in [-1e-9, pi + 1e-9] when this test runs).
template <class M>
__device__ __forceinline__ bool near_axis(const Ray<M>& ry) {
  if constexpr (M::kMixed) {
    const double th = ry.y[CTH];
    return fmin(fabs(th), fabs(PI - th)) < AXIS_SIN_TOL;
  } else {
    using S = typename M::S;
    return fabs((S)ry.tr.s) < (S)AXIS_SIN_TOL;
  }
}

// Termination rules in the reference priority (numba_kernel.py:293-311).  Thresholds are
// compared in the state type like the reference's working-dtype constants.
// check_finite = false where the state and its right-hand side are already known finite (an
// accepted step: the attempt checked the candidate and k6; p_t and p_phi never change).
template <class M>
__device__ __forceinline__ int classify(const Params& P, const Ray<M>& ry, bool check_h, bool check_finite = true) {
  using S = typename M::S;
  if (check_finite && !all_finite<M>(ry.y, ry.pt, ry.pph, ry.f)) return FAILURE;
  if (check_h && ry.h < (S)P.h_min) return FAILURE;
  const S r = ry.y[CR], th = ry.y[CTH];
  if (r < (S)0.0 || th < (S)(-THETA_TOL) || th > (S)(PI + THETA_TOL)) return OUT_OF_DOMAIN;
  if (ry.pph != (S)0.0 && near_axis<M>(ry)) return OUT_OF_DOMAIN;
  if (r <= (S)P.r_capture) return CAPTURED;
  // dr/dlambda = Delta p_r / Sigma has the sign of p_r outside the horizon; the mixed mode's
  // ry.f[CR] may hold its deviation from p_r, so it reads p_r.
  const bool outward = M::kMixed ? ry.y[CPR] > (S)0.0 : ry.f[CR] > (typename M::K)0.0;
  if (r >= (S)P.r_escape && outward) return ESCAPED;
  if (ry.lam >= P.lambda_max || (long long)ry.n_steps >= P.max_steps) return MAX_AFFINE;
  return RUNNING;
}

// |(1/2) p_mu dx^mu/dlambda| in FP64, sequential order (numba_kernel.py:315-321).
template <class M>
__device__ __forceinline__ double null_error(const Ray<M>& ry) {
  if constexpr (M::kMixed) {  // FP32, like the stages it checks
    const Motion<float>& mo = ry.sh.mo;
    float total = fmaf(-mo.e, ry.f[CT], -mo.e * mo.e);  // -E (E + deviation)
    total = fmaf(ry.sh.pp.x, ry.sh.far ? ry.sh.pp.x + ry.f[CR] : ry.f[CR], total);
    total = fmaf(ry.sh.pp.y, ry.f[CTH], total);
    total = fmaf(mo.l, ry.f[CPH], total);
    return (double)fabsf(0.5f * total);
  }
  double total = (double)ry.pt * (double)ry.f[CT];
  total = total + (double)ry.y[CPR] * (double)ry.f[CR];
  total = total + (double)ry.y[CPTH] * (double)ry.f[CTH];
  total = total + (double)ry.pph * (double)ry.f[CPH];
  return fabs(0.5 * total);
}

// Null Carter constant in FP64 (numba_kernel.py:325-336).
template <class M>
__device__ __forceinline__ double carter(const Params& P, const Ray<M>& ry) {
  if constexpr (M::kMixed) {  // FP32 from the shadow, like the stages
    const Mixed::Shadow& sh = ry.sh;
    const float s = sh.s0, c = sh.c0, pth = sh.pp.y;
    const float lz2_over_s2 = (sh.mo.l != 0.0f) ? (sh.mo.l * sh.mo.l) * rcp_fast(s * s) : 0.0f;
    return (double)fmaf(pth, pth, (c * c) * (lz2_over_s2 - sh.mo.ae * sh.mo.ae));
  }
  const double p_th = (double)ry.y[CPTH];
  const double lz = (double)ry.pph;
  const double e = -(double)ry.pt;
  const double s = ry.tr.s, c = ry.tr.c;
  double lz2_over_s2 = 0.0;
  if constexpr (M::kFused) {
    if (lz != 0.0) lz2_over_s2 = (lz * lz) * rcp_newton<2>(s * s);
  } else {
    if (lz != 0.0) lz2_over_s2 = (lz * lz) / (s * s);
  }
  return p_th * p_th + (c * c) * (lz2_over_s2 - P.a2 * e * e);
}

// Set up a ray from its initial 8-state (numba_kernel.py:355-375).  q0 comes from the caller
// (the same closed form evaluated at the initial state).
template <class M>
__device__ __forceinline__ void ray_init(const Params& P, const double y0[8], double q0, Ray<M>& ry) {
  using S = typename M::S;
  ry.y[CT] = (S)y0[0];
  ry.y[CR] = (S)y0[1];
  ry.y[CTH] = (S)y0[2];
  ry.y[CPH] = (S)y0[3];
  ry.pt = (S)y0[4];
  ry.y[CPR] = (S)y0[5];
  ry.y[CPTH] = (S)y0[6];
  ry.pph = (S)y0[7];
  // Drift floors (photons/constants.py:163-171): |E0| (1 if E0 == 0), E0^2 M^2.
  double fe = fabs(y0[4]);
  fe = (fe > 0.0) ? fe : 1.0;
  const double fq = fe * fe * P.mass * P.mass;
  const double q_den = py_max(fabs(q0), fq);
  const double e_den = fe * fe;
  using D = typename M::D;
  ry.ref.q0 = q0;
  ry.ref.q_den = (D)(M::kFused ? 1.0 / q_den : q_den);
  ry.ref.e_den = (D)(M::kFused ? 1.0 / e_den : e_den);
  M::init_rhs(P, ry.y, ry.pt, ry.pph, ry.sh, ry.f, ry.tr);
  ry.m_null = (D)drift<M>(null_error<M>(ry), (double)ry.ref.e_den);
  ry.m_q = (D)0.0;
  ry.lam = 0.0;
  S h = (S)P.h0;
  if (!P.rk4 && (double)h > P.h_max) h = (S)P.h_max;
  ry.h = h;
  ry.attempts = 0;
  ry.n_steps = 0;
  ry.n_rej = 0;
  ry.rejected_before = false;
  ry.state = classify<M>(P, ry, false);
}

// Step factor min(5, max(0.2, 0.9 en^(-1/5))), 5 for en = 0, capped at 1 after a rejection
// (numba_kernel.py:272-281), with pow in the working type (the reference modes).
template <class M>
__device__ __forceinline__ typename M::N step_factor(typename M::N en, bool rejected_before) {
  using N = typename M::N;
  N factor;
  if (en == (N)0.0) {
    factor = (N)FACTOR_MAX;
  } else {
    N raw;
    if constexpr (sizeof(N) == 4) {
      // float32 working precision: the power evaluated in double and rounded once to float,
      // i.e. the correctly rounded powf of the reference's float32 ** float32.
      raw = (N)SAFETY * (N)pow((double)en, (double)(N)ERROR_EXPONENT);
    } else {
      raw = (N)SAFETY * pow(en, (N)ERROR_EXPONENT);
    }
    factor = py_min((N)FACTOR_MAX, py_max((N)FACTOR_MIN, raw));
  }
  if (rejected_before) factor = py_min(factor, (N)1.0);
  return factor;
}

// The fast modes' step factor from en^2: 0.9 en^(-1/5) = 0.9 (en^2)^(-1/10), in single precision.
template <class M>
__device__ __forceinline__ typename M::N step_factor_sq(typename M::N en2, bool rejected_before) {
  using N = typename M::N;
  N factor = (N)FACTOR_MAX;
  if (en2 != (N)0.0) {
    float lg, ex;
    if constexpr (M::kMixed) {  // the bare hardware approximations (subnormals flush to zero): +1 %
      asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(lg) : "f"((float)en2));
      asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ex) : "f"(-0.1f * lg));
    } else {
      ex = exp2f(-0.1f * __log2f((float)en2));
    }
    const N raw = (N)(0.9f * ex);
    factor = py_min((N)FACTOR_MAX, py_max((N)FACTOR_MIN, raw));
  }
  if (rejected_before) factor = py_min(factor, (N)1.0);
  return factor;
}

// The stages of one step of size h from ry.y with FSAL stage ry.f (numba_kernel.py:201-257):
// the candidate state yn, k6 = f(yn) and, for DP5, the error sum sum_i E_i k_i.  The solution
// and error sums are accumulated in the reference's order of terms as soon as their stages are
// known (the same values, fewer stages held live).  With acc_rec, the stage-input sums acc_s
// (stage input = y + h * acc_s) are recorded for s = 1..6 (the adjoint rebuilds the stage
// inputs from them).
template <class M, bool RK4>
__device__ __forceinline__ void dp_stages_scalar(const Params& P, const Ray<M>& ry, typename M::K h, typename M::K k6[NV],
                                          typename M::S yn[NV], typename M::K esum[NV], Trig& tr,
                                          typename M::K (*acc_rec)[NV] = nullptr) {
  using K = typename M::K;
  const K* k0 = ry.f;
  auto c = [](double x) { return (K)x; };
  K acc[NV];
  auto store = [&](int s) {
#pragma unroll
    for (int i = 0; i < NV; ++i) acc_rec[s][i] = acc[i];
  };
  // Stage inputs: the reference's sums (same terms and order, zero coefficients skipped);
  // madd fuses them in the fast modes and rounds each operation in the reference modes.
  if constexpr (!RK4) {
    K k1[NV], k2[NV], k3[NV], k4[NV], k5[NV], bsum[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = c(dp::A10) * k0[i];
    if (acc_rec) store(0);
    M::template stage<false, 1>(P, ry, h, acc, k1, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = madd<M>(c(dp::A20) * k0[i], c(dp::A21), k1[i]);
    if (acc_rec) store(1);
    M::template stage<false, 2>(P, ry, h, acc, k2, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = madd<M>(madd<M>(c(dp::A30) * k0[i], c(dp::A31), k1[i]), c(dp::A32), k2[i]);
    if (acc_rec) store(2);
    M::template stage<false, 3>(P, ry, h, acc, k3, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const K a = madd<M>(c(dp::A40) * k0[i], c(dp::A41), k1[i]);
      acc[i] = madd<M>(madd<M>(a, c(dp::A42), k2[i]), c(dp::A43), k3[i]);
    }
    if (acc_rec) store(3);
    M::template stage<false, 4>(P, ry, h, acc, k4, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const K a = madd<M>(c(dp::A50) * k0[i], c(dp::A51), k1[i]);
      acc[i] = madd<M>(madd<M>(madd<M>(a, c(dp::A52), k2[i]), c(dp::A53), k3[i]), c(dp::A54), k4[i]);
      // b = (35/384, 0, 500/1113, 125/192, -2187/6784, 11/84) and E = b_hat - b through k4.
      bsum[i] = madd<M>(madd<M>(madd<M>(c(dp::B0) * k0[i], c(dp::B2), k2[i]), c(dp::B3), k3[i]), c(dp::B4), k4[i]);
      esum[i] = madd<M>(madd<M>(madd<M>(c(dp::E0) * k0[i], c(dp::E2), k2[i]), c(dp::E3), k3[i]), c(dp::E4), k4[i]);
    }
    if (acc_rec) store(4);
    M::template stage<false, 5>(P, ry, h, acc, k5, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      acc[i] = madd<M>(bsum[i], c(dp::B5), k5[i]);
      esum[i] = madd<M>(esum[i], c(dp::E5), k5[i]);
    }
    if (acc_rec) store(5);
    M::template stage<true, 6>(P, ry, h, acc, k6, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) esum[i] = madd<M>(esum[i], c(dp::E6), k6[i]);
  } else {
    K k1[NV], k2[NV], k3[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = c(0.5) * k0[i];
    if (acc_rec) store(0);
    M::template stage<false, 1>(P, ry, h, acc, k1, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = c(0.5) * k1[i];
    if (acc_rec) store(1);
    M::template stage<false, 2>(P, ry, h, acc, k2, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = c(1.0) * k2[i];
    if (acc_rec) store(2);
    M::template stage<false, 3>(P, ry, h, acc, k3, tr, yn);
#pragma unroll
    for (int i = 0; i < NV; ++i)
      acc[i] = madd<M>(madd<M>(madd<M>(c(dp::RK4_B0) * k0[i], c(dp::RK4_B1), k1[i]), c(dp::RK4_B2), k2[i]),
                       c(dp::RK4_B3), k3[i]);
    if (acc_rec) store(5);
    M::template stage<true, 6>(P, ry, h, acc, k6, tr, yn);
  }
}

// The mixed mode's stages on packed FP32 pairs.  sm_100 executes two FP32 multiply-adds in one
// instruction (fma.rn.f32x2); with the components paired as (r, theta), (p_r, p_theta) and
// (t, phi), each stage sum takes one packed operation per pair where the scalar form takes
// two.  Every lane rounds exactly like the scalar operation and the sums keep the reference's
// order of terms, so the values are those of the scalar form.  Only the pairs the right-hand
// side reads are formed for the inner stages; (t, phi) enters the solution and error sums.
__device__ __forceinline__ float2 mul2(float a, float2 x) { return __fmul2_rn(make_float2(a, a), x); }
__device__ __forceinline__ float2 madd2(float2 acc, float a, float2 x) { return __ffma2_rn(make_float2(a, a), x, acc); }

template <class M>
__device__ __forceinline__ void dp_stages_mixed(const Params& P, const Ray<M>& ry, float h, float k6[NV],
                                                double yn[NV], float esum[NV]) {
  auto c = [](double x) { return (float)x; };
  const Mixed::Shadow& sh = ry.sh;
  float2 k0[3], k1[3], k2[3], k3[3], k4[3], k5[3], kl[3], acc[3], bs[3], es[3];
  k0[0] = make_float2(ry.f[CR], ry.f[CTH]);
  k0[1] = make_float2(ry.f[CPR], ry.f[CPTH]);
  k0[2] = make_float2(ry.f[CT], ry.f[CPH]);
#pragma unroll
  for (int j = 0; j < 2; ++j) acc[j] = mul2(c(dp::A10), k0[j]);
  Mixed::stage(P, sh, h, 0.2f, acc, k1);
#pragma unroll
  for (int j = 0; j < 2; ++j) acc[j] = madd2(mul2(c(dp::A20), k0[j]), c(dp::A21), k1[j]);
  Mixed::stage(P, sh, h, 0.3f, acc, k2);
#pragma unroll
  for (int j = 0; j < 2; ++j) acc[j] = madd2(madd2(mul2(c(dp::A30), k0[j]), c(dp::A31), k1[j]), c(dp::A32), k2[j]);
  Mixed::stage(P, sh, h, 0.8f, acc, k3);
#pragma unroll
  for (int j = 0; j < 2; ++j)
    acc[j] = madd2(madd2(madd2(mul2(c(dp::A40), k0[j]), c(dp::A41), k1[j]), c(dp::A42), k2[j]), c(dp::A43), k3[j]);
  Mixed::stage(P, sh, h, c(8.0 / 9.0), acc, k4);
#pragma unroll
  for (int j = 0; j < 2; ++j)
    acc[j] = madd2(madd2(madd2(madd2(mul2(c(dp::A50), k0[j]), c(dp::A51), k1[j]), c(dp::A52), k2[j]), c(dp::A53), k3[j]),
                   c(dp::A54), k4[j]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    bs[j] = madd2(madd2(madd2(mul2(c(dp::B0), k0[j]), c(dp::B2), k2[j]), c(dp::B3), k3[j]), c(dp::B4), k4[j]);
    es[j] = madd2(madd2(madd2(mul2(c(dp::E0), k0[j]), c(dp::E2), k2[j]), c(dp::E3), k3[j]), c(dp::E4), k4[j]);
  }
  Mixed::stage(P, sh, h, 1.0f, acc, k5);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    acc[j] = madd2(bs[j], c(dp::B5), k5[j]);
    es[j] = madd2(es[j], c(dp::E5), k5[j]);
  }
  float dev6;
  Mixed::stage(P, sh, h, 1.0f, acc, kl, &dev6);
  float2 ha[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    es[j] = madd2(es[j], c(dp::E6), kl[j]);
    ha[j] = mul2(h, acc[j]);
  }
  // The candidate: h * acc rounded in FP32, accumulated into the FP64 state; t adds h E in FP64
  // beside h times its stages' deviations from E (the weights b sum to 1).
  yn[CR] = sh.far ? ry.y[CR] + fma((double)h, ry.y[CPR], (double)ha[0].x) : ry.y[CR] + (double)ha[0].x;
  yn[CTH] = ry.y[CTH] + (double)ha[0].y;
  yn[CPR] = ry.y[CPR] + (double)ha[1].x;
  yn[CPTH] = ry.y[CPTH] + (double)ha[1].y;
  yn[CT] = ry.y[CT] + fma((double)h, -ry.pt, (double)ha[2].x);
  yn[CPH] = ry.y[CPH] + (double)ha[2].y;
  k6[CR] = sh.far ? dev6 : kl[0].x;  // the candidate's deviation from its own p_r, or dr/dlambda
  k6[CTH] = kl[0].y;
  k6[CPR] = kl[1].x;
  k6[CPTH] = kl[1].y;
  k6[CT] = kl[2].x;
  k6[CPH] = kl[2].y;
  esum[CR] = es[0].x;
  esum[CTH] = es[0].y;
  esum[CPR] = es[1].x;
  esum[CPTH] = es[1].y;
  esum[CT] = es[2].x;
  esum[CPH] = es[2].y;
}

template <class M, bool RK4>
__device__ __forceinline__ void dp_stages(const Params& P, const Ray<M>& ry, typename M::K h, typename M::K k6[NV],
                                          typename M::S yn[NV], typename M::K esum[NV], Trig& tr,
                                          typename M::K (*acc_rec)[NV] = nullptr) {
  if constexpr (M::kMixed) {
    static_assert(!RK4, "the mixed mode integrates with Dormand-Prince 5(4) only");
    dp_stages_mixed<M>(P, ry, h, k6, yn, esum);
  } else {
    dp_stages_scalar<M, RK4>(P, ry, h, k6, yn, esum, tr, acc_rec);
  }
}

// One step attempt (numba_kernel.py:376-455): DP5(4) (or RK4) step, error norm, controller,
// accept/reject, diagnostics and classification.  Returns with ry.state updated.
template <class M, bool RK4>
__device__ __forceinline__ void attempt(const Params& P, Ray<M>& ry, double* __restrict__ event_y,
                                        unsigned char* __restrict__ event_hit) {
  using S = typename M::S;
  using K = typename M::K;
  using N = typename M::N;
  ry.attempts += 1;
  if (ry.attempts > P.guard) {  // defensive guard (integrators.py:151-162)
    ry.state = FAILURE;
    return;
  }
  const double remaining = P.lambda_max - ry.lam;
  const bool last = (double)ry.h >= remaining;
  const S h_eff = last ? (S)remaining : ry.h;
  const K h = (K)h_eff;
  K k6[NV], esum[NV];
  S yn[NV];
  Trig tr;
  dp_stages<M, RK4>(P, ry, h, k6, yn, esum, tr);
  // The candidate and k6 must be finite (numba_kernel.py:394-395).  In the fast DP5 modes the
  // error norm decides it: every stage k_j except k1 enters sum E_j k_j (E_1 = 0, and k1 only
  // feeds the later stages), yn derives from the same stages, and a non-finite yn makes its
  // scale's Newton reciprocal NaN, so total is finite exactly when yn and k6 are.
  bool finite = true;
  if constexpr (RK4 || !M::kFused) {
#pragma unroll
    for (int i = 0; i < NV; ++i) finite = finite && finite_(yn[i]) && finite_(k6[i]);
  }
  bool accept = finite;
  S h_new = ry.h;
  if constexpr (!RK4) {
    if (finite) {
      // HNW scaled RMS norm, pairwise order ((q0+q1)+(q2+q3))+((q4+q5)+(q6+q7)) with the two
      // constant components contributing exact zeros (numba_kernel.py:261-268).  The fast
      // modes multiply by a Newton reciprocal of the scale and compare en^2 = total / 8 with 1
      // instead of taking the square root (the step factor is a power of en^2 as well).
      N q[NV];
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const K e = h * esum[i];
        const N scale = madd<M>((N)P.atol, (N)P.rtol, py_max((N)fabs(ry.y[i]), (N)fabs(yn[i])));
        N v;
        if constexpr (M::kFused) v = (N)e * rcp_newton<1>(scale);
        else v = (N)e / scale;
        q[i] = v * v;
      }
      // Full-state slots: 0 t, 1 r, 2 th, 3 ph, 4 p_t (0), 5 p_r, 6 p_th, 7 p_phi (0).
      const N total = ((q[CT] + q[CR]) + (q[CTH] + q[CPH])) + (q[CPR] + q[CPTH]);
      if constexpr (M::kFused) {
        if (!M::kSaturate && !finite_(total)) {
          finite = false;
          accept = false;
        } else {
          const N en2 = total * (N)0.125;
          accept = en2 <= (N)1.0;
          const N factor = step_factor_sq<M>(en2, ry.rejected_before);
          if (!(accept && last)) {
            h_new = (S)((N)h_eff * factor);
            if ((double)h_new > P.h_max) h_new = (S)P.h_max;
          }
        }
      } else {
        const N en = sqrt(total / (N)8.0);
        if (!finite_(en)) {
          finite = false;
          accept = false;
        } else {
          accept = en <= (N)1.0;
          const N factor = step_factor<M>(en, ry.rejected_before);
          if (!(accept && last)) {
            h_new = (S)((N)h_eff * factor);
            if ((double)h_new > P.h_max) h_new = (S)P.h_max;
          }
        }
      }
    }
  }
  if (!finite) {
    ry.state = FAILURE;
    return;
  }
  const bool rejected = !accept;
  if (rejected) ry.n_rej += 1;
  ry.rejected_before = rejected;
  ry.h = h_new;
  if (rejected) {
    if (h_new < (S)P.h_min) ry.state = FAILURE;
    return;
  }
  S y_prev_th = ry.y[CTH];
  S y_prev[NV];
  if (P.disk) {
#pragma unroll
    for (int i = 0; i < NV; ++i) y_prev[i] = ry.y[i];
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    ry.y[i] = yn[i];
    ry.f[i] = k6[i];
  }
  ry.tr = M::accept_trig((double)ry.y[CTH], tr);
  if constexpr (M::kMixed) {
    const bool far_old = ry.sh.far;
    M::accepted(P, ry.y, ry.sh, ry.tr);
    Mixed::rebase_fsal(far_old, ry.sh, ry.f);
  } else {
    M::accepted(P, ry.y, ry.sh, ry.tr);
  }
  const double lam_old = ry.lam;
  ry.lam = last ? P.lambda_max : ry.lam + (double)h_eff;
  ry.n_steps += 1;
  ry.h_taken = h_eff;
  // E and L_z drifts are identically zero (p_t, p_phi never change); Q and the null error:
  using D = typename M::D;
  ry.m_q = py_max(ry.m_q, (D)drift<M>(fabs(carter<M>(P, ry) - ry.ref.q0), (double)ry.ref.q_den));
  ry.m_null = py_max(ry.m_null, (D)drift<M>(null_error<M>(ry), (double)ry.ref.e_den));
  int code = classify<M>(P, ry, true, false);
  if (P.disk) {  // disk-plane event, numba_kernel.py:439-454
    const double half_pi = 0.5 * PI;
    const double th_old = (double)y_prev_th;
    const double th_new = (double)ry.y[CTH];
    if ((th_old - half_pi) * (th_new - half_pi) < 0.0) {
      const double s = (half_pi - th_old) / (th_new - th_old);
      S ev[NV];
#pragma unroll
      for (int i = 0; i < NV; ++i) ev[i] = y_prev[i] + (S)(s * (double)(ry.y[i] - y_prev[i]));
      ev[CTH] = (S)half_pi;
      if (ev[CR] >= (S)P.r_in && ev[CR] <= (S)P.r_out) {
#pragma unroll
        for (int i = 0; i < NV; ++i) ry.y[i] = ev[i];
        if (event_y) {
          event_y[0] = (double)ev[CT];
          event_y[1] = (double)ev[CR];
          event_y[2] = (double)ev[CTH];
          event_y[3] = (double)ev[CPH];
          event_y[4] = (double)ry.pt;
          event_y[5] = (double)ev[CPR];
          event_y[6] = (double)ev[CPTH];
          event_y[7] = (double)ry.pph;
        }
        if (event_hit) *event_hit = 1;
        ry.lam = lam_old + s * (double)h_eff;
        code = DISK_HIT;
      }
    }
  }
  ry.state = code;
}

// Null Carter constant of an initial 8-state with the sin^2/cos^2 form of
// photons/constants.py:75-90 (the conservation reference Q0).
__device__ __forceinline__ double carter_initial(const Params& P, const double y0[8]) {
  const double th = y0[2], p_th = y0[6], lz = y0[7], e = -y0[4];
  const double s = sin(th);
  const double c = cos(th);
  const double s2 = s * s;
  double lz2_over_s2 = 0.0;
  if (lz != 0.0) lz2_over_s2 = (lz * lz) / s2;
  return p_th * p_th + (c * c) * (lz2_over_s2 - P.a2 * e * e);
}

// Output arrays of a batch (device pointers; any may be null except Y and state).
struct Outputs {
  double* Y;            // (N, 8)
  long long* state;     // (N,)
  long long* n_steps;   // (N,)
  long long* n_rej;     // (N,)
  double* lam;          // (N,)
  double* max_null;     // (N,)
  double* max_e;        // (N,)  identically zero (E is exact here)
  double* max_lz;       // (N,)  identically zero (L_z is exact here)
  double* max_q;        // (N,)
  double* event_Y;      // (N, 8) or null
  unsigned char* event_hit;  // (N,) or null
};

template <class M>
__device__ __forceinline__ void ray_store(const Ray<M>& ry, const Outputs& o, long long n) {
  double* Y = o.Y + n * 8;
  Y[0] = (double)ry.y[CT];
  Y[1] = (double)ry.y[CR];
  Y[2] = (double)ry.y[CTH];
  Y[3] = (double)ry.y[CPH];
  Y[4] = (double)ry.pt;
  Y[5] = (double)ry.y[CPR];
  Y[6] = (double)ry.y[CPTH];
  Y[7] = (double)ry.pph;
  o.state[n] = ry.state;
  if (o.n_steps) o.n_steps[n] = ry.n_steps;
  if (o.n_rej) o.n_rej[n] = ry.n_rej;
  if (o.lam) o.lam[n] = ry.lam;
  if (o.max_null) o.max_null[n] = (double)ry.m_null;
  if (o.max_e) o.max_e[n] = 0.0;
  if (o.max_lz) o.max_lz[n] = 0.0;
  if (o.max_q) o.max_q[n] = (double)ry.m_q;
}

}  // namespace krr
