// Adjoint of the discretised Dormand-Prince 5(4) map: derivatives of a ray's terminal celestial
// direction with respect to (alpha, beta, spin, inclination).
//
// For each ray (one thread):
//   1. the camera state y0 and its Jacobian d y0 / d(alpha, beta, a, theta_o) by forward-mode
//      dual numbers through the camera (raytracing/camera.py:225-381);
//   2. the forward integration in FP64 (the Fast64 arithmetic and the reference's controller),
//      recording every accepted step size and the state every K accepted steps (checkpoints);
//   3. the output: theta and phi at the termination surface r_s (the escape radius, or the
//      capture radius r_plus + epsilon). The last accepted step is replaced by the DP5 step
//      from the previous state whose length lands on r_s (Newton on the step length; it is
//      recorded like any other step), then the remaining residual is removed by one linear
//      step along the flow: x_e = x_N - (f_x / f_r)(r_N - r_s) (the event-time correction:
//      d lambda_e = -d r / f_r, exact to first order since x_e is stationary in the landing
//      step's length);
//   4. the reverse sweep over the recorded step sequence with the controller held fixed: each
//      K-step segment is recomputed from its checkpoint, then the adjoint of each DP5 step runs
//      back through its six stages; the right-hand side's vector-Jacobian product is the
//      hand-written reverse-mode derivative of the separated right-hand side the steps evaluate;
//   5. the chain through the camera Jacobian.
// Both outputs (theta_e, phi_e) are swept together (two cotangent rows).
//
// Steps 1 (its values), 2 and 3 run in k_lensing_forward, which writes each ray's landed final
// state to the workspace; steps 1 (its Jacobian), 4 and 5 in k_lensing_reverse. Two kernels
// instead of one keep each within the instruction cache and give each its own register budget:
// the forward pass is the fast64 step loop, the reverse sweep holds the stage cotangents.
#include <cuda_runtime.h>

#include "krr_device.cuh"
#include "krr_dual.cuh"
#include "krr_launch.h"
#include <math_constants.h>

namespace krr {

namespace {

constexpr int NC = 2;     // cotangent rows: theta_e, phi_e
constexpr int NX = NV + 2;  // adjoint state: the six integrated components, p_t, p_phi
constexpr int XPT = NV, XPPH = NV + 1;

// d(v . f)/d(state, a) at (r, theta, p_t, p_r, p_theta, p_phi) for NC cotangents v (each over
// the six integrated components of f); accumulates into xbar and abar.  f is the right-hand
// side in Carter's separated form, the one the forward steps evaluate (Fast64::rhs_sc):
//   Delta = r^2 - 2Mr + a^2, Sigma = r^2 + a^2 - a^2 sin^2, K = (r^2 + a^2) E - a L,
//   v = L / sin - a E sin, B = v^2 - K^2 / Delta + Delta p_r^2 + p_theta^2  (2 H = B / Sigma),
//   f_t = (a sin v + (r^2 + a^2) K / Delta) / Sigma,  f_r = Delta p_r / Sigma,
//   f_theta = p_theta / Sigma,  f_phi = (a K / Delta + L / sin^2 - a E) / Sigma,
//   f_pr = (r B / Sigma - (r - M) p_r^2 - (K / Delta)((K / Delta)(r - M) - 2 E r)) / Sigma,
//   f_ptheta = cos (v (L / sin^2 + a E) - a^2 sin B / Sigma) / Sigma,
// with E = -p_t, L = p_phi (1 / sin dropped for L = 0, the axis guard).  The product is taken by
// reverse-mode differentiation of that evaluation, written out by hand: the forward values once,
// then each intermediate's adjoint for both cotangent rows.  Out of line: the reverse sweep
// calls it seven times per step.
__device__ __noinline__ void rhs_vjp(double m, double a, double r, double th, double pt, double pr, double pth, double pph,
                        const double v_[NC][NV], double xbar[NC][NX], double abar[NC]) {
  // The translation unit rounds every product and sum separately (-fmad=false); the products
  // accumulated here are fused explicitly (fma), which this derivative needs for no bit pattern.
  double s, c;
  sincos(th, &s, &c);
  const double E = -pt, L = pph, ae = a * E;
  const double dlt = fma(r, r - 2.0 * m, a * a), r2a2 = fma(r, r, a * a);
  const double as = a * s, a2s = a * as;
  const double K = fma(r2a2, E, -a * L);
  const double isig = 1.0 / fma(-a2s, s, r2a2);
  const double iD = 1.0 / dlt;
  const double kd = K * iD;
  const bool axis = L == 0.0;
  const double is = axis ? 0.0 : 1.0 / s;
  const double lis = L * is;
  const double v = fma(-ae, s, lis);
  const double rm = r - m, pr2 = pr * pr;
  const double B = fma(v, v, fma(-K, kd, fma(dlt, pr2, pth * pth)));
  const double bs = B * isig;
  const double T1 = fma(as, v, kd * r2a2);
  const double T2 = fma(a, kd, fma(lis, is, -ae));
  const double T5 = fma(kd, rm, -2.0 * E * r);
  const double T4 = fma(rm, pr2, kd * T5);
  const double T3 = fma(r, bs, -T4);
  const double T7 = fma(lis, is, ae);
  const double T6 = fma(v, T7, -a2s * bs);
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const double wt = v_[q][CT], wr = v_[q][CR], wth = v_[q][CTH], wph = v_[q][CPH], wpr = v_[q][CPR],
                 wpth = v_[q][CPTH];
    double u_isig = fma(wt, T1, fma(wr * dlt, pr, fma(wth, pth, fma(wph, T2, fma(wpr, T3, wpth * c * T6)))));
    const double uT1 = wt * isig, uT2 = wph * isig, uT3 = wpr * isig, uT6 = wpth * isig * c;
    const double u_c = wpth * isig * T6;
    double u_as = uT1 * v;
    double u_v = fma(uT1, as, uT6 * T7);
    double u_kd = fma(uT1, r2a2, uT2 * a);
    double u_r2a2 = uT1 * kd;
    double u_D = wr * pr * isig;
    double u_pr = wr * dlt * isig;
    double u_pth = wth * isig;
    double u_a = uT2 * kd;
    double u_lis = uT2 * is;
    double u_is = uT2 * lis;
    double u_ae = -uT2;
    double u_r = uT3 * bs;
    double u_bs = uT3 * r;
    const double uT4 = -uT3;
    double u_rm = uT4 * pr2;
    double u_pr2 = uT4 * rm;
    u_kd = fma(uT4, T5, u_kd);
    const double uT5 = uT4 * kd;
    u_kd = fma(uT5, rm, u_kd);
    u_rm = fma(uT5, kd, u_rm);
    double u_E = -2.0 * r * uT5;
    u_r = fma(-2.0 * E, uT5, u_r);
    const double uT7 = uT6 * v;
    double u_a2s = -uT6 * bs;
    u_bs = fma(-uT6, a2s, u_bs);
    u_lis = fma(uT7, is, u_lis);
    u_is = fma(uT7, lis, u_is);
    u_ae += uT7;
    const double u_B = u_bs * isig;
    u_isig = fma(u_bs, B, u_isig);
    u_v = fma(2.0 * v, u_B, u_v);
    double u_K = -u_B * kd;
    u_kd = fma(-u_B, K, u_kd);
    u_D = fma(u_B, pr2, u_D);
    u_pr2 = fma(u_B, dlt, u_pr2);
    u_pth = fma(2.0 * pth, u_B, u_pth);
    u_pr = fma(2.0 * pr, u_pr2, u_pr);
    u_r += u_rm;
    u_lis += u_v;
    u_ae = fma(-u_v, s, u_ae);
    double u_s = -u_v * ae;
    double u_L = u_lis * is;
    u_is = fma(u_lis, L, u_is);
    if (!axis) u_s = fma(-u_is * is, is, u_s);
    u_K = fma(u_kd, iD, u_K);
    u_D = fma(-u_kd * K, iD * iD, u_D);
    const double u_S = -u_isig * isig * isig;
    u_r2a2 += u_S;
    u_a2s = fma(-u_S, s, u_a2s);
    u_s = fma(-u_S, a2s, u_s);
    u_r2a2 = fma(u_K, E, u_r2a2);
    u_E = fma(u_K, r2a2, u_E);
    u_a = fma(-u_K, L, u_a);
    u_L = fma(-u_K, a, u_L);
    u_a = fma(u_a2s, as, u_a);
    u_as = fma(u_a2s, a, u_as);
    u_a = fma(u_as, s, u_a);
    u_s = fma(u_as, a, u_s);
    u_a = fma(u_ae, E, u_a);
    u_E = fma(u_ae, a, u_E);
    u_r = fma(2.0 * r, u_r2a2, u_r);
    u_a = fma(2.0 * a, u_r2a2, u_a);
    u_r = fma(2.0 * rm, u_D, u_r);
    u_a = fma(2.0 * a, u_D, u_a);
    xbar[q][CR] += u_r;
    xbar[q][CTH] += fma(u_s, c, -u_c * s);
    xbar[q][CPR] += u_pr;
    xbar[q][CPTH] += u_pth;
    xbar[q][XPT] -= u_E;
    xbar[q][XPPH] += u_L;
    abar[q] += u_a;
  }
}

// Stage coefficients of the Dormand-Prince 5(4) map in the 1..6 numbering of its new stages:
// stage input s (s = 1..5) uses a[s][j] for j < s; the new state uses b[j].
__device__ __forceinline__ double dp_a(int s, int j) {
  const double A[6][6] = {
      {dp::A10, 0, 0, 0, 0, 0},
      {dp::A20, dp::A21, 0, 0, 0, 0},
      {dp::A30, dp::A31, dp::A32, 0, 0, 0},
      {dp::A40, dp::A41, dp::A42, dp::A43, 0, 0},
      {dp::A50, dp::A51, dp::A52, dp::A53, dp::A54, 0},
      {dp::B0, 0.0, dp::B2, dp::B3, dp::B4, dp::B5},
  };
  return A[s][j];
}

struct LensArgs {
  Params P;  // integrator/termination parameters (spin and mass included)
  double spin, mass, r_o, th_o, ph_o;
  int K;    // checkpoint interval (accepted steps)
  int cap;  // tape capacity (accepted steps per ray)
  const double* alpha;
  const double* beta;
  long long n;
  double* theta;
  double* phi;
  double* jac;  // (n, 2, 4): rows theta_e, phi_e; columns alpha, beta, spin, theta_o (rad)
  long long* state;
  long long* n_steps;
  int* status;  // 0 ok, 1 tape full, 2 ended neither ESCAPED nor CAPTURED
  double* tape_h;   // (n, cap)
  double* tape_ck;  // (n, cap / K + 1, NV)
  double* final_rec;  // (n, FINAL_REC): the landed final state y, f = f(y), p_t, p_phi
};

constexpr int FINAL_REC = 16;  // y[NV], f[NV], p_t, p_phi, two unused

__device__ __forceinline__ double surface_radius(const Params& P, int state) {
  return state == ESCAPED ? P.r_escape : P.r_capture;
}

// One fixed step of size h from (y, f = f(y)): the forward map the adjoint differentiates; with
// recorded stage sums for the reverse pass.
__device__ __forceinline__ void fixed_step(const Params& P, Ray<Fast64>& ry, double h, double acc[6][NV],
                                           double k[6][NV]) {
  double yn[NV], esum[NV];
  Trig tr;
  dp_stages<Fast64, false>(P, ry, h, k[5], yn, esum, tr, acc);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    ry.y[i] = yn[i];
    ry.f[i] = k[5][i];
  }
  ry.tr = tr;  // sin and cos at the new state: the next step's stages shift from them
}

// Replaces the last accepted step (y_prev -> ry, length h_last) by the DP5 step from y_prev
// that ends on r = rs: Newton on the step length, r(Phi(y_prev, h)) = rs with dr/dh = f_r at
// the step's end, three iterations from the linear estimate h_last - (r_N - rs) / f_r(y_N).
// The last step otherwise overshoots the surface by up to tens of M, and the output's
// linear projection back to rs then carries a second-order residual (theta'' dr^2 / 2, about
// 1e-5 rad at r = 1000) whose parameter derivative is not that of the crossing point. The
// accepted step is kept when an iterate leaves (0, h_last] or is not finite.
__device__ void land_on_surface(const Params& P, Ray<Fast64>& ry, const double y_prev[NV], double rs,
                                double& h_last) {
  double h = h_last - (ry.y[CR] - rs) / ry.f[CR];
  double acc[6][NV], k[6][NV];
  Ray<Fast64> st = ry;
  for (int it = 0; it <= 3; ++it) {
    if (!(isfinite(h) && h / h_last > 0.0 && h / h_last <= 1.0)) return;
#pragma unroll
    for (int i = 0; i < NV; ++i) st.y[i] = y_prev[i];
    Fast64::init_rhs(P, st.y, st.pt, st.pph, st.sh, st.f, st.tr);
    fixed_step(P, st, h, acc, k);
    if (it < 3) h -= (st.y[CR] - rs) / st.f[CR];
  }
#pragma unroll
  for (int i = 0; i < NV; ++i)
    if (!isfinite(st.y[i]) || !isfinite(st.f[i])) return;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    ry.y[i] = st.y[i];
    ry.f[i] = st.f[i];
  }
  h_last = h;
}

// Forward pass: camera, the integration with the reference controller recording the tape,
// the landing on the termination surface, the map's value, and the landed final state.
__global__ void __launch_bounds__(128, 3) k_lensing_forward(LensArgs A) {
  const long long ray = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n) return;
  const Params& P = A.P;
  double y0[8];
  camera_state_t<double>(A.alpha[ray], A.beta[ray], A.P.a, A.th_o, A.r_o, A.ph_o, A.mass, y0);
  double* tape_h = A.tape_h + ray * (long long)A.cap;
  const int n_ck = A.cap / A.K + 1;
  double* tape_ck = A.tape_ck + ray * (long long)n_ck * NV;
  Ray<Fast64> ry;
  ray_init<Fast64>(P, y0, carter_initial(P, y0), ry);
#pragma unroll
  for (int i = 0; i < NV; ++i) tape_ck[i] = ry.y[i];
  int status = 0;
  double y_prev[NV] = {};  // the state before the last accepted step
  while (ry.state == RUNNING) {
    const int before = ry.n_steps;
    double y_cur[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) y_cur[i] = ry.y[i];
    attempt<Fast64, false>(P, ry, nullptr, nullptr);
    if (ry.n_steps != before) {
      const int n = ry.n_steps;
      if (n > A.cap) {
        status = 1;
        break;
      }
#pragma unroll
      for (int i = 0; i < NV; ++i) y_prev[i] = y_cur[i];
      tape_h[n - 1] = ry.h_taken;
      if (n % A.K == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) tape_ck[(n / A.K) * NV + i] = ry.y[i];
      }
    }
  }
  const int N = ry.n_steps;
  A.state[ray] = ry.state;
  A.n_steps[ray] = N;
  if (status == 0 && ry.state != ESCAPED && ry.state != CAPTURED) status = 2;
  const double rs = surface_radius(P, ry.state);
  if (status == 0 && N > 0) land_on_surface(P, ry, y_prev, rs, tape_h[N - 1]);
  // 3. the output at the termination surface (event-time correction)
  const double dr = ry.y[CR] - rs;
  const double fr = ry.f[CR];
  A.theta[ray] = ry.y[CTH] - ry.f[CTH] / fr * dr;
  A.phi[ray] = ry.y[CPH] - ry.f[CPH] / fr * dr;
  A.status[ray] = status;
  double* rec = A.final_rec + ray * FINAL_REC;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    rec[i] = ry.y[i];
    rec[NV + i] = ry.f[i];
  }
  rec[2 * NV] = ry.pt;
  rec[2 * NV + 1] = ry.pph;
}

// Reverse pass: the cotangents of the landed output, the checkpointed reverse sweep over the
// recorded steps, and the chain through the camera's Jacobian.
#ifndef KRR_LENS_REVERSE_MINB
#define KRR_LENS_REVERSE_MINB 1  // resident blocks per SM the reverse kernel's registers allow for
#endif
__global__ void __launch_bounds__(128, KRR_LENS_REVERSE_MINB) k_lensing_reverse(LensArgs A) {
  const long long ray = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n) return;
  double* J = A.jac + ray * 8;
  if (A.status[ray] != 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) J[i] = CUDART_NAN;
    return;
  }
  const Params& P = A.P;
  const double m = A.mass, a = A.P.a;
  const int N = (int)A.n_steps[ray];
  const int state = (int)A.state[ray];
  const double rs = surface_radius(P, state);
  const double* tape_h = A.tape_h + ray * (long long)A.cap;
  const int n_ck = A.cap / A.K + 1;
  const double* tape_ck = A.tape_ck + ray * (long long)n_ck * NV;
  const double* rec = A.final_rec + ray * FINAL_REC;
  double yN[NV], fN[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    yN[i] = rec[i];
    fN[i] = rec[NV + i];
  }
  Ray<Fast64> ry{};  // carries the constants p_t, p_phi into the recomputed steps
  ry.pt = rec[2 * NV];
  ry.pph = rec[2 * NV + 1];
  // 3'. the cotangents of the output x_e = x_N - (f_x / f_r)(r_N - r_s)
  const double dr = yN[CR] - rs;
  const double fr = fN[CR];
  const int out_comp[NC] = {CTH, CPH};
  double xbar[NC][NX];
  double abar[NC] = {0.0, 0.0};
  {
    double v[NC][NV];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int i = 0; i < NX; ++i) xbar[c][i] = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) v[c][i] = 0.0;
      const double fx = fN[out_comp[c]];
      xbar[c][out_comp[c]] = 1.0;
      xbar[c][CR] -= fx / fr;
      v[c][out_comp[c]] = -dr / fr;
      v[c][CR] = dr * fx / (fr * fr);
    }
    rhs_vjp(m, a, yN[CR], yN[CTH], ry.pt, yN[CPR], yN[CPTH], ry.pph, v, xbar, abar);
    if (state == CAPTURED) {  // r_s = r_plus(a) + epsilon moves with a
      const double drp_da = -a / sqrt(m * m - a * a);
#pragma unroll
      for (int c = 0; c < NC; ++c) abar[c] += fN[out_comp[c]] / fr * drp_da;
    }
  }
  // 4. reverse sweep, segment by segment from the last
  // The segment's states (K <= 64): r, theta, p_r, p_theta only -- t and phi do not enter the
  // right-hand side, so the recomputed steps and the stage inputs need neither.
  constexpr int NS = 4;
  double seg[64][NS];
  auto seg_put = [&](int j, const double y[NV]) {
    seg[j][0] = y[CR];
    seg[j][1] = y[CTH];
    seg[j][2] = y[CPR];
    seg[j][3] = y[CPTH];
  };
  for (int c0 = (N - 1) / A.K; c0 >= 0; --c0) {
    const int n0 = c0 * A.K, n1 = min(N, n0 + A.K);
    Ray<Fast64> rs_ray = ry;
#pragma unroll
    for (int i = 0; i < NV; ++i) rs_ray.y[i] = tape_ck[c0 * NV + i];
    Fast64::init_rhs(P, rs_ray.y, rs_ray.pt, rs_ray.pph, rs_ray.sh, rs_ray.f, rs_ray.tr);
    double acc[6][NV], k[6][NV];
    for (int n = n0; n < n1; ++n) {
      seg_put(n - n0, rs_ray.y);
      if (n + 1 < n1) fixed_step(P, rs_ray, tape_h[n], acc, k);
    }
    for (int n = n1 - 1; n >= n0; --n) {
      const double h = tape_h[n];
      Ray<Fast64> st = ry;
      st.y[CT] = 0.0;
      st.y[CPH] = 0.0;
      st.y[CR] = seg[n - n0][0];
      st.y[CTH] = seg[n - n0][1];
      st.y[CPR] = seg[n - n0][2];
      st.y[CPTH] = seg[n - n0][3];
      Fast64::init_rhs(P, st.y, st.pt, st.pph, st.sh, st.f, st.tr);
      fixed_step(P, st, h, acc, k);
      // Reverse of: Y_s = y + h acc_s (s = 1..5 -> k_s = f(Y_s)); y_new = y + h acc_6; the
      // stage-s sums are linear in k_0 = f(y) and k_1..k_{s-1} with the tableau weights.
      double kbar[NC][6][NV];  // cotangents of k_0..k_5 (k_0 = f(y), k_s = f(Y_s))
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < 6; ++j)
#pragma unroll
          for (int i = 0; i < NV; ++i) kbar[c][j][i] = (h * dp_a(5, j)) * xbar[c][i];
      for (int s = 5; s >= 1; --s) {  // stage inputs Y_s, s = 5..1, produced k_s
        double v[NC][NV], ybar_s[NC][NX];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
#pragma unroll
          for (int i = 0; i < NV; ++i) v[c][i] = kbar[c][s][i];
#pragma unroll
          for (int i = 0; i < NX; ++i) ybar_s[c][i] = 0.0;
        }
        const int sm = s - 1;  // acc index of stage input s
        // The stage input exactly as the forward formed it (upd<Fast64>: one fused step).
        const double Yr = fma(h, acc[sm][CR], seg[n - n0][0]);
        const double Yth = fma(h, acc[sm][CTH], seg[n - n0][1]);
        const double Ypr = fma(h, acc[sm][CPR], seg[n - n0][2]);
        const double Ypth = fma(h, acc[sm][CPTH], seg[n - n0][3]);
        rhs_vjp(m, a, Yr, Yth, ry.pt, Ypr, Ypth, ry.pph, v, ybar_s, abar);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
#pragma unroll
          for (int i = 0; i < NX; ++i) xbar[c][i] += ybar_s[c][i];
          for (int j = 0; j < s; ++j) {
            const double w = h * dp_a(sm, j);
            if (w != 0.0) {
#pragma unroll
              for (int i = 0; i < NV; ++i) kbar[c][j][i] = fma(w, ybar_s[c][i], kbar[c][j][i]);
            }
          }
        }
      }
      {  // k_0 = f(y)
        double v[NC][NV];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int i = 0; i < NV; ++i) v[c][i] = kbar[c][0][i];
        rhs_vjp(m, a, seg[n - n0][0], seg[n - n0][1], ry.pt, seg[n - n0][2], seg[n - n0][3], ry.pph, v, xbar, abar);
      }
    }
  }
  // 1'. the camera state's Jacobian in (alpha, beta, a, theta_o) by dual numbers
  Dual<4> y0d[8];
  camera_state_t<Dual<4>>(Dual<4>::var(A.alpha[ray], 0), Dual<4>::var(A.beta[ray], 1), Dual<4>::var(a, 2),
                          Dual<4>::var(A.th_o, 3), A.r_o, A.ph_o, m, y0d);
  // 5. chain through the camera: d/d(alpha, beta, a, theta_o), then a = spin * M
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    double g[4] = {0.0, 0.0, 0.0, 0.0};
    const int map[8] = {CT, CR, CTH, CPH, XPT, CPR, CPTH, XPPH};  // 8-state slot -> adjoint slot
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double xb = xbar[c][map[i]];
#pragma unroll
      for (int p = 0; p < 4; ++p) g[p] = fma(xb, y0d[i].d[p], g[p]);
    }
    g[2] += abar[c];
    J[c * 4 + 0] = g[0];
    J[c * 4 + 1] = g[1];
    J[c * 4 + 2] = g[2] * m;
    J[c * 4 + 3] = g[3];
  }
}


// Replay: the same camera and the recorded step sequence without the controller (the map the
// adjoint differentiates), for finite-difference checks.
__global__ void __launch_bounds__(128) k_lensing_replay(LensArgs A) {
  const long long ray = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n) return;
  const Params& P = A.P;
  double y0[8];
  camera_state_t<double>(A.alpha[ray], A.beta[ray], A.P.a, A.th_o, A.r_o, A.ph_o, A.mass, y0);
  Ray<Fast64> ry;
  ray_init<Fast64>(P, y0, carter_initial(P, y0), ry);
  const long long N = A.n_steps[ray];
  const double* tape_h = A.tape_h + ray * (long long)A.cap;
  double acc[6][NV], k[6][NV];
  for (long long n = 0; n < N; ++n) fixed_step(P, ry, tape_h[n], acc, k);
  const int state = (int)A.state[ray];
  const double rs = surface_radius(P, state);
  const double dr = ry.y[CR] - rs;
  A.theta[ray] = ry.y[CTH] - ry.f[CTH] / ry.f[CR] * dr;
  A.phi[ray] = ry.y[CPH] - ry.f[CPH] / ry.f[CR] * dr;
  A.status[ray] = 0;
}

}  // namespace

cudaError_t lensing_adjoint(const LensLaunch& L, bool replay, cudaStream_t s) {
  if (L.n <= 0) return cudaSuccess;
  LensArgs A{};
  A.P = L.P;
  A.spin = L.spin;
  A.mass = L.mass;
  A.r_o = L.r_o;
  A.th_o = L.th_o;
  A.ph_o = L.ph_o;
  A.K = L.K;
  A.cap = L.cap;
  A.alpha = L.alpha;
  A.beta = L.beta;
  A.n = L.n;
  A.theta = L.theta;
  A.phi = L.phi;
  A.jac = L.jac;
  A.state = L.state;
  A.n_steps = L.n_steps;
  A.status = L.status;
  A.tape_h = L.tape_h;
  A.tape_ck = L.tape_ck;
  A.final_rec = L.final_rec;
  const int block = 128;
  const unsigned grid = (unsigned)((L.n + block - 1) / block);
  if (replay) {
    k_lensing_replay<<<grid, block, 0, s>>>(A);
    return cudaGetLastError();
  }
  k_lensing_forward<<<grid, block, 0, s>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_lensing_reverse<<<grid, block, 0, s>>>(A);
  return cudaGetLastError();
}

}  // namespace krr
