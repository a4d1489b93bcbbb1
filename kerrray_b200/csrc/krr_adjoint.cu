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
//   4. the reverse sweep over the recorded step sequence with the controller held fixed: the
//      adjoint of each DP5 step runs back through its six stages; the right-hand side's
//      vector-Jacobian product is the hand-written reverse-mode derivative of the separated
//      right-hand side the steps evaluate;
//   5. the chain through the camera Jacobian.
//
// The stage tape.  The forward pass also writes every accepted step's six stage inputs --
// (r, p_r, p_theta, sin theta, cos theta) of each, the values its right-hand sides were
// evaluated at, 240 B per step -- into a pool of 16-step chunks taken from the workspace by an
// atomic counter (a chunk table per ray).  Each thread builds the record of the step it is
// attempting in shared memory and, once the step is accepted, hands it to the bulk-copy engine
// as one 240 B copy (cp.async.bulk, shared to global): one instruction instead of thirty
// scattered 8 B stores, and nothing written for rejected attempts.  The reverse sweep of a ray whose chunks all fit
// (k_lensing_reverse_staged) reads them back and runs only the vector-Jacobian products, one
// thread per cotangent row (theta_e, phi_e), two threads per ray reading the same records.  A
// ray the pool could not hold is swept by k_lensing_reverse instead: each K-step segment
// recomputed from its checkpoint, both rows in one thread.
//
// Steps 1 (its values), 2 and 3 run in k_lensing_forward, which writes each ray's landed final
// state to the workspace; steps 1 (its Jacobian), 4 and 5 in the reverse kernels. Separate
// kernels keep each within the instruction cache and give each its own register budget.
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

// One cotangent row w = (w_r, w_theta, w_phi, w_pr, w_ptheta) of d(w . f)/d(r, theta, p_r,
// p_theta) into yb, and of d(w . f)/d(p_t, p_phi, a) into *pt_b, *pph_b, *a_b, at a stage input
// given by (r, p_r, p_theta) and the sine and cosine its right-hand side was evaluated with
// (Fast64::stage: the shifted pair for stages 1..5, sincos at accepted states).  The same
// separated form and reverse-mode evaluation as rhs_vjp, with its reciprocals taken like the
// forward's (rcp_fast).  The cotangent of f_t is zero on every call: neither output depends on
// t and f does not either, so no cotangent ever reaches the t slot, and its terms are left out.
__device__ __forceinline__ void rhs_vjp_row(double m, double a, double r, double s, double c, double pt, double pr,
                                            double pth, double pph, double wr, double wth, double wph, double wpr,
                                            double wpth, double yb[4], double* pt_b, double* pph_b, double* a_b) {
  const double E = -pt, L = pph, ae = a * E;
  const double dlt = fma(r, r - 2.0 * m, a * a), r2a2 = fma(r, r, a * a);
  const double as = a * s, a2s = a * as;
  const double K = fma(r2a2, E, -a * L);
  const double isig = rcp_fast(fma(-a2s, s, r2a2));
  const double iD = rcp_fast(dlt);
  const double kd = K * iD;
  const bool axis = L == 0.0;
  const double is = axis ? 0.0 : rcp_fast(s);
  const double lis = L * is;
  const double v = fma(-ae, s, lis);
  const double rm = r - m, pr2 = pr * pr;
  const double B = fma(v, v, fma(-K, kd, fma(dlt, pr2, pth * pth)));
  const double bs = B * isig;
  const double T2 = fma(a, kd, fma(lis, is, -ae));
  const double T5 = fma(kd, rm, -2.0 * E * r);
  const double T4 = fma(rm, pr2, kd * T5);
  const double T3 = fma(r, bs, -T4);
  const double T7 = fma(lis, is, ae);
  const double T6 = fma(v, T7, -a2s * bs);
  const double wpc = wpth * c;
  double u_isig = fma(wr * dlt, pr, fma(wth, pth, fma(wph, T2, fma(wpr, T3, wpc * T6))));
  const double uT2 = wph * isig, uT3 = wpr * isig, uT6 = wpc * isig;
  const double u_c = wpth * isig * T6;
  double u_v = uT6 * T7;
  double u_kd = uT2 * a;
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
  double u_r2a2 = u_S;
  u_a2s = fma(-u_S, s, u_a2s);
  u_s = fma(-u_S, a2s, u_s);
  u_r2a2 = fma(u_K, E, u_r2a2);
  u_E = fma(u_K, r2a2, u_E);
  u_a = fma(-u_K, L, u_a);
  u_L = fma(-u_K, a, u_L);
  u_a = fma(u_a2s, as, u_a);
  const double u_as = u_a2s * a;
  u_a = fma(u_as, s, u_a);
  u_s = fma(u_as, a, u_s);
  u_a = fma(u_ae, E, u_a);
  u_E = fma(u_ae, a, u_E);
  u_r = fma(2.0 * r, u_r2a2, u_r);
  u_a = fma(2.0 * a, u_r2a2, u_a);
  u_r = fma(2.0 * rm, u_D, u_r);
  u_a = fma(2.0 * a, u_D, u_a);
  yb[0] = u_r;
  yb[1] = fma(u_s, c, -u_c * s);
  yb[2] = u_pr;
  yb[3] = u_pth;
  *pt_b -= u_E;
  *pph_b += u_L;
  *a_b += u_a;
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
  long long first, n;  // this launch's rays: [first, n)
  double* theta;
  double* phi;
  double* jac;  // (n, 2, 4): rows theta_e, phi_e; columns alpha, beta, spin, theta_o (rad)
  long long* state;
  long long* n_steps;
  int* status;  // 0 ok, 1 tape full, 2 ended neither ESCAPED nor CAPTURED
  double* tape_h;   // (n, cap)
  double* tape_ck;  // (n, cap / K + 1, NV)
  double* final_rec;  // (n, FINAL_REC): the landed final state y, f = f(y), p_t, p_phi
  // The stage tape: a pool of chunks (STAGE_CHUNK steps of STEP_REC doubles), the chunk each
  // ray's k-th group of STAGE_CHUNK steps went to (n, cap / STAGE_CHUNK + 1), the chunks handed
  // out so far, and whether a ray's whole tape is there.
  double* pool;
  long long pool_chunks;
  unsigned long long* pool_next;
  int* chunk_tab;
  unsigned char* staged;
};

constexpr int FINAL_REC = 16;  // y[NV], f[NV], p_t, p_phi, two unused

// The forward pass's mode: Fast64 arithmetic whose inner stages write their inputs into the
// record of the step being attempted (a rejected attempt's record is overwritten by the next).
struct Fast64Taped : Fast64 {
  struct Shadow {
    static constexpr bool kTape = true;
    double* slot;  // the step's record in shared memory: stage inputs 0..5 x (r, p_r, p_theta, sin, cos)
    __device__ void record(int idx, double r, double pr, double pth, double s, double c) const {
      double* q = slot + STAGE_REC * idx;
      q[0] = r;
      q[1] = pr;
      q[2] = pth;
      q[3] = s;
      q[4] = c;
    }
  };
  __device__ static void init_rhs(const Params& P, const S y[NV], S pt, S pph, Shadow&, K f[NV], Trig& tr) {
    rhs(P, y[CR], y[CTH], pt, y[CPR], y[CPTH], pph, f, tr);
  }
  __device__ static void accepted(const Params&, const S[NV], Shadow&, const Trig&) {}
};

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

// One step of size h from the state in ry (f = f(y) and its trig with it), into ry.
template <class M>
__device__ __forceinline__ void step_to(const Params& P, Ray<M>& ry, double h) {
  double yn[NV], esum[NV], k6[NV];
  Trig tr;
  dp_stages<M, false>(P, ry, h, k6, yn, esum, tr);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    ry.y[i] = yn[i];
    ry.f[i] = k6[i];
  }
  ry.tr = tr;
}

// Replaces the last accepted step (y_prev -> ry, length h_last) by the DP5 step from y_prev
// that ends on r = rs: Newton on the step length, r(Phi(y_prev, h)) = rs with dr/dh = f_r at
// the step's end, three iterations from the linear estimate h_last - (r_N - rs) / f_r(y_N).
// The last step otherwise overshoots the surface by up to tens of M, and the output's
// linear projection back to rs then carries a second-order residual (theta'' dr^2 / 2, about
// 1e-5 rad at r = 1000) whose parameter derivative is not that of the crossing point. The
// accepted step is kept when an iterate leaves (0, h_last] or is not finite.  Each iteration
// records its stages in the last step's record (ry.sh); when the accepted step is kept after an
// iteration ran, the step of length h_last is run once more to record its own stages again
// (from y_prev, with f and the trig recomputed there: the values the accepted attempt used).
template <class M>
__device__ void land_on_surface(const Params& P, Ray<M>& ry, const double y_prev[NV], double rs, double& h_last) {
  double h = h_last - (ry.y[CR] - rs) / ry.f[CR];
  Ray<M> st = ry;
  auto from_prev = [&]() {
#pragma unroll
    for (int i = 0; i < NV; ++i) st.y[i] = y_prev[i];
    M::init_rhs(P, st.y, st.pt, st.pph, st.sh, st.f, st.tr);
  };
  bool ran = false, landed = true;
  for (int it = 0; it <= 3; ++it) {
    if (!(isfinite(h) && h / h_last > 0.0 && h / h_last <= 1.0)) {
      landed = false;
      break;
    }
    from_prev();
    step_to(P, st, h);
    ran = true;
    if (it < 3) h -= (st.y[CR] - rs) / st.f[CR];
  }
  if (landed) {
#pragma unroll
    for (int i = 0; i < NV; ++i) landed = landed && isfinite(st.y[i]) && isfinite(st.f[i]);
  }
  if (!landed) {
    if constexpr (decltype(st.sh)::kTape) {
      if (ran) {
        from_prev();
        step_to(P, st, h_last);
      }
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    ry.y[i] = st.y[i];
    ry.f[i] = st.f[i];
  }
  h_last = h;
}

// The bulk copy of a record (shared -> global, 240 B, both 16 B aligned) and the waits on it.
__device__ __forceinline__ void record_copy(double* dst, const double* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(src);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the record's generic stores, before the copy reads
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(s),
               "r"((unsigned)(STEP_REC * sizeof(double)))
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void record_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void record_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

constexpr int FWD_BLOCK = 128;

// Forward pass: camera, the integration with the reference controller recording the tape (step
// sizes, checkpoints, stage records), the landing on the termination surface, the map's value,
// and the landed final state.  Two blocks per SM (228 registers, no spills): a map of more rays
// than that holds starts its later blocks as earlier ones end, the rays in trace order (longest
// first by default); three blocks per SM (168 registers, spilling) ran 0.5-1 % slower.
__global__ void __launch_bounds__(FWD_BLOCK, 2) k_lensing_forward(LensArgs A) {
  __shared__ __align__(16) double recs[FWD_BLOCK * STEP_REC];
  const long long ray = A.first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n) return;
  const Params& P = A.P;
  double y0[8];
  camera_state_t<double>(A.alpha[ray], A.beta[ray], A.P.a, A.th_o, A.r_o, A.ph_o, A.mass, y0);
  double* tape_h = A.tape_h + ray * (long long)A.cap;
  const int n_ck = A.cap / A.K + 1;
  double* tape_ck = A.tape_ck + ray * (long long)n_ck * NV;
  int* tab = A.chunk_tab + ray * (long long)(A.cap / STAGE_CHUNK + 1);
  Ray<Fast64Taped> ry;
  ray_init<Fast64Taped>(P, y0, carter_initial(P, y0), ry);
  ry.sh.slot = recs + threadIdx.x * STEP_REC;
#pragma unroll
  for (int i = 0; i < NV; ++i) tape_ck[i] = ry.y[i];
  int status = 0;
  bool staged = A.pool_chunks > 0;
  int group = -1;            // the step group (STAGE_CHUNK steps) whose chunk `chunk` is
  int recorded = -1;         // the step whose record holds stage input 0 (its start state)
  double* chunk = nullptr;
  double y_prev[NV] = {};  // the state before the last accepted step
  while (ry.state == RUNNING) {
    const int n = ry.n_steps;  // the step being attempted
    if (staged && n / STAGE_CHUNK != group) {
      group = n / STAGE_CHUNK;
      const unsigned long long id = atomicAdd(A.pool_next, 1ull);
      if (id < (unsigned long long)A.pool_chunks) {
        chunk = A.pool + (long long)id * (STAGE_CHUNK * STEP_REC);
        tab[group] = (int)id;
      } else {
        staged = false;
      }
    }
    if (recorded != n) {
      record_wait_read();  // the last step's copy has read the slot
      ry.sh.record(0, ry.y[CR], ry.y[CPR], ry.y[CPTH], ry.tr.s, ry.tr.c);
      recorded = n;
    }
    double y_cur[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) y_cur[i] = ry.y[i];
    attempt<Fast64Taped, false>(P, ry, nullptr, nullptr);
    if (ry.n_steps != n) {
      const int n1 = ry.n_steps;
      if (n1 > A.cap) {
        status = 1;
        break;
      }
      // The record goes out now, unless this step ended the ray: the landing rewrites it first.
      if (staged && ry.state == RUNNING) record_copy(chunk + (n % STAGE_CHUNK) * STEP_REC, ry.sh.slot);
#pragma unroll
      for (int i = 0; i < NV; ++i) y_prev[i] = y_cur[i];
      tape_h[n1 - 1] = ry.h_taken;
      if (n1 % A.K == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) tape_ck[(n1 / A.K) * NV + i] = ry.y[i];
      }
    }
  }
  const int N = ry.n_steps;
  A.state[ray] = ry.state;
  A.n_steps[ray] = N;
  if (status == 0 && ry.state != ESCAPED && ry.state != CAPTURED) status = 2;
  const double rs = surface_radius(P, ry.state);
  if (status == 0 && N > 0) {
    record_wait_read();
    land_on_surface(P, ry, y_prev, rs, tape_h[N - 1]);  // rewrites the last step's record
    if (staged) record_copy(chunk + ((N - 1) % STAGE_CHUNK) * STEP_REC, ry.sh.slot);
  }
  record_wait_all();
  // 3. the output at the termination surface (event-time correction); a ray whose tape ran
  // out, or that reached neither surface, has no output (NaN, like its Jacobian)
  const double dr = ry.y[CR] - rs;
  const double fr = ry.f[CR];
  A.theta[ray] = status == 0 ? ry.y[CTH] - ry.f[CTH] / fr * dr : CUDART_NAN;
  A.phi[ray] = status == 0 ? ry.y[CPH] - ry.f[CPH] / fr * dr : CUDART_NAN;
  A.status[ray] = status;
  A.staged[ray] = (status == 0 && staged && N > 0) ? 1 : 0;
  double* rec = A.final_rec + ray * FINAL_REC;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    rec[i] = ry.y[i];
    rec[NV + i] = ry.f[i];
  }
  rec[2 * NV] = ry.pt;
  rec[2 * NV + 1] = ry.pph;
}

// The reverse sweep from the stage tape: one thread per (ray, cotangent row), two threads per
// ray.  Rays not on the tape (status != 0, or chunks the pool could not hold) are left to
// k_lensing_reverse.
__global__ void __launch_bounds__(128) k_lensing_reverse_staged(LensArgs A) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ray = A.first + (t >> 1);
  const int row = (int)(t & 1);  // 0: theta_e, 1: phi_e
  if (ray >= A.n || !A.staged[ray]) return;
  const Params& P = A.P;
  const double m = A.mass, a = A.P.a;
  const int N = (int)A.n_steps[ray];
  const int state = (int)A.state[ray];
  const double rs = surface_radius(P, state);
  const double* tape_h = A.tape_h + ray * (long long)A.cap;
  const int* tab = A.chunk_tab + ray * (long long)(A.cap / STAGE_CHUNK + 1);
  const double* fin = A.final_rec + ray * FINAL_REC;
  const double pt = fin[2 * NV], pph = fin[2 * NV + 1];
  const int oc = row ? CPH : CTH;
  // Cotangent of the state (r, theta, p_r, p_theta), of p_t, p_phi and of a.  Those of t and phi
  // stay what the output gives them (0 and [row == 1]): f depends on neither.
  double xr, xth, xpr, xpth, xpt = 0.0, xpph = 0.0, xa = 0.0;
  const double xph = row ? 1.0 : 0.0;
  {
    // 3'. the output x_e = x_N - (f_x / f_r)(r_N - r_s)
    const double dr = fin[CR] - rs, fr = fin[NV + CR], fx = fin[NV + oc];
    double sN, cN;
    sincos(fin[CTH], &sN, &cN);
    const double wo = -dr / fr, wr = dr * fx / (fr * fr);
    double yb[4];
    rhs_vjp_row(m, a, fin[CR], sN, cN, pt, fin[CPR], fin[CPTH], pph, wr, row ? 0.0 : wo, row ? wo : 0.0, 0.0, 0.0,
                yb, &xpt, &xpph, &xa);
    xr = yb[0] - fx / fr;
    xth = yb[1] + (row ? 0.0 : 1.0);
    xpr = yb[2];
    xpth = yb[3];
    if (state == CAPTURED) xa += fx / fr * (-a / sqrt(m * m - a * a));  // r_s = r_plus(a) + epsilon
  }
  // 4. reverse over the steps: y_new = y + h sum_j b_j k_j, stage input Y_s = y + h sum_{j<s}
  // a_sj k_j, k_s = f(Y_s); record s of step n holds Y_s (Y_0 = y).
  // Each step's record address is formed a step ahead and its lines prefetched into L1.
  auto rec_of = [&](int n) {
    return A.pool + (long long)tab[n / STAGE_CHUNK] * (STAGE_CHUNK * STEP_REC) + (n % STAGE_CHUNK) * STEP_REC;
  };
  const double* rec_next = rec_of(N - 1);
  for (int n = N - 1; n >= 0; --n) {
    const double* rec = rec_next;
    if (n > 0) {
      rec_next = rec_of(n - 1);
      asm volatile("prefetch.global.L1 [%0];" ::"l"(rec_next));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(rec_next + 16));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(rec_next + STEP_REC - 1));
    }
    const double h = tape_h[n];
    double kb[6][4];  // cotangents of k_0..k_5 over (r, theta, p_r, p_theta)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const double w = h * dp_a(5, j);
      kb[j][0] = w * xr;
      kb[j][1] = w * xth;
      kb[j][2] = w * xpr;
      kb[j][3] = w * xpth;
    }
#pragma unroll
    for (int sg = 5; sg >= 0; --sg) {
      const double* q = rec + STAGE_REC * sg;
      double yb[4];
      rhs_vjp_row(m, a, q[0], q[3], q[4], pt, q[1], q[2], pph, kb[sg][0], kb[sg][1], h * dp_a(5, sg) * xph,
                  kb[sg][2], kb[sg][3], yb, &xpt, &xpph, &xa);
      xr += yb[0];
      xth += yb[1];
      xpr += yb[2];
      xpth += yb[3];
#pragma unroll
      for (int j = 0; j < sg; ++j) {
        const double w = h * dp_a(sg - 1, j);
        if (w != 0.0) {
#pragma unroll
          for (int i = 0; i < 4; ++i) kb[j][i] = fma(w, yb[i], kb[j][i]);
        }
      }
    }
  }
  // 1'. the camera state's Jacobian in (alpha, beta, a, theta_o); 5. the chain
  Dual<4> y0d[8];
  camera_state_t<Dual<4>>(Dual<4>::var(A.alpha[ray], 0), Dual<4>::var(A.beta[ray], 1), Dual<4>::var(a, 2),
                          Dual<4>::var(A.th_o, 3), A.r_o, A.ph_o, m, y0d);
  const double xb8[8] = {0.0, xr, xth, xph, xpt, xpr, xpth, xpph};  // the 8-state order
  double g[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int p = 0; p < 4; ++p) g[p] = fma(xb8[i], y0d[i].d[p], g[p]);
  }
  double* J = A.jac + ray * 8 + row * 4;
  J[0] = g[0];
  J[1] = g[1];
  J[2] = (g[2] + xa) * m;
  J[3] = g[3];
}

// Reverse pass of the rays not on the stage tape: the cotangents of the landed output, the
// checkpointed reverse sweep over the recorded steps (both rows in one thread), and the chain
// through the camera's Jacobian.
#ifndef KRR_LENS_REVERSE_MINB
#define KRR_LENS_REVERSE_MINB 1  // resident blocks per SM the reverse kernel's registers allow for
#endif
__global__ void __launch_bounds__(128, KRR_LENS_REVERSE_MINB) k_lensing_reverse(LensArgs A) {
  const long long ray = A.first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n || A.staged[ray]) return;
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
// adjoint differentiates), for finite-difference checks.  A ray with more steps than the tape
// holds (status 1) or that reached neither surface (status 2) has no recorded map: NaN.
__global__ void __launch_bounds__(128) k_lensing_replay(LensArgs A) {
  const long long ray = A.first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ray >= A.n) return;
  const long long n_rec = A.n_steps[ray];
  const int st = (int)A.state[ray];
  const int bad = (n_rec < 0 || n_rec > A.cap) ? 1 : (st != ESCAPED && st != CAPTURED) ? 2 : 0;
  if (bad) {
    A.theta[ray] = CUDART_NAN;
    A.phi[ray] = CUDART_NAN;
    A.status[ray] = bad;
    return;
  }
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
  A.pool = L.pool;
  A.pool_chunks = L.pool_chunks;
  A.pool_next = L.pool_next;
  A.chunk_tab = L.chunk_tab;
  A.staged = L.staged;
  const int block = FWD_BLOCK;
  const unsigned grid = (unsigned)((L.n + block - 1) / block);
  if (replay) {
    k_lensing_replay<<<grid, block, 0, s>>>(A);
    return cudaGetLastError();
  }
  cudaError_t e = cudaMemsetAsync(L.pool_next, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  // Two halves (the first rounded to whole blocks) on two streams when the caller gave a second:
  // the half whose forward pass ends first runs its reverse sweeps beside the other's forward
  // tail (5.5 against 5.8 ms for the 55k-ray edge map; halves of 35, 42 and 58 % of the rays no
  // faster, four quarters, whose forward passes fill too few SMs, 7.0 ms).  The halves share the
  // stage pool, first come first served; every ray's results are the same either way.
  const bool split = L.aux && L.n > 2 * block;
  const long long half = split ? (L.n / 2 + block - 1) / block * block : L.n;
  if (split) {
    if ((e = cudaEventRecord(L.ev_fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(L.aux, L.ev_fork, 0)) != cudaSuccess) return e;
  }
  for (int part = 0; part < (split ? 2 : 1) && e == cudaSuccess; ++part) {
    cudaStream_t st = part ? L.aux : s;
    A.first = part ? half : 0;
    A.n = part ? L.n : half;
    const long long cnt = A.n - A.first;
    const unsigned g = (unsigned)((cnt + block - 1) / block);
    k_lensing_forward<<<g, block, 0, st>>>(A);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    k_lensing_reverse_staged<<<(unsigned)((2 * cnt + block - 1) / block), block, 0, st>>>(A);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    k_lensing_reverse<<<g, block, 0, st>>>(A);
    e = cudaGetLastError();
  }
  // Once forked, the second stream joins back even after a failed launch, so that a capture of
  // the caller's stream can still end; the first error is the one returned.
  if (split) {
    cudaError_t j = cudaEventRecord(L.ev_join, L.aux);
    if (j == cudaSuccess) j = cudaStreamWaitEvent(s, L.ev_join, 0);
    if (e == cudaSuccess) e = j;
  }
  return e;
}

}  // namespace krr
