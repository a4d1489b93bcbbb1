// Internal launch interface between the host ABI (krr_abi.cu) and the two kernel translation
// units: krr_ref.cu (reference operation order, compiled with -fmad=false) and krr_fast.cu
// (FMA contraction: FP64 and the FP32/FP64 mixed mode).
#pragma once

#include <cuda_runtime.h>

#include "krr_kernels.cuh"

namespace krr {

// Reference order: dtype32 selects the reference's float32 working precision.
cudaError_t ref_plain(bool dtype32, bool rk4, const PlainArgs& a, int block, cudaStream_t s);
const Variant* ref_variants(bool dtype32, bool rk4, int* count);

// Fast modes: mixed selects FP32 stages with FP64 accumulation; otherwise FP64.
cudaError_t fast_plain(bool mixed, bool rk4, const PlainArgs& a, int block, cudaStream_t s);
const Variant* fast_variants(bool mixed, bool rk4, int* count);
const Variant* mixed_sat_variant();

// theta and phi where each escaped ray (state ESCAPED) crosses r = r_s, flown back from its final
// state Y; NaN for the other rows.
cudaError_t escape_directions(const Params& P, double r_s, const double* Y, const long long* state, long long n,
                              double* theta, double* phi, cudaStream_t s);

// Disk shading of n crossing states (see k_disk_shading): g, I_obs and r of each hit row.
cudaError_t disk_shading(double m, double a, int prograde, double r_in, double r_out, double p_index, int n_pow,
                         const double* Y, const unsigned char* hit, long long n, double* g, double* inten, double* r_hit,
                         cudaStream_t s);

// Adds to *count (device) the number of non-finite values among the n doubles at x (device).
cudaError_t count_nonfinite(const double* x, long long n, unsigned long long* count, int sms, cudaStream_t s);

// The step kernels' sine and cosine forms at given angles (which: 0 FP32 reduced, 1 FP32 shift,
// 2 FP64 shift; see k_trig_eval).
cudaError_t trig_eval(int which, const double* theta, const double* delta, long long n, double* s_out, double* c_out,
                      cudaStream_t s);

// Edge bisection launches (persistent, one item per lane).
cudaError_t ref_bisect(const EdgeArgs& a, cudaStream_t s);
cudaError_t fast_bisect(bool mixed, const EdgeArgs& a, cudaStream_t s);

// Lensing-map adjoint (krr_adjoint.cu): derivatives of the terminal celestial direction with
// respect to (alpha, beta, spin, theta_o); replay = the recorded step sequence without them.
// The lensing adjoint's stage tape: per accepted step, six stage inputs of STAGE_REC doubles
// (r, p_r, p_theta, sin theta, cos theta); pool chunks of STAGE_CHUNK steps.
constexpr int STAGE_REC = 5;
constexpr int STEP_REC = 6 * STAGE_REC;
constexpr int STAGE_CHUNK = 16;

struct LensLaunch {
  Params P;
  double spin, mass, r_o, th_o, ph_o;
  int K, cap;
  const double* alpha;
  const double* beta;
  long long n;
  double* theta;
  double* phi;
  double* jac;
  long long* state;
  long long* n_steps;
  int* status;
  double* tape_h;
  double* tape_ck;
  double* final_rec;  // (n, 16) landed final states, written by the forward kernel
  double* pool;       // stage-tape chunks (pool_chunks x STAGE_CHUNK x STEP_REC doubles)
  long long pool_chunks;
  unsigned long long* pool_next;  // chunks handed out (zeroed before the forward kernel)
  int* chunk_tab;                 // (n, cap / STAGE_CHUNK + 1)
  unsigned char* staged;          // (n): the ray's whole stage tape is in the pool
  // A second stream and two events of the caller's: with them the rays run as two halves, the
  // second on `aux` (forked from and joined back to the launch stream), so that one half's
  // reverse sweep fills the SMs the other half's forward pass leaves idle.  Null: one stream.
  cudaStream_t aux;
  cudaEvent_t ev_fork, ev_join;
};
cudaError_t lensing_adjoint(const LensLaunch& L, bool replay, cudaStream_t s);

// Append the pixels to re-trace in FP64 (failures and the shadow edge) to `list`.
cudaError_t flag_boundary(const Image* images, int n_images, long long total, const long long* state, long long* list,
                          Queue* q, cudaStream_t s);

// The critical-set pipeline: analytic classes of every photon (critical ones appended to
// `list`), the reference-order kernel whose blocks fill an SM each, and the check of the mixed
// results against the analytic classes (disagreements appended to `list`).
cudaError_t risk_prepass(const Image* images, int n_images, long long total, const double* Y0, unsigned char* risk,
                         long long* list, Queue* q, long long* near_list, Queue* q_near, cudaStream_t s);
// One block of 384 threads per SM in fast FP64 (its registers fill the SM): the near-edge
// photons of the mixed pipeline, on SMs of their own beside the mixed trace.
const Variant* near_wide_variant();
const Variant* ref_wide_variant();
cudaError_t check_risk(const Image* images, int n_images, long long total, const unsigned char* risk,
                       const long long* state, long long* list, Queue* q, bool recheck, cudaStream_t s);

// Camera initial states for a pixel grid (alpha == beta == nullptr) or for points.
cudaError_t camera_states(const Frame& F, double fov, long long res, const double* alpha, const double* beta,
                          long long n, double* Y0, int* err, cudaStream_t s);

}  // namespace krr
