/*
 * kerrray_cuda.h -- C ABI of the B200 (sm_100a) backend of KerrRay's per-ray hot path.
 *
 * The library (kerrray_b200/libkerrray_cuda.so) fills the "cuda" slot of KerrRay's backend
 * registry.  Every entry point takes plain pointers and sizes; none keeps a pointer after it
 * returns.  All functions return a status code (KRR_OK on success); krr_last_error() gives a
 * thread-local message for the last failure on the calling thread.  Calls are thread-safe: the
 * host-buffer entry points serialise per device, and krr_lensing_adjoint holds the same lock
 * while it enqueues its work (on the caller's stream and the library's second stream).
 *
 * Reference interfaces replaced (file:line within joelprince2601/kerrray):
 *   krr_integrate_batch         Backend.integrate_batch
 *                               (src/kerrray/raytracing/backends/base.py:53-68), whose CPU forms are
 *                               integrate_batch_numba (raytracing/backends/numba_backend.py:131-207)
 *                               and integrate_rays_kernel (raytracing/backends/numba_kernel.py:467-474)
 *   krr_integrate_batch_device  the same on device-resident buffers and a caller stream
 *   krr_camera_states           initial_states (src/kerrray/raytracing/camera.py:298-381) for a
 *                               pixel grid or for arbitrary image points (the PointCamera of
 *                               scripts/study_edge_bisection.py:39-50)
 *   krr_trace_images            compute_shadow (src/kerrray/raytracing/shadow.py:179-211) for many
 *                               images in one persistent launch (camera, integration and
 *                               classification on the device)
 *   krr_max_attempts            max_attempts (src/kerrray/geodesics/integrators.py:151-162)
 */
#ifndef KERRRAY_CUDA_H
#define KERRRAY_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KRR_ABI_VERSION 6

#if defined(__GNUC__)
#define KRR_API __attribute__((visibility("default")))
#else
#define KRR_API
#endif

/* Status codes. */
enum {
  KRR_OK = 0,
  KRR_ERR_INVALID = 1,     /* invalid argument (the reference raises ValueError)            */
  KRR_ERR_NO_DEVICE = 2,   /* no CUDA device / driver (the reference raises BackendUnavailable) */
  KRR_ERR_CUDA = 3,        /* CUDA runtime error                                            */
  KRR_ERR_TIMEOUT = 4,     /* a bounded device wait or deadline expired                     */
  KRR_ERR_UNSUPPORTED = 5, /* option combination not supported by this build                */
  KRR_ERR_NOT_NULL = 6     /* camera projection not null to 1e-10 (the reference raises RuntimeError) */
};

/* Arithmetic of the step loop. */
enum {
  KRR_PREC_REFERENCE = 0, /* reference operation order, no contraction; FP64 or the FP32 dtype */
  KRR_PREC_FAST64 = 1,    /* FP64 with FMA contraction, sincos and reciprocals                */
  KRR_PREC_MIXED = 2      /* FP32 stages, FP64 state accumulation, Delta and error norm       */
};

/* FP64 re-trace after (or beside) a mixed-precision trace (krr_launch.retrace). */
enum {
  KRR_RETRACE_NONE = 0,
  KRR_RETRACE_EDGE = 1,     /* after the trace: every pixel that did not end ESCAPED or CAPTURED or
                               whose code differs from one of its 8 neighbours */
  KRR_RETRACE_CRITICAL = 2, /* before the trace, each photon's analytic class from its constants of
                               motion (radial potential R(r)); photons within a band of the
                               critical curve run in reference order on SMs of their own, beside
                               the main trace; afterwards photons whose code is not their analytic
                               class are traced again in FP64, and what still disagrees (or ended
                               within 1 % of its affine or step budget) in reference order: the
                               plain FP64 kernel's mask */
  KRR_RETRACE_CRITICAL_NEAR = 3  /* KRR_RETRACE_CRITICAL and, for a mixed trace, the escaping photons
                               within 0.35 M of the critical curve traced in fast FP64 on SMs of their
                               own as well: exit directions within the oracle's bar there too */
};

/* termination codes (photons/classification.py:60-69) */
enum {
  KRR_RUNNING = 0, KRR_ESCAPED = 1, KRR_CAPTURED = 2, KRR_MAX_AFFINE_PARAMETER = 3,
  KRR_NUMERICAL_FAILURE = 4, KRR_OUT_OF_DOMAIN = 5, KRR_DISK_HIT = 6
};

/* IntegratorOptions + TerminationOptions + EventOptions (geodesics/integrators.py:71-148). */
typedef struct krr_options {
  int32_t method;          /* 0 = "rk45" (Dormand-Prince 5(4)), 1 = "rk4" */
  int32_t dtype;           /* 0 = "float64", 1 = "float32" (reference precision mode) */
  double rtol, atol;
  double step_size;        /* initial (rk45) or fixed (rk4) step */
  double lambda_max;
  double h_min;
  double h_max;            /* +inf for None */
  int64_t max_steps;
  double horizon_epsilon;  /* capture at r <= r_plus + horizon_epsilon */
  double escape_radius;
  int32_t disk_plane;      /* equatorial disk-plane event */
  int32_t reserved;
  double r_in, r_out;
} krr_options;

/* BatchResult (photons/trajectories.py:100-128).  Y, state must be non-null; the rest may be
 * null when not wanted.  event_Y / event_hit are written only with disk_plane set. */
typedef struct krr_result {
  double* Y;                /* (N, 8) final states */
  int64_t* state;           /* (N,) termination codes */
  int64_t* n_steps;         /* (N,) accepted steps */
  int64_t* n_rejected;      /* (N,) rejected attempts */
  double* lam;              /* (N,) final affine parameter */
  double* max_null_error;   /* (N,) */
  double* max_energy_drift; /* (N,) */
  double* max_lz_drift;     /* (N,) */
  double* max_carter_drift; /* (N,) */
  double* event_Y;          /* (N, 8) */
  uint8_t* event_hit;       /* (N,) */
} krr_result;

/* Camera (raytracing/camera.py:99-204). */
typedef struct krr_camera {
  double radius;           /* observer Boyer-Lindquist radius r_o (M) */
  double inclination_deg;  /* clamped into [1e-3, 180 - 1e-3] like the reference */
  double phi_deg;
  double fov;              /* half-width of the image plane (M) */
  int64_t resolution;      /* even, >= 2 */
} krr_camera;

/* One image of a batched launch, or a range of its pixels: with pixel_count > 0 the entry
 * traces pixels first_pixel .. first_pixel + pixel_count - 1 of the camera's grid (row-major),
 * and its result rows are those pixels in order; pixel_count == 0 (with first_pixel == 0) is the
 * whole image.  Ranges let several GPUs share one image (KRR_RETRACE_EDGE needs whole images). */
typedef struct krr_image {
  double mass, spin;
  krr_camera camera;
  krr_options options;
  int64_t first_pixel;
  int64_t pixel_count;
} krr_image;

/* Launch shape of the persistent kernel (0 = library default / autotuned). */
typedef struct krr_launch {
  int32_t precision;         /* KRR_PREC_* */
  int32_t block;             /* threads per block */
  int32_t blocks_per_sm;     /* resident blocks per SM */
  int32_t refill_threshold;  /* idle lanes of a warp before it refills from the queue */
  int32_t plain;             /* 1: one thread per photon, no work queue (the plain kernel) */
  int32_t variant;           /* compiled launch shape of the persistent kernel (krr_list_variants) */
  int32_t retrace;           /* KRR_RETRACE_*: settle the pixels a mixed trace could classify
                                differently with the reference-order FP64 kernel (rk45, float64,
                                persistent launches) */
  int32_t critical_sms;      /* KRR_RETRACE_CRITICAL: SMs of the critical-set kernel (0: 1/37 of
                                the SMs, at least 2) */
} krr_launch;

/* A compiled launch shape of the persistent kernel: threads per block and the launch-bounds
 * minimum of resident blocks per SM (its register cap), with the registers and the resident
 * blocks per SM the device reports. */
typedef struct krr_variant_info {
  int32_t block, min_blocks, registers, blocks_per_sm;
} krr_variant_info;

/* Counters of a batched launch. */
typedef struct krr_stats {
  uint64_t photons;     /* photons in the launch */
  uint64_t retired;     /* photons written back (== photons) */
  uint64_t attempts;    /* step attempts (accepted + rejected) */
  uint64_t accepted;    /* accepted steps */
  uint64_t lane_slots;  /* warp iterations x 32 */
  uint64_t busy_slots;  /* lane slots that advanced a running photon */
  double kernel_ms;     /* device time of the trace kernel (CUDA events on its stream) */
  uint64_t retraced;    /* photons traced in reference-order FP64 by the re-trace */
  uint64_t retrace_attempts;
  double retrace_ms;    /* device time of the flagging and the re-trace after the main trace */
  uint64_t critical;    /* KRR_RETRACE_CRITICAL: photons in the critical band (traced beside) */
  uint64_t rechecked;   /* KRR_RETRACE_CRITICAL: photons traced again after the check */
  double critical_ms;   /* KRR_RETRACE_CRITICAL: device time of the critical-set kernel */
  uint64_t speculative; /* krr_bisect_edges: photons traced ahead of their bracket by idle lanes */
  uint64_t discarded_attempts; /* krr_bisect_edges: attempts of those photons whose side was not
                                  taken (not in `attempts`, which counts the sequential bisection's) */
  uint64_t near_edge;   /* KRR_RETRACE_CRITICAL_NEAR with KRR_PREC_MIXED: escaping photons within
                           the near-edge band of the shadow boundary, traced in fast FP64 beside
                           the mixed trace (their exit directions need FP64) */
  uint64_t near_edge_attempts;
} krr_stats;

KRR_API const char* krr_last_error(void);
KRR_API int krr_abi_version(void);
KRR_API int krr_device_count(int* count);
KRR_API int krr_max_attempts(const krr_options* options, int64_t* out);

/* Integrate n initial states Y0 (n x 8, host) in spacetime (mass, spin) and write the result
 * into host arrays.  runtime_s (nullable) receives the wall-clock seconds of the call. */
KRR_API int krr_integrate_batch(int device, double mass, double spin, const double* Y0, int64_t n,
                        const krr_options* options, int32_t precision, const krr_result* out,
                        double* runtime_s);

/* The same on device buffers (Y0 and every result array on `device`), enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream); returns without synchronising.  index
 * (nullable, device) selects rows: ray i integrates Y0[index[i]] and writes row index[i]. */
KRR_API int krr_integrate_batch_device(int device, double mass, double spin, const double* d_Y0,
                               const int64_t* d_index, int64_t n, const krr_options* options,
                               int32_t precision, const krr_result* d_out, void* stream);

/* Where each escaped ray crosses r = r_surface: theta and phi of the rays whose state is ESCAPED
 * (device arrays d_Y (n x 8), d_state (n)), flown back from the final state -- the first
 * accepted state beyond the escape radius, which overshoots the surface by up to a step -- along
 * the same Hamiltonian (FP64 RK4 substeps, Newton on the affine offset); NaN for the other rows.
 * Two integrations of a ray are comparable there whatever steps they took.  Enqueued on
 * `stream` without synchronising.  No counterpart in the reference. */
KRR_API int krr_escape_directions(int device, double mass, double spin, double r_surface, const double* d_Y,
                                  const int64_t* d_state, int64_t n, double* d_theta, double* d_phi, void* stream);

/* Initial states of a pixel grid (alpha == beta == NULL: resolution^2 rows, row-major) or of n
 * arbitrary image points (alpha, beta host arrays of length n), written to host Y0 (rows x 8). */
KRR_API int krr_camera_states(int device, double mass, double spin, const krr_camera* camera,
                      const double* alpha, const double* beta, int64_t n, double* Y0);

/* Trace many images in one persistent launch.  The photons of image k are its pixels, in
 * row-major order, at global rows offset_k .. offset_k + resolution_k^2 (images in the given
 * order, offsets the running sum).  Y0 (nullable, host, total x 8) replaces the camera as the
 * photon source.  Results go to host arrays of total rows. */
KRR_API int krr_trace_images(int device, const krr_image* images, int32_t n_images, const double* Y0,
                     const krr_launch* launch, const krr_result* out, krr_stats* stats);

/* Device form of krr_trace_images: d_Y0 (nullable) and d_out on `device`; `workspace` is at
 * least krr_workspace_size(n_images, retrace ? total photons : 0) bytes of device memory owned
 * by the caller; stream as above.  Synchronises the stream before returning (the statistics
 * are read back). */
KRR_API size_t krr_workspace_size(int32_t n_images, int64_t retrace_photons);

/* Analytic class of n initial states (host arrays; no device needed): 0 escapes, 1 is captured,
 * 2 lies within the critical band (risk_band: max(2e-3, 2e3 rtol) M in the image plane) of the
 * boundary between the two, or is not an inward ray outside r_+ + horizon_epsilon.  From the
 * radial potential of the photon's constants of motion (Carter 1968); the classes the
 * KRR_RETRACE_CRITICAL pipeline uses.  No counterpart in the reference. */
KRR_API int krr_analytic_classes(double mass, double spin, double rtol, double horizon_epsilon, const double* Y0,
                                 int64_t n, uint8_t* out);

/* The launch shapes compiled for (precision, options.method, options.dtype): *count receives
 * their number; up to max_out are described in out (nullable) for `device`.  Measurement
 * support for the autotuner; no counterpart in the reference. */
KRR_API int krr_list_variants(int device, int32_t precision, const krr_options* options, krr_variant_info* out,
                              int32_t max_out, int32_t* count);
KRR_API int krr_trace_images_device(int device, const krr_image* images, int32_t n_images, const double* d_Y0,
                            const krr_launch* launch, const krr_result* d_out, void* workspace,
                            size_t workspace_bytes, void* stream, krr_stats* stats);

/* A batched launch captured once as a CUDA graph and replayed: krr_plan_create waits for the
 * device to finish its pending work (so a workspace still being filled on another stream is
 * safe), uploads the image descriptors into `workspace` (krr_workspace_size bytes,
 * caller-owned, like the outputs and d_Y0 it must outlive the plan) and captures the whole
 * launch sequence (counter resets,
 * persistent trace, and with retrace the flagging and FP64 re-trace, whose size is read on the
 * device); krr_plan_launch enqueues it on `stream` without synchronising; krr_plan_stats
 * synchronises `stream` and reads the counters of the last launch (kernel times 0: time the
 * launches with events on your stream).  Replaces compute_shadow
 * (src/kerrray/raytracing/shadow.py:179-211) repeated over the same images. */
typedef struct krr_plan krr_plan;
KRR_API int krr_plan_create(int device, const krr_image* images, int32_t n_images, const double* d_Y0,
                            const krr_launch* launch, const krr_result* d_out, void* workspace,
                            size_t workspace_bytes, krr_plan** plan);
KRR_API int krr_plan_launch(krr_plan* plan, void* stream);
KRR_API int krr_plan_stats(krr_plan* plan, void* stream, krr_stats* stats);
KRR_API int krr_plan_destroy(krr_plan* plan);

/* One case of a batched edge bisection: spacetime, observer, integrator options and the
 * image-plane centre the polar angles are measured about. */
typedef struct krr_edge_case {
  double mass, spin;
  double radius, inclination_deg, phi_deg;
  krr_options options;
  double centre_alpha, centre_beta;
} krr_edge_case;

/* Bisect the image radius of the shadow edge along n_items polar directions on the device
 * (scripts/study_edge_bisection.py:53-68, bisect_edge, with its PointCamera :39-50): item k
 * belongs to case item_case[k], looks along (cos_phi[k], sin_phi[k]) and starts from the
 * bracket [lo[k], hi[k]] (captured at lo, escaped at hi); each of `iterations` halvings traces
 * the photon at mid = (lo + hi) / 2 and moves hi to mid if it ESCAPED, lo otherwise.  lo and hi
 * are updated in place (host arrays); failures[k] (nullable) counts results that were neither
 * ESCAPED nor CAPTURED.  All iterations of all items run in one persistent launch. */
KRR_API int krr_bisect_edges(int device, const krr_edge_case* cases, int32_t n_cases, const int32_t* item_case,
                             const double* cos_phi, const double* sin_phi, double* lo, double* hi,
                             int64_t* failures, int64_t n_items, int32_t iterations, int32_t precision,
                             krr_stats* stats);

/* The lensing map of one observer, differentiated: for n image points (alpha, beta) the terminal
 * celestial direction (theta_e, phi_e) -- theta and phi located on the termination surface
 * (escape radius, or capture radius) from the last accepted state by one step along the flow;
 * on the capture surface r_+ + epsilon the Boyer-Lindquist coordinates are singular (phi grows
 * like log(r - r_+), the derivatives like 1 / (r - r_+)), so the derivatives are meant for
 * escaping rays --
 * and its Jacobian d(theta_e, phi_e)/d(alpha, beta, spin, theta_o [rad]) (jac: n x 2 x 4), by the
 * adjoint of the discretised Dormand-Prince 5(4) map over the recorded accepted steps with the
 * controller held fixed.  FP64.  No counterpart in the reference (its gradients are finite
 * differences of raytracing/backends/numba_backend.py runs).  Device buffers; `workspace` (256-byte
 * aligned, as cudaMalloc returns it) holds the tape and must be kept for krr_lensing_replay.
 * The tape: every accepted step's size, the state every `checkpoint_every` steps, and -- in
 * whatever workspace lies beyond krr_lensing_workspace_size bytes -- a pool of stage records
 * (the six stage inputs of each step, 240 B per step, in 16-step chunks).  A ray whose records
 * all fit is swept back from them; the others recompute each checkpoint segment in the reverse
 * sweep (the same derivative to rounding, several times slower).  krr_lensing_workspace_size
 * is the minimum (no pool); krr_lensing_workspace_size_staged adds a pool for `stage_steps`
 * accepted steps in all (their sum over the rays, plus one chunk of rounding per ray).  The rays
 * in flight take chunks first come, first served, so a pool well short of the total keeps
 * whole record sets only for the rays that finish before it runs out.
 * status[k]: 0 ok, 1 more accepted steps than tape_capacity, 2 neither ESCAPED nor CAPTURED; a ray
 * with status 1 or 2 gets NaN for theta, phi and its Jacobian, and krr_lensing_replay gives it NaN
 * and the same status.
 * Asynchronous on `stream`: beyond 256 rays the second half of them runs on a stream of the
 * library's own, forked from `stream` and joined back to it before the call returns, so work
 * ordered after the call on `stream` sees every ray's results, and a capture of `stream` holds
 * both halves. */
typedef struct krr_lens_params {
  double mass, spin;
  double radius, inclination_deg, phi_deg;
  krr_options options;  /* rk45, float64, no events */
  int32_t checkpoint_every;  /* K, 1..64 */
  int32_t tape_capacity;     /* accepted steps recorded per ray */
} krr_lens_params;
KRR_API size_t krr_lensing_workspace_size(int64_t n, int32_t tape_capacity, int32_t checkpoint_every);
KRR_API size_t krr_lensing_workspace_size_staged(int64_t n, int32_t tape_capacity, int32_t checkpoint_every,
                                                 int64_t stage_steps);
KRR_API int krr_lensing_adjoint(int device, const krr_lens_params* params, const double* d_alpha, const double* d_beta,
                                int64_t n, double* d_theta, double* d_phi, double* d_jac, int64_t* d_state,
                                int64_t* d_n_steps, int32_t* d_status, void* workspace, size_t workspace_bytes,
                                void* stream);
/* After krr_lensing_adjoint on this workspace (same params and n): rays swept from the stage
 * records, pool chunks taken and pool chunks the workspace holds.  Synchronises `stream`. */
KRR_API int krr_lensing_tape_usage(const krr_lens_params* params, int64_t n, const void* workspace,
                                   size_t workspace_bytes, int64_t* staged_rays, int64_t* chunks_used,
                                   int64_t* chunks_total, void* stream);
/* Re-run the map with the step sequence recorded by the last krr_lensing_adjoint call on this
 * workspace (same n, states and step counts), for other (alpha, beta, spin, inclination): the
 * discrete map the adjoint differentiates, without the controller. */
KRR_API int krr_lensing_replay(int device, const krr_lens_params* params, const double* d_alpha, const double* d_beta,
                               int64_t n, const int64_t* d_state, const int64_t* d_n_steps, double* d_theta,
                               double* d_phi, int32_t* d_status, const void* workspace, size_t workspace_bytes,
                               void* stream);

/* Allocation-free form of krr_trace_images_device.  No counterpart in the reference.  For
 * callers that cannot allocate device memory on this path (an application that owns a fixed
 * device-memory budget and forbids allocations after start-up, a plug-in whose host owns all
 * device memory): the launch's scratch (work-queue counters and image descriptors) lives in a
 * static array in the library's device image, sized for at most KRR_NOALLOC_MAX_IMAGES images
 * (about 47 KB per device, held until exit); larger batches are rejected with KRR_ERR_INVALID.
 * Inputs (d_Y0, nullable) and outputs (d_out) are the caller's device buffers; nothing is
 * allocated.  The first call on a device looks up the array's device address.  All calls share
 * the one array (its counters, and the disk-event outputs when given, are cleared at the start
 * of each call): calls that overlap on the GPU race, so serialise them (one stream, or one call
 * at a time).  The call is synchronous: it uploads the descriptors from host memory, reads the
 * counters back and synchronises `stream`, so it must not run during a stream capture (a
 * capturing stream is refused with KRR_ERR_UNSUPPORTED).  kernel_ms is reported as 0. */
#define KRR_NOALLOC_MAX_IMAGES 128
KRR_API int krr_trace_images_noalloc(int device, const krr_image* images, int32_t n_images, const double* d_Y0,
                                     const krr_launch* launch, const krr_result* d_out, void* stream,
                                     krr_stats* stats);

/* Measurement utility with no counterpart in the reference (which reports no GPU number):
 * the FP64 (fp64 != 0) or FP32 FMA throughput of `device` in TFLOP/s (2 FLOP per FMA), from
 * dependent FMA chains timed with CUDA events; the roofline denominator of the step kernels. */
KRR_API int krr_fma_peak(int device, int fp64, double* tflops);

/* Accretion-disk shading (raytracing/renderer.py:188-199, render_disk's step 3; physics/
 * redshift.py:131 redshift_factor; physics/accretion.py:180-195 observed_intensity) of n traced rays, device arrays,
 * enqueued on `stream`: for every row with d_hit[i] != 0, the redshift factor g = nu_obs / nu_em
 * of the crossing state d_event_Y[i] (n x 8, the stored reversed momentum as the integrator
 * writes it) for a circular equatorial Keplerian emitter (prograde != 0: a L_z > 0), and
 * I_obs = g^redshift_power (r / r_in)^-emissivity_index on r_in <= r <= r_out, 0 outside;
 * d_r_hit = r.  Rows without a hit get g = r_hit = NaN and I = 0.  A hit that is not equatorial
 * (to 1e-6), lies where no circular orbit exists, or gives g <= 0 gets g = NaN: the reference
 * raises ValueError there, and so do this library's Python bindings. */
KRR_API int krr_disk_shading(int device, double mass, double spin, int32_t prograde, double r_in, double r_out,
                             double emissivity_index, int32_t redshift_power, const double* d_event_Y,
                             const uint8_t* d_hit, int64_t n, double* d_g, double* d_intensity, double* d_r_hit,
                             void* stream);

/* Accuracy utility with no counterpart in the reference: the step kernels' own sine and cosine
 * forms at n angles (device arrays), enqueued on `stream`.  which 0: the FP32 sine and cosine of
 * an FP64 angle (reduced by the nearest multiple of pi/2; the mixed mode's accepted states);
 * 1: the FP32 small-angle shift from the FP32-rounded sine and cosine of theta by (float)delta
 * (the mixed stages); 2: the FP64 shift by delta (the fast64 stages).  Results as FP64; NaN where
 * a shift declines (|delta| above 1/4 in FP32, 1/10 in FP64).  d_delta may be NULL for which 0. */
KRR_API int krr_trig_eval(int device, int32_t which, const double* d_theta, const double* d_delta, int64_t n,
                          double* d_sin, double* d_cos, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* KERRRAY_CUDA_H */
