// Host side of the C ABI declared in include/kerrray_cuda.h: argument validation with the
// reference's rules, parameter packing, per-device contexts with cached device buffers, and
// the launches of the kernels in krr_ref.cu / krr_fast.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kerrray_cuda.h"
#include "krr_host.h"
#include "krr_launch.h"

namespace krr_host {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define KRR_CUDA(call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return fail(KRR_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

constexpr double kInclinationEps = 1e-3;  // utils/config.py INCLINATION_EPSILON_DEG (camera.py:155)
constexpr double kSafety = 0.9, kFactorMax = 5.0;

// ------------------------------------------------------------------------------------------
// Validation and packing (geodesics/integrators.py:98-129, numba_backend.py:87-115).
// ------------------------------------------------------------------------------------------
bool finite_pos(double x) { return std::isfinite(x) && x > 0.0; }

int validate_options(const krr_options* o) {
  if (!o) return fail(KRR_ERR_INVALID, "options must not be NULL");
  if (o->method != 0 && o->method != 1) return fail(KRR_ERR_INVALID, "method must be 'rk45' (0) or 'rk4' (1), got %d", o->method);
  if (o->dtype != 0 && o->dtype != 1) return fail(KRR_ERR_INVALID, "dtype must be float64 (0) or float32 (1), got %d", o->dtype);
  const struct { const char* name; double v; } pos[] = {{"rtol", o->rtol}, {"atol", o->atol}, {"step_size", o->step_size},
                                                      {"lambda_max", o->lambda_max}, {"h_min", o->h_min}};
  for (const auto& p : pos)
    if (!finite_pos(p.v)) return fail(KRR_ERR_INVALID, "%s must be a finite number > 0, got %g", p.name, p.v);
  if (!(std::isinf(o->h_max) && o->h_max > 0) && !finite_pos(o->h_max))
    return fail(KRR_ERR_INVALID, "h_max must be None or a finite number > 0, got %g", o->h_max);
  if (o->max_steps < 1) return fail(KRR_ERR_INVALID, "max_steps must be >= 1, got %lld", (long long)o->max_steps);
  if (!(std::isfinite(o->horizon_epsilon) && o->horizon_epsilon >= 0.0))
    return fail(KRR_ERR_INVALID, "horizon_epsilon must be >= 0, got %g", o->horizon_epsilon);
  if (!finite_pos(o->escape_radius)) return fail(KRR_ERR_INVALID, "escape_radius must be > 0, got %g", o->escape_radius);
  if (o->disk_plane && !(0.0 < o->r_in && o->r_in <= o->r_out))
    return fail(KRR_ERR_INVALID, "need 0 < r_in <= r_out, got r_in=%g, r_out=%g", o->r_in, o->r_out);
  return KRR_OK;
}

int validate_spacetime(double mass, double spin) {
  if (!finite_pos(mass)) return fail(KRR_ERR_INVALID, "mass must be a finite number > 0, got %g", mass);
  if (!(std::isfinite(spin) && std::fabs(spin) < 1.0)) return fail(KRR_ERR_INVALID, "spin must satisfy abs(spin) < 1, got %g", spin);
  return KRR_OK;
}

long long max_attempts(const krr_options* o) {  // integrators.py:151-162
  const double h_max = std::max(o->lambda_max, o->step_size);
  const double rej = (std::log(h_max / o->h_min) + (double)o->max_steps * std::log(kFactorMax)) / std::log(1.0 / kSafety);
  return o->max_steps + (long long)std::ceil(rej) + 1;
}

double outer_horizon(double mass, double a) { return mass + std::sqrt(mass * mass - a * a); }  // horizons.py:33-42

krr::Params make_params(double mass, double spin, const krr_options* o) {
  krr::Params P{};
  const double m = mass, a = spin * mass;
  P.mass = m;
  P.a = a;
  P.a2 = a * a;
  P.neg_2ma = (-2.0 * m) * a;
  P.pos_2ma = (2.0 * m) * a;
  P.two_m = 2.0 * m;
  P.two_a2 = 2.0 * (a * a);
  P.rtol = o->rtol;
  P.atol = o->atol;
  P.h0 = o->step_size;
  P.h_min = o->h_min;
  P.h_max = o->h_max;
  P.lambda_max = o->lambda_max;
  P.r_capture = outer_horizon(m, a) + o->horizon_epsilon;
  P.r_escape = o->escape_radius;
  P.r_in = o->disk_plane ? o->r_in : 0.0;
  P.r_out = o->disk_plane ? o->r_out : 0.0;
  P.max_steps = o->max_steps;
  P.guard = max_attempts(o);
  P.rk4 = o->method == 1;
  P.disk = o->disk_plane != 0;
  P.r_plus = outer_horizon(m, a);
  P.f_mass = (float)m;
  P.f_a = (float)P.a;
  P.f_a2 = (float)P.a2;
  P.f_rpm = (float)(2.0 * std::sqrt(m * m - a * a));
  return P;
}

// Observer frame at (r_o, theta_o, phi_o): covariant metric (geometry/metric.py:147-163), ZAMO
// tetrad (raytracing/camera.py:225-262) and contravariant metric (metric.py:166-195).
int make_frame(double mass, double spin, const krr_camera* c, krr::Frame& F) {
  if (!c) return fail(KRR_ERR_INVALID, "camera must not be NULL");
  if (!finite_pos(c->radius)) return fail(KRR_ERR_INVALID, "radius must be a finite number > 0, got %g", c->radius);
  if (!(std::isfinite(c->inclination_deg) && c->inclination_deg >= 0.0 && c->inclination_deg <= 180.0))
    return fail(KRR_ERR_INVALID, "inclination_deg must lie in [0, 180], got %g", c->inclination_deg);
  if (!std::isfinite(c->phi_deg)) return fail(KRR_ERR_INVALID, "phi_deg must be finite, got %g", c->phi_deg);
  const double m = mass, a = spin * mass;
  const double r = c->radius;
  if (r <= outer_horizon(m, a))
    return fail(KRR_ERR_INVALID, "camera radius %.6g must exceed the outer horizon r_plus = %.6g", r, outer_horizon(m, a));
  const double incl = std::min(std::max(c->inclination_deg, kInclinationEps), 180.0 - kInclinationEps);
  const double th = incl * (M_PI / 180.0);
  F.r_o = r;
  F.th_o = th;
  F.ph_o = c->phi_deg * (M_PI / 180.0);
  const double sn = std::sin(th), cs = std::cos(th);
  const double s2 = sn * sn;
  const double sig = r * r + (a * a) * (cs * cs);
  const double dlt = r * r - 2.0 * m * r + a * a;
  const double g_tt = -(1.0 - 2.0 * m * r / sig);
  const double g_tphi = -2.0 * m * a * r * s2 / sig;
  const double g_rr = sig / dlt;
  const double g_thth = sig + 0.0 * dlt;
  const double g_phph = (r * r + a * a + 2.0 * m * (a * a) * r * s2 / sig) * s2;
  const double omega = -g_tphi / g_phph;
  const double lapse2 = -(g_tt - (g_tphi * g_tphi) / g_phph);
  if (!(lapse2 > 0.0)) return fail(KRR_ERR_INVALID, "lapse^2 = Sigma Delta / A is not positive: point is not outside the horizon");
  const double lapse = std::sqrt(lapse2);
  F.e00 = 1.0 / lapse;
  F.e03 = omega / lapse;
  F.e11 = 1.0 / std::sqrt(g_rr);
  F.e22 = 1.0 / std::sqrt(g_thth);
  F.e33 = 1.0 / std::sqrt(g_phph);
  F.g_tt = g_tt;
  F.g_tphi = g_tphi;
  F.g_rr = g_rr;
  F.g_thth = g_thth;
  F.g_phph = g_phph;
  const double r2a2 = r * r + a * a;
  const double big_a = r2a2 * r2a2 - (a * a) * dlt * s2;
  const double sd = sig * dlt;
  F.gi_tt = -big_a / sd;
  F.gi_tphi = -2.0 * m * a * r / sd;
  F.gi_rr = dlt / sig;
  F.gi_thth = 1.0 / sig + 0.0 * dlt;
  F.gi_phph = (dlt - (a * a) * s2) / (sd * s2);
  return KRR_OK;
}

int validate_grid(const krr_camera* c) {
  if (!finite_pos(c->fov)) return fail(KRR_ERR_INVALID, "fov must be a finite number > 0, got %g", c->fov);
  if (c->resolution < 2 || c->resolution % 2 != 0)
    return fail(KRR_ERR_INVALID, "resolution must be an even integer >= 2, got %lld", (long long)c->resolution);
  // The outermost pixel centre has the largest alpha^2 + beta^2 (camera.py:342-348).
  const double n = (double)c->resolution;
  const double edge = c->fov * (2.0 * (n - 1.0) + 1.0 - n) / n;
  if ((edge * edge + edge * edge) / (c->radius * c->radius) >= 1.0)
    return fail(KRR_ERR_INVALID, "fov = %.6g is too large for radius = %.6g (need fov < radius / sqrt(2))", c->fov, c->radius);
  return KRR_OK;
}

// ------------------------------------------------------------------------------------------
// Per-device context: a stream, events and grow-only device buffers, behind a mutex.
// ------------------------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
};

enum BufId { B_Y0, B_Y, B_STATE, B_STEPS, B_REJ, B_LAM, B_NULL, B_E, B_LZ, B_Q, B_EVY, B_EVHIT, B_IMAGES, B_QUEUE, B_AB, B_ERR, B_FINITE, B_COUNT };

struct Context {
  std::mutex mu;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  cudaStream_t copy_stream = nullptr;   // device-to-host copies beside the trace (krr_trace_images)
  cudaStream_t h2d_stream = nullptr;    // host-to-device copies of Y0 ahead of the trace
  cudaEvent_t chunk_ev[4] = {};         // the end of each chunk's trace
  cudaEvent_t h2d_ev[4] = {};           // each chunk's Y0 on the device
  cudaStream_t trace2 = nullptr;        // every other chunk's trace, so consecutive traces overlap their tails
  cudaEvent_t fork_ev = nullptr;        // trace2 starts after the setup on the main stream
  cudaStream_t lens_aux = nullptr;      // the lensing map's second half of the rays
  cudaEvent_t lens_fork = nullptr, lens_join = nullptr;
  int sm_count = 0;
  DevBuf buf[B_COUNT];
};

std::mutex g_ctx_mu;
std::vector<std::unique_ptr<Context>> g_ctx;

int get_context(int device, Context** out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(KRR_ERR_NO_DEVICE, "no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  if (device < 0 || device >= count) return fail(KRR_ERR_INVALID, "device %d out of range [0, %d)", device, count);
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if ((int)g_ctx.size() < count) g_ctx.resize(count);
  if (!g_ctx[device]) {
    auto c = std::make_unique<Context>();
    c->device = device;
    KRR_CUDA(cudaSetDevice(device));
    KRR_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    KRR_CUDA(cudaEventCreate(&c->ev0));
    KRR_CUDA(cudaEventCreate(&c->ev1));
    KRR_CUDA(cudaEventCreate(&c->ev2));
    KRR_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    KRR_CUDA(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
    KRR_CUDA(cudaStreamCreateWithFlags(&c->trace2, cudaStreamNonBlocking));
    KRR_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    KRR_CUDA(cudaStreamCreateWithFlags(&c->lens_aux, cudaStreamNonBlocking));
    KRR_CUDA(cudaEventCreateWithFlags(&c->lens_fork, cudaEventDisableTiming));
    KRR_CUDA(cudaEventCreateWithFlags(&c->lens_join, cudaEventDisableTiming));
    for (auto& ev : c->chunk_ev) KRR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (auto& ev : c->h2d_ev) KRR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    KRR_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    g_ctx[device] = std::move(c);
  }
  *out = g_ctx[device].get();
  return KRR_OK;
}

// Every value finite: a branch-free pass over the exponent fields (vectorised by the host
// compiler; an early-exit isfinite loop ran at a fraction of the memory bandwidth).
bool all_finite(const double* x, size_t n) {
  const uint64_t* b = reinterpret_cast<const uint64_t*>(x);
  constexpr uint64_t kExp = 0x7ff0000000000000ull;
  uint64_t bad = 0;
  for (size_t i = 0; i < n; ++i) bad |= (uint64_t)((b[i] & kExp) == kExp);
  return bad == 0;
}

// all_finite over up to 16 host threads for large arrays (memory-bandwidth bound).
bool all_finite_parallel(const double* x, size_t n) {
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < ((size_t)1 << 22) || hw == 1) return all_finite(x, n);
  std::vector<char> ok(hw, 1);
  std::vector<std::thread> threads;
  const size_t per = (n + hw - 1) / hw;
  for (unsigned t = 0; t < hw; ++t)
    threads.emplace_back([&, t] {
      const size_t a = t * per, b = std::min(n, a + per);
      if (a < b) ok[t] = all_finite(x + a, b - a);
    });
  for (auto& th : threads) th.join();
  return std::all_of(ok.begin(), ok.end(), [](char v) { return v != 0; });
}

// Host Y0 (rows x 8) to the device buffer B_Y0, checked there for non-finite values before any
// trace work (the reference raises on them).  The check runs on the device: a host scan of a
// large sweep's Y0 (~1e8 doubles) took longer than the copy itself.  Waits for the stream.
int upload_y0(Context* c, const double* Y0, long long rows, const double** d_out) {
  const size_t bytes = (size_t)rows * 8 * sizeof(double);
  KRR_CUDA(c->buf[B_Y0].ensure(bytes));
  KRR_CUDA(c->buf[B_FINITE].ensure(sizeof(unsigned long long)));
  auto* d_count = static_cast<unsigned long long*>(c->buf[B_FINITE].p);
  KRR_CUDA(cudaMemcpyAsync(c->buf[B_Y0].p, Y0, bytes, cudaMemcpyHostToDevice, c->stream));
  KRR_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), c->stream));
  KRR_CUDA(krr::count_nonfinite(static_cast<const double*>(c->buf[B_Y0].p), rows * 8, d_count, c->sm_count, c->stream));
  unsigned long long bad = 0;
  KRR_CUDA(cudaMemcpyAsync(&bad, d_count, sizeof(bad), cudaMemcpyDeviceToHost, c->stream));
  KRR_CUDA(cudaStreamSynchronize(c->stream));
  if (bad) return fail(KRR_ERR_INVALID, "Y0 must be finite (%llu non-finite values)", bad);
  *d_out = static_cast<const double*>(c->buf[B_Y0].p);
  return KRR_OK;
}

int sm_count_of(int device) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n;
}

krr::Outputs to_outputs(const krr_result* r) {
  krr::Outputs o{};
  o.Y = r->Y;
  o.state = reinterpret_cast<long long*>(r->state);
  o.n_steps = reinterpret_cast<long long*>(r->n_steps);
  o.n_rej = reinterpret_cast<long long*>(r->n_rejected);
  o.lam = r->lam;
  o.max_null = r->max_null_error;
  o.max_e = r->max_energy_drift;
  o.max_lz = r->max_lz_drift;
  o.max_q = r->max_carter_drift;
  o.event_Y = r->event_Y;
  o.event_hit = r->event_hit;
  return o;
}

int check_precision(int32_t precision, const krr_options* o) {
  if (precision < KRR_PREC_REFERENCE || precision > KRR_PREC_MIXED)
    return fail(KRR_ERR_INVALID, "precision must be 0 (reference), 1 (fast64) or 2 (mixed), got %d", precision);
  if (precision != KRR_PREC_REFERENCE && o->dtype == 1)
    return fail(KRR_ERR_UNSUPPORTED, "dtype float32 runs in the reference precision mode only");
  if (precision == KRR_PREC_MIXED && o->method == 1)
    return fail(KRR_ERR_UNSUPPORTED, "the mixed precision mode integrates with rk45 only");
  return KRR_OK;
}

cudaError_t launch_plain(int32_t precision, const krr_options* o, const krr::PlainArgs& a, cudaStream_t s) {
  const bool rk4 = o->method == 1;
  const int block = 128;  // a multiple of 32 (the kernel's warp-aggregated counters assume it)
  if (precision == KRR_PREC_REFERENCE) return krr::ref_plain(o->dtype == 1, rk4, a, block, s);
  return krr::fast_plain(precision == KRR_PREC_MIXED, rk4, a, block, s);
}

// Allocate (in the context) a device copy of each requested result array.
int device_results(Context* c, int64_t n, const krr_result* host, bool disk, krr_result* dev) {
  std::memset(dev, 0, sizeof(*dev));
  struct Item { BufId id; size_t bytes; bool want; void** slot; };
  const size_t n8 = (size_t)n * 8 * sizeof(double), n1 = (size_t)n * sizeof(double);
  Item items[] = {
      {B_Y, n8, true, (void**)&dev->Y},
      {B_STATE, n1, true, (void**)&dev->state},
      {B_STEPS, n1, host->n_steps != nullptr, (void**)&dev->n_steps},
      {B_REJ, n1, host->n_rejected != nullptr, (void**)&dev->n_rejected},
      {B_LAM, n1, host->lam != nullptr, (void**)&dev->lam},
      {B_NULL, n1, host->max_null_error != nullptr, (void**)&dev->max_null_error},
      {B_E, n1, host->max_energy_drift != nullptr, (void**)&dev->max_energy_drift},
      {B_LZ, n1, host->max_lz_drift != nullptr, (void**)&dev->max_lz_drift},
      {B_Q, n1, host->max_carter_drift != nullptr, (void**)&dev->max_carter_drift},
      {B_EVY, n8, disk && host->event_Y != nullptr, (void**)&dev->event_Y},
      {B_EVHIT, (size_t)n, disk && host->event_hit != nullptr, (void**)&dev->event_hit},
  };
  for (auto& it : items) {
    if (!it.want) continue;
    KRR_CUDA(c->buf[it.id].ensure(std::max<size_t>(it.bytes, 16)));
    *it.slot = c->buf[it.id].p;
  }
  if (dev->event_Y) KRR_CUDA(cudaMemsetAsync(dev->event_Y, 0, n8, c->stream));
  if (dev->event_hit) KRR_CUDA(cudaMemsetAsync(dev->event_hit, 0, (size_t)n, c->stream));
  return KRR_OK;
}

int copy_results_back(Context* c, int64_t n, const krr_result* dev, const krr_result* host) {
  const size_t n8 = (size_t)n * 8 * sizeof(double), n1 = (size_t)n * sizeof(double);
  struct Pair { void* dst; const void* src; size_t bytes; };
  Pair pairs[] = {
      {host->Y, dev->Y, n8}, {host->state, dev->state, n1}, {host->n_steps, dev->n_steps, n1},
      {host->n_rejected, dev->n_rejected, n1}, {host->lam, dev->lam, n1},
      {host->max_null_error, dev->max_null_error, n1}, {host->max_energy_drift, dev->max_energy_drift, n1},
      {host->max_lz_drift, dev->max_lz_drift, n1}, {host->max_carter_drift, dev->max_carter_drift, n1},
      {host->event_Y, dev->event_Y, n8}, {host->event_hit, dev->event_hit, (size_t)n},
  };
  for (auto& p : pairs)
    if (p.dst && p.src && p.bytes) KRR_CUDA(cudaMemcpyAsync(p.dst, p.src, p.bytes, cudaMemcpyDeviceToHost, c->stream));
  return KRR_OK;
}

// Rows [r0, r1) of every requested result, device to host, on stream s.
int copy_rows_back(const krr_result* dev, const krr_result* host, long long r0, long long r1, cudaStream_t s) {
  const size_t n = (size_t)(r1 - r0), o = (size_t)r0;
  struct Slice { void* dst; const void* src; size_t row; };
  Slice sl[] = {
      {host->Y, dev->Y, 64}, {host->state, dev->state, 8}, {host->n_steps, dev->n_steps, 8},
      {host->n_rejected, dev->n_rejected, 8}, {host->lam, dev->lam, 8}, {host->max_null_error, dev->max_null_error, 8},
      {host->max_energy_drift, dev->max_energy_drift, 8}, {host->max_lz_drift, dev->max_lz_drift, 8},
      {host->max_carter_drift, dev->max_carter_drift, 8}, {host->event_Y, dev->event_Y, 64},
      {host->event_hit, dev->event_hit, 1},
  };
  for (auto& x : sl)
    if (x.dst && x.src && n)
      KRR_CUDA(cudaMemcpyAsync(static_cast<char*>(x.dst) + o * x.row, static_cast<const char*>(x.src) + o * x.row,
                               n * x.row, cudaMemcpyDeviceToHost, s));
  return KRR_OK;
}

// The pixels an image entry covers: [first_pixel, first_pixel + pixel_count) of its grid, or
// the whole grid when pixel_count is 0.
int pixel_range(const krr_image& im, long long* first, long long* count) {
  const long long all = im.camera.resolution * im.camera.resolution;
  if (im.pixel_count == 0) {
    if (im.first_pixel != 0) return fail(KRR_ERR_INVALID, "first_pixel must be 0 when pixel_count is 0 (the whole image)");
    *first = 0;
    *count = all;
    return KRR_OK;
  }
  if (im.pixel_count < 0 || im.first_pixel < 0 || im.first_pixel > all - im.pixel_count)
    return fail(KRR_ERR_INVALID, "pixel range [%lld, %lld) lies outside the %lld pixels of the image",
                (long long)im.first_pixel, (long long)(im.first_pixel + im.pixel_count), all);
  *first = im.first_pixel;
  *count = im.pixel_count;
  return KRR_OK;
}

// Images -> device descriptors with running offsets.
int build_images(const krr_image* images, int32_t n_images, std::vector<krr::Image>& out, long long& total) {
  if (!images || n_images < 1) return fail(KRR_ERR_INVALID, "need at least one image");
  out.resize(n_images);
  total = 0;
  for (int k = 0; k < n_images; ++k) {
    const krr_image& im = images[k];
    int rc = validate_spacetime(im.mass, im.spin);
    if (rc) return rc;
    rc = validate_options(&im.options);
    if (rc) return rc;
    rc = make_frame(im.mass, im.spin, &im.camera, out[k].F);
    if (rc) return rc;
    rc = validate_grid(&im.camera);
    if (rc) return rc;
    rc = pixel_range(im, &out[k].first, &out[k].count);
    if (rc) return rc;
    out[k].P = make_params(im.mass, im.spin, &im.options);
    out[k].fov = im.camera.fov;
    out[k].res = im.camera.resolution;
    out[k].offset = total;
    total += out[k].count;
  }
  // All images of one launch share the scheme and working precision (one kernel instance).
  for (int k = 1; k < n_images; ++k)
    if (images[k].options.method != images[0].options.method || images[k].options.dtype != images[0].options.dtype)
      return fail(KRR_ERR_UNSUPPORTED, "all images of one launch must share method and dtype");
  return KRR_OK;
}

struct LaunchShape {
  const krr::Variant* v;
  int grid, refill;
};

const krr::Variant* variants_for(int32_t precision, const krr_options* o, int* count) {
  const bool rk4 = o->method == 1;
  if (precision == KRR_PREC_REFERENCE) return krr::ref_variants(o->dtype == 1, rk4, count);
  return krr::fast_variants(precision == KRR_PREC_MIXED, rk4, count);
}

int persistent_shape(int device, int32_t precision, const krr_options* o, const krr_launch* l, LaunchShape& s) {
  int count = 0;
  const krr::Variant* vs = variants_for(precision, o, &count);
  if (!vs || count < 1) return fail(KRR_ERR_UNSUPPORTED, "no persistent kernel for this precision/method");
  const int idx = (l && l->variant > 0) ? l->variant : 0;
  if (idx >= count) return fail(KRR_ERR_INVALID, "launch variant %d out of range [0, %d)", idx, count);
  s.v = &vs[idx];
  int occ = s.v->occupancy();
  if (occ < 1) return fail(KRR_ERR_CUDA, "persistent kernel variant %d cannot be resident on this device", idx);
  const int bps = (l && l->blocks_per_sm > 0) ? std::min(l->blocks_per_sm, occ) : occ;
  s.grid = sm_count_of(device) * bps;
  s.refill = (l && l->refill_threshold > 0) ? std::min(l->refill_threshold, 32) : 1;
  return KRR_OK;
}

// Device layout of a batched launch's workspace: four queue counters (the main trace; the
// reference-order trace of the edge or of the critical photons; with the critical set, the
// FP64 re-trace of photons unlike their analytic class and the reference-order re-trace of
// what remains), the image descriptors, then, with the re-trace on, the photon list (one
// int64 per photon) and the analytic classes (one byte per photon).
struct WorkLayout {
  krr::Queue* q0;
  krr::Queue* q1;
  krr::Queue* q2;
  krr::Queue* q3;
  krr::Queue* q4;  // the near-edge photons of the critical-set pipeline
  krr::Image* images;
  long long* list;
  long long* near_list;
  unsigned char* risk;
};

constexpr size_t round256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kQueueArea = 1280;  // five queues, 256 bytes apart
static_assert(sizeof(krr::Queue) <= 256, "a queue must fit its 256-byte slot of the workspace");

// With re-trace entries: the list, the near-edge list (8 bytes per entry each) and the
// analytic classes (1 byte).
size_t work_bytes(int n_images, long long list_entries) {
  const size_t n = (size_t)std::max(list_entries, 0LL);
  return kQueueArea + round256((size_t)std::max(n_images, 0) * sizeof(krr::Image)) + 2 * round256(n * 8) + n;
}

WorkLayout work_layout(void* base, int n_images, long long list_entries) {
  char* b = static_cast<char*>(base);
  WorkLayout w;
  w.q0 = reinterpret_cast<krr::Queue*>(b);
  w.q1 = reinterpret_cast<krr::Queue*>(b + 256);
  w.q2 = reinterpret_cast<krr::Queue*>(b + 512);
  w.q3 = reinterpret_cast<krr::Queue*>(b + 768);
  w.q4 = reinterpret_cast<krr::Queue*>(b + 1024);
  const size_t list_at = kQueueArea + round256((size_t)n_images * sizeof(krr::Image));
  const size_t list_bytes = round256((size_t)std::max(list_entries, 0LL) * 8);
  w.images = reinterpret_cast<krr::Image*>(b + kQueueArea);
  w.list = reinterpret_cast<long long*>(b + list_at);
  w.near_list = reinterpret_cast<long long*>(b + list_at + list_bytes);
  w.risk = reinterpret_cast<unsigned char*>(b + list_at + 2 * list_bytes);
  return w;
}

// Everything a batched launch enqueues, resolved and validated up front.
struct Pipeline {
  int device = 0;
  int n_images = 0;
  long long total = 0;
  bool plain = false;
  int plain_block = 128;
  int32_t precision = KRR_PREC_FAST64;
  bool dtype32 = false, rk4 = false, disk = false;
  bool retrace = false;
  int retrace_mode = 0;  // KRR_RETRACE_*
  WorkLayout w{};
  krr_result out{};
  krr::PersistArgs main{};
  const krr::Variant* main_v = nullptr;
  krr::PersistArgs re{};
  const krr::Variant* re_v = nullptr;
  krr::PersistArgs crit{};  // KRR_RETRACE_CRITICAL: the critical photons, on SMs of their own
  const krr::Variant* crit_v = nullptr;
  krr::PersistArgs fix{};   // the FP64 re-trace of photons unlike their analytic class
  const krr::Variant* fix_v = nullptr;
  bool near = false;        // KRR_RETRACE_CRITICAL of a mixed trace: the near-edge photons in fast FP64
  krr::PersistArgs nearby{};
  const krr::Variant* near_v = nullptr;
};

// Registers one resident block of a kernel holds (allocated per warp in units of 256).
int block_registers(int threads, int regs_per_thread) {
  const int warps = (threads + 31) / 32;
  return warps * ((regs_per_thread * 32 + 255) / 256 * 256);
}

int prepare_pipeline(int device, const krr_image* images, int n_images, long long total, const double* d_Y0,
                     const krr_launch* launch, const krr_result* d_out, void* d_work, size_t work_size, Pipeline& p) {
  const int32_t precision = launch ? launch->precision : KRR_PREC_FAST64;
  const krr_options* o0 = &images[0].options;
  int rc = check_precision(precision, o0);
  if (rc) return rc;
  p.device = device;
  p.n_images = n_images;
  p.total = total;
  p.precision = precision;
  p.dtype32 = o0->dtype == 1;
  p.rk4 = o0->method == 1;
  p.disk = o0->disk_plane != 0;
  p.plain = launch && launch->plain;
  p.plain_block = (launch && launch->block > 0 && launch->block % 32 == 0) ? launch->block : 128;
  p.retrace_mode = launch ? launch->retrace : 0;
  if (p.retrace_mode < KRR_RETRACE_NONE || p.retrace_mode > KRR_RETRACE_CRITICAL_NEAR)
    return fail(KRR_ERR_INVALID, "retrace must be 0, 1 (edge), 2 (critical) or 3 (critical and near-edge), got %d",
                p.retrace_mode);
  // KRR_RETRACE_CRITICAL_NEAR is the critical-set pipeline with the near-edge band.
  const bool near_band = p.retrace_mode == KRR_RETRACE_CRITICAL_NEAR;
  if (near_band) p.retrace_mode = KRR_RETRACE_CRITICAL;
  p.retrace = p.retrace_mode != KRR_RETRACE_NONE;
  if (p.retrace && (p.rk4 || p.dtype32 || p.plain))
    return fail(KRR_ERR_UNSUPPORTED, "the FP64 re-trace follows persistent rk45 float64 launches only");
  if (p.retrace_mode == KRR_RETRACE_CRITICAL) {
    for (int k = 0; k < n_images; ++k)
      if (images[k].options.disk_plane)
        return fail(KRR_ERR_UNSUPPORTED, "the critical-set re-trace classifies ESCAPED/CAPTURED only (no disk events)");
  }
  if (p.retrace_mode == KRR_RETRACE_EDGE) {
    for (int k = 0; k < n_images; ++k)
      if (images[k].pixel_count != 0)
        return fail(KRR_ERR_UNSUPPORTED, "the edge re-trace compares every pixel with its 8 neighbours: whole images only");
  }
  const size_t need = work_bytes(n_images, p.retrace ? total : 0);
  if (work_size < need) return fail(KRR_ERR_INVALID, "workspace of %zu bytes is smaller than the %zu needed", work_size, need);
  p.w = work_layout(d_work, n_images, p.retrace ? total : 0);
  p.out = *d_out;
  LaunchShape shape{};
  rc = persistent_shape(device, precision, o0, launch, shape);
  if (rc) return rc;
  p.main_v = shape.v;
  p.main.images = p.w.images;
  p.main.n_images = n_images;
  p.main.total = total;
  p.main.Y0 = d_Y0;
  p.main.o = to_outputs(d_out);
  p.main.q = p.w.q0;
  p.main.refill_threshold = shape.refill;
  p.main.grid = shape.grid;
  p.main.block = shape.v->block;
  if (p.retrace) {
    LaunchShape rs{};
    krr_launch rl{};
    rl.precision = KRR_PREC_REFERENCE;
    rc = persistent_shape(device, KRR_PREC_REFERENCE, o0, &rl, rs);
    if (rc) return rc;
    p.re_v = rs.v;
    p.re = p.main;
    p.re.q = p.w.q1;
    p.re.grid = rs.grid;
    p.re.block = rs.v->block;
    p.re.refill_threshold = 1;
    p.re.index = p.w.list;
    p.re.d_total = &p.w.q0->flagged;
  }
  if (p.retrace_mode == KRR_RETRACE_CRITICAL) {
    // The reference-order kernel takes the critical photons on a few SMs: launched first,
    // each of its blocks fills an SM's register file, and it lets the main (mixed) trace launch
    // as soon as its blocks run (programmatic dependent launch), so the main trace -- which
    // skips the critical photons -- spreads over the other SMs and the two run side by side.
    // The main trace keeps its full grid: the blocks that do not fit wait for the critical
    // kernel's SMs and join the work queue when its blocks exit.  It waits for the critical
    // kernel only at its own exit.  Afterwards the photons unlike their analytic class are
    // traced again in fast FP64, and what still disagrees (or ended near its budget) in
    // reference order.
    const krr::Variant* wv = krr::ref_wide_variant();
    if (wv->occupancy() < 1) return fail(KRR_ERR_UNSUPPORTED, "the critical-set kernel cannot be resident");
    const int sms = std::max(sm_count_of(device), 2);
    const int crit_sms = std::min(sms - 1, (launch && launch->critical_sms > 0) ? launch->critical_sms : std::max(2, sms / 37));
    p.main.risk = p.w.risk;
    p.main.pdl = krr::PDL_WAIT;
    p.crit = p.main;
    p.crit_v = wv;
    p.crit.q = p.w.q1;
    p.crit.grid = crit_sms;
    p.crit.block = wv->block;
    p.crit.refill_threshold = 1;
    p.crit.index = p.w.list;
    p.crit.d_total = &p.w.q1->flagged;
    p.crit.risk = nullptr;
    p.crit.flags = krr::TRACE_SPREAD;
    p.crit.pdl = krr::PDL_TRIGGER | krr::PDL_STAMP;
    // Photons unlike their analytic class: after a mixed trace, rays an FP32 overflow ended
    // early, traced again with the overflow taken as a rejection (MixedSat); otherwise in FP64.
    int nf = 0;
    const krr::Variant* fv = krr::fast_variants(false, false, &nf);
    if (!fv || nf < 1) return fail(KRR_ERR_UNSUPPORTED, "no FP64 re-trace kernel");
    p.fix_v = (precision == KRR_PREC_MIXED) ? krr::mixed_sat_variant() : &fv[0];
    if (p.fix_v->occupancy() < 1) return fail(KRR_ERR_UNSUPPORTED, "the re-trace kernel cannot be resident");
    p.fix = p.crit;
    p.fix.q = p.w.q2;
    p.fix.grid = sms * p.fix_v->occupancy();
    p.fix.block = p.fix_v->block;
    p.fix.d_total = &p.w.q2->flagged;
    p.fix.pdl = 0;
    if (precision == KRR_PREC_MIXED) p.fix.flags |= krr::TRACE_RESUME;  // continue where the overflow stopped it
    p.re = p.fix;
    p.re.flags = krr::TRACE_SPREAD;  // from the camera: the plain kernel's exact arithmetic
    p.re.q = p.w.q3;
    p.re.grid = sms * p.re_v->occupancy();
    p.re.block = p.re_v->block;
    p.re.d_total = &p.w.q3->flagged;
    if (near_band && precision == KRR_PREC_MIXED) {
      // Escaping photons near the shadow edge (krr_radial.cuh:near_band) pass near the
      // unstable photon orbit, which magnifies the FP32 stages' round-off in their exit
      // direction: they are traced in fast FP64 by a third kernel, and the mixed trace skips
      // them.  It is launched first, one block filling each of a third of the SMs (a fifth, a
      // quarter and two fifths ran 3-7 % slower at 1024^2, the same at 2048^2), and lets the
      // critical kernel launch as soon as its blocks run; the critical kernel, launched as its
      // programmatic dependent, waits for it at its own exit, so the mixed trace's exit wait
      // covers all three.  Its blocks exit when its short queue is drained, and the mixed
      // trace's waiting blocks take their SMs.
      const krr::Variant* nv = krr::near_wide_variant();
      if (nv->occupancy() < 1) return fail(KRR_ERR_UNSUPPORTED, "the near-edge kernel cannot be resident");
      p.near = true;
      p.near_v = nv;
      p.nearby = p.crit;
      p.nearby.q = p.w.q4;
      p.nearby.grid = std::max(1, std::min(sms - crit_sms - 1, sms / 3));
      p.nearby.block = nv->block;
      p.nearby.index = p.w.near_list;
      p.nearby.d_total = &p.w.q4->flagged;
      p.nearby.risk = p.w.risk;  // a photon ending near a budget is marked for the re-check
      p.nearby.flags = krr::TRACE_SPREAD;
      p.nearby.pdl = krr::PDL_TRIGGER;
      p.crit.pdl |= krr::PDL_WAIT;
      p.main.flags |= krr::TRACE_SKIP_NEAR;
    }
  }
  return KRR_OK;
}

// The launch sequence (also what a plan captures): clear the counters, trace, and, with the
// re-trace on, flag the edge and failed pixels and trace them again in reference-order FP64.
// Events (nullable) bracket the main kernel (ev0, ev1) and the re-trace (ev1, ev2).
cudaError_t enqueue_critical(const Pipeline& p, cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, cudaEvent_t ev2) {
  cudaError_t e = cudaMemsetAsync(p.w.q0, 0, kQueueArea, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(&p.w.q1->t_first, 0xff, sizeof(unsigned long long), s);
  if (e == cudaSuccess && ev0) e = cudaEventRecord(ev0, s);
  const long long* state = reinterpret_cast<const long long*>(p.out.state);
  if (e == cudaSuccess)
    e = krr::risk_prepass(p.w.images, p.n_images, p.total, p.main.Y0, p.w.risk, p.w.list, p.w.q1,
                          p.near ? p.w.near_list : nullptr, p.w.q4, s);
  if (e == cudaSuccess && p.near) e = p.near_v->run(p.nearby, s);  // near-edge photons, fast FP64
  if (e == cudaSuccess) e = p.crit_v->run(p.crit, s);  // critical photons, reference order
  if (e == cudaSuccess) e = p.main_v->run(p.main, s);  // programmatic dependent: runs beside it
  if (e == cudaSuccess && ev1) e = cudaEventRecord(ev1, s);
  if (e == cudaSuccess) e = krr::check_risk(p.w.images, p.n_images, p.total, p.w.risk, state, p.w.list, p.w.q2, false, s);
  if (e == cudaSuccess) e = p.fix_v->run(p.fix, s);
  if (e == cudaSuccess) e = krr::check_risk(p.w.images, p.n_images, p.total, p.w.risk, state, p.w.list, p.w.q3, true, s);
  if (e == cudaSuccess) e = p.re_v->run(p.re, s);
  if (e == cudaSuccess && ev2) e = cudaEventRecord(ev2, s);
  return e;
}

cudaError_t enqueue_pipeline(const Pipeline& p, cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, cudaEvent_t ev2) {
  if (p.retrace_mode == KRR_RETRACE_CRITICAL) return enqueue_critical(p, s, ev0, ev1, ev2);
  cudaError_t e = cudaMemsetAsync(p.w.q0, 0, kQueueArea, s);
  if (e == cudaSuccess && p.out.event_Y) e = cudaMemsetAsync(p.out.event_Y, 0, (size_t)p.total * 8 * sizeof(double), s);
  if (e == cudaSuccess && p.out.event_hit) e = cudaMemsetAsync(p.out.event_hit, 0, (size_t)p.total, s);
  if (e == cudaSuccess && ev0) e = cudaEventRecord(ev0, s);
  if (e != cudaSuccess) return e;
  if (p.plain) {
    krr::PlainArgs pa{};
    pa.images = p.w.images;
    pa.n_images = p.n_images;
    pa.Y0 = p.main.Y0;
    pa.n = p.total;
    pa.o = p.main.o;
    pa.q = p.w.q0;
    e = p.precision == KRR_PREC_REFERENCE ? krr::ref_plain(p.dtype32, p.rk4, pa, p.plain_block, s)
                                          : krr::fast_plain(p.precision == KRR_PREC_MIXED, p.rk4, pa, p.plain_block, s);
  } else {
    e = p.main_v->run(p.main, s);
  }
  if (e == cudaSuccess && ev1) e = cudaEventRecord(ev1, s);
  if (e == cudaSuccess && p.retrace) {
    e = krr::flag_boundary(p.w.images, p.n_images, p.total, reinterpret_cast<const long long*>(p.out.state), p.w.list,
                           p.w.q0, s);
    if (e == cudaSuccess) e = p.re_v->run(p.re, s);
  }
  if (e == cudaSuccess && ev2) e = cudaEventRecord(ev2, s);
  return e;
}

// Read the counters back (synchronises the stream) and check the queue's bookkeeping.
int finish_pipeline(const Pipeline& p, cudaStream_t s, krr_stats* stats, cudaEvent_t ev0, cudaEvent_t ev1,
                    cudaEvent_t ev2) {
  krr::Queue q[5];
  std::memset(q, 0, sizeof(q));
  KRR_CUDA(cudaMemcpyAsync(&q[0], p.w.q0, sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(&q[1], p.w.q1, sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(&q[2], p.w.q2, sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(&q[3], p.w.q3, sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  if (p.near) KRR_CUDA(cudaMemcpyAsync(&q[4], p.w.q4, sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaStreamSynchronize(s));
  const bool crit = p.retrace_mode == KRR_RETRACE_CRITICAL;
  float ms = 0.0f, ms2 = 0.0f;
  if (ev0 && ev1) KRR_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  if (ev1 && ev2) KRR_CUDA(cudaEventElapsedTime(&ms2, ev1, ev2));
  const double ms_c = (crit && q[1].t_last >= q[1].t_first) ? 1e-6 * (double)(q[1].t_last - q[1].t_first) : 0.0;
  if (stats) {
    stats->photons = (uint64_t)p.total;
    stats->retired = q[0].retired;
    stats->attempts = q[0].attempts;
    stats->accepted = q[0].accepted;
    stats->lane_slots = q[0].lane_iters;
    stats->busy_slots = q[0].busy_iters;
    stats->kernel_ms = ms;
    stats->retraced = crit ? q[1].flagged + q[2].flagged + q[3].flagged : (p.retrace ? q[0].flagged : 0);
    stats->retrace_attempts = q[1].attempts + q[2].attempts + q[3].attempts;
    stats->retrace_ms = p.retrace ? ms2 : 0.0;
    stats->critical = crit ? q[1].flagged : 0;
    stats->critical_ms = ms_c;
    stats->rechecked = crit ? q[2].flagged + q[3].flagged : 0;
    stats->near_edge = p.near ? q[4].flagged : 0;
    stats->near_edge_attempts = p.near ? q[4].attempts : 0;
  }
  if (q[0].error || q[1].error || q[2].error || q[3].error || q[4].error)
    return fail(KRR_ERR_NOT_NULL, "tetrad projection is not null to 1e-10 (or no null momentum exists)");
  if (q[0].retired != (unsigned long long)p.total)
    return fail(KRR_ERR_CUDA, "work-queue inconsistency: %llu photons retired of %lld", q[0].retired, p.total);
  if (crit && (q[1].retired != q[1].flagged || q[2].retired != q[2].flagged || q[3].retired != q[3].flagged))
    return fail(KRR_ERR_CUDA, "critical-set inconsistency: %llu of %llu critical, %llu of %llu and %llu of %llu "
                "rechecked photons retired", q[1].retired, q[1].flagged, q[2].retired, q[2].flagged, q[3].retired,
                q[3].flagged);
  if (p.near && q[4].retired != q[4].flagged)
    return fail(KRR_ERR_CUDA, "near-edge inconsistency: %llu of %llu photons retired", q[4].retired, q[4].flagged);
  if (p.retrace && !crit && q[1].retired != q[0].flagged)
    return fail(KRR_ERR_CUDA, "re-trace inconsistency: %llu photons retired of %llu flagged", q[1].retired, q[0].flagged);
  return KRR_OK;
}

int run_images(Context* c, const krr_image* images, const std::vector<krr::Image>& ims, long long total,
               const double* d_Y0, const krr_launch* launch, const krr_result* d_out, void* d_work, size_t work_size,
               cudaStream_t s, krr_stats* stats) {
  Pipeline p;
  int rc = prepare_pipeline(c->device, images, (int)ims.size(), total, d_Y0, launch, d_out, d_work, work_size, p);
  if (rc) return rc;
  KRR_CUDA(cudaMemcpyAsync(p.w.images, ims.data(), ims.size() * sizeof(krr::Image), cudaMemcpyHostToDevice, s));
  KRR_CUDA(enqueue_pipeline(p, s, c->ev0, c->ev1, c->ev2));
  return finish_pipeline(p, s, stats, c->ev0, c->ev1, c->ev2);
}

// krr_trace_images with host results and no re-trace: the photons in up to four consecutive
// ranges, one persistent launch each (queue k starts at its range's first photon), each
// range's results copied to the host on a second stream while the next range is traced, and a
// host Y0 copied in range by range on a third.  The copies (0.8 GB in, 1.6 GB out for the
// 12.4M-photon sweep) then hide behind the trace except the first range's input and the last
// range's output; each extra launch costs one tail of idle lanes.
constexpr long long kChunkPhotons = 2'000'000;  // ranges of at least this many photons

int run_images_overlapped(Context* c, const krr_image* images, const std::vector<krr::Image>& ims, long long total,
                          const double* host_Y0, const krr_launch* launch, const krr_result* d_out,
                          const krr_result* host_out, void* d_work, size_t work_size, krr_stats* stats) {
  const cudaStream_t s = c->stream;
  // Whatever path returns, no copy may still read or write the caller's buffers afterwards.
  struct Drain {
    cudaStream_t trace, trace2, out, in;
    ~Drain() {
      cudaStreamSynchronize(trace);
      cudaStreamSynchronize(trace2);
      cudaStreamSynchronize(out);
      cudaStreamSynchronize(in);
    }
  } drain{s, c->trace2, c->copy_stream, c->h2d_stream};
  const int chunks = (int)std::min<long long>(4, std::max<long long>(1, total / kChunkPhotons));
  // Ranges weighted 1:3:...:3:1: the first range's upload and the last range's copy-out are the
  // ones not hidden behind a trace.
  long long bound[5], wts[4], wsum = 0, acc = 0;
  for (int k = 0; k < chunks; ++k) wsum += (wts[k] = (k == 0 || k == chunks - 1) ? 1 : 3);
  for (int k = 0; k <= chunks; ++k) {
    bound[k] = (k == chunks) ? total : total * acc / wsum;
    if (k < chunks) acc += wts[k];
  }
  // A host Y0 goes up range by range on its own stream.  The host checks it (every value
  // finite) while the ranges are traced, and a non-finite value fails the call before any result
  // is copied out: such a photon ends as a NUMERICAL_FAILURE at its first classification, so the
  // traces it reaches only run to completion.  (Checked before the launches, the scan of a
  // large sweep's Y0 held back the first trace by ~10 ms.)
  const double* d_Y0 = nullptr;
  if (host_Y0) {
    KRR_CUDA(c->buf[B_Y0].ensure((size_t)total * 8 * sizeof(double)));
    double* dst = static_cast<double*>(c->buf[B_Y0].p);
    for (int k = 0; k < chunks; ++k) {
      const size_t off = (size_t)bound[k] * 8, n = (size_t)(bound[k + 1] - bound[k]) * 8;
      KRR_CUDA(cudaMemcpyAsync(dst + off, host_Y0 + off, n * sizeof(double), cudaMemcpyHostToDevice, c->h2d_stream));
      KRR_CUDA(cudaEventRecord(c->h2d_ev[k], c->h2d_stream));
    }
    d_Y0 = dst;
  }
  Pipeline p;
  int rc = prepare_pipeline(c->device, images, (int)ims.size(), total, d_Y0, launch, d_out, d_work, work_size, p);
  if (rc) return rc;
  krr::Queue* qs[4] = {p.w.q0, p.w.q1, p.w.q2, p.w.q3};
  krr::Queue init[4];
  std::memset(init, 0, sizeof(init));
  KRR_CUDA(cudaMemcpyAsync(p.w.images, ims.data(), ims.size() * sizeof(krr::Image), cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemsetAsync(p.w.q0, 0, kQueueArea, s));
  for (int k = 0; k < chunks; ++k) {
    init[k].head = (unsigned long long)bound[k];
    KRR_CUDA(cudaMemcpyAsync(qs[k], &init[k], sizeof(krr::Queue), cudaMemcpyHostToDevice, s));
  }
  if (p.out.event_Y) KRR_CUDA(cudaMemsetAsync(p.out.event_Y, 0, (size_t)total * 8 * sizeof(double), s));
  if (p.out.event_hit) KRR_CUDA(cudaMemsetAsync(p.out.event_hit, 0, (size_t)total, s));
  // Consecutive ranges on alternate streams: a range's persistent blocks start on SMs that the
  // previous range's blocks leave in its tail (the ranges share no data; each has its own queue).
  KRR_CUDA(cudaEventRecord(c->ev0, s));
  KRR_CUDA(cudaEventRecord(c->fork_ev, s));
  KRR_CUDA(cudaStreamWaitEvent(c->trace2, c->fork_ev, 0));
  const cudaStream_t ts[2] = {s, c->trace2};
  for (int k = 0; k < chunks; ++k) {
    const cudaStream_t st = ts[k & 1];
    krr::PersistArgs a = p.main;
    a.q = qs[k];
    a.total = bound[k + 1];
    if (host_Y0) KRR_CUDA(cudaStreamWaitEvent(st, c->h2d_ev[k], 0));
    KRR_CUDA(p.main_v->run(a, st));
    KRR_CUDA(cudaEventRecord(c->chunk_ev[k], st));
  }
  for (int k = 1; k < chunks; k += 2) KRR_CUDA(cudaStreamWaitEvent(s, c->chunk_ev[k], 0));
  KRR_CUDA(cudaEventRecord(c->ev1, s));
  if (host_Y0 && !all_finite_parallel(host_Y0, (size_t)total * 8)) return fail(KRR_ERR_INVALID, "Y0 must be finite");
  // Every launch is queued before the first copy-out: a copy into pageable host memory returns
  // only when it has finished, and must not hold back the next range's launch.
  for (int k = 0; k < chunks; ++k) {
    KRR_CUDA(cudaStreamWaitEvent(c->copy_stream, c->chunk_ev[k], 0));
    rc = copy_rows_back(d_out, host_out, bound[k], bound[k + 1], c->copy_stream);
    if (rc) return rc;
  }
  krr::Queue q[4];
  std::memset(q, 0, sizeof(q));
  for (int k = 0; k < chunks; ++k) KRR_CUDA(cudaMemcpyAsync(&q[k], qs[k], sizeof(krr::Queue), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaStreamSynchronize(s));
  KRR_CUDA(cudaStreamSynchronize(c->copy_stream));
  KRR_CUDA(cudaStreamSynchronize(c->h2d_stream));
  float ms = 0.0f;
  KRR_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  krr::Queue sum{};
  for (int k = 0; k < chunks; ++k) {
    if (q[k].error) return fail(KRR_ERR_NOT_NULL, "tetrad projection is not null to 1e-10 (or no null momentum exists)");
    if (q[k].retired != (unsigned long long)(bound[k + 1] - bound[k]))
      return fail(KRR_ERR_CUDA, "work-queue inconsistency: %llu photons retired of %lld in range %d", q[k].retired,
                  bound[k + 1] - bound[k], k);
    sum.retired += q[k].retired;
    sum.attempts += q[k].attempts;
    sum.accepted += q[k].accepted;
    sum.lane_iters += q[k].lane_iters;
    sum.busy_iters += q[k].busy_iters;
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->photons = (uint64_t)total;
    stats->retired = sum.retired;
    stats->attempts = sum.attempts;
    stats->accepted = sum.accepted;
    stats->lane_slots = sum.lane_iters;
    stats->busy_slots = sum.busy_iters;
    stats->kernel_ms = ms;
  }
  return KRR_OK;
}

}  // namespace krr_host

using namespace krr_host;

struct krr_plan {
  int device;
  Pipeline p;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

extern "C" {

const char* krr_last_error(void) { return g_last_error.c_str(); }

int krr_abi_version(void) { return KRR_ABI_VERSION; }

int krr_device_count(int* count) {
  if (!count) return fail(KRR_ERR_INVALID, "count must not be NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *count = 0;
    return fail(KRR_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  *count = n;
  return KRR_OK;
}

int krr_max_attempts(const krr_options* options, int64_t* out) {
  int rc = validate_options(options);
  if (rc) return rc;
  if (!out) return fail(KRR_ERR_INVALID, "out must not be NULL");
  *out = max_attempts(options);
  return KRR_OK;
}

int krr_integrate_batch_device(int device, double mass, double spin, const double* d_Y0, const int64_t* d_index,
                               int64_t n, const krr_options* options, int32_t precision, const krr_result* d_out,
                               void* stream) {
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  rc = validate_options(options);
  if (rc) return rc;
  rc = check_precision(precision, options);
  if (rc) return rc;
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0, got %lld", (long long)n);
  if (n == 0) return KRR_OK;
  if (!d_Y0 || !d_out || !d_out->Y || !d_out->state) return fail(KRR_ERR_INVALID, "Y0, Y and state must not be NULL");
  KRR_CUDA(cudaSetDevice(device));
  krr::PlainArgs a{};
  a.P = make_params(mass, spin, options);
  a.images = nullptr;
  a.n_images = 0;
  a.Y0 = d_Y0;
  a.index = reinterpret_cast<const long long*>(d_index);
  a.n = n;
  a.o = to_outputs(d_out);
  a.q = nullptr;
  KRR_CUDA(launch_plain(precision, options, a, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_integrate_batch(int device, double mass, double spin, const double* Y0, int64_t n, const krr_options* options,
                        int32_t precision, const krr_result* out, double* runtime_s) {
  const auto t0 = std::chrono::steady_clock::now();
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  rc = validate_options(options);
  if (rc) return rc;
  rc = check_precision(precision, options);
  if (rc) return rc;
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0, got %lld", (long long)n);
  if (!out || (n > 0 && (!Y0 || !out->Y || !out->state))) return fail(KRR_ERR_INVALID, "Y0, Y and state must not be NULL");
  if (n > 0 && !all_finite(Y0, (size_t)n * 8)) return fail(KRR_ERR_INVALID, "Y0 must be finite");
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  if (n > 0) {
    KRR_CUDA(c->buf[B_Y0].ensure((size_t)n * 8 * sizeof(double)));
    KRR_CUDA(cudaMemcpyAsync(c->buf[B_Y0].p, Y0, (size_t)n * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double* d_Y0 = static_cast<const double*>(c->buf[B_Y0].p);
    krr_result dev;
    rc = device_results(c, n, out, options->disk_plane != 0, &dev);
    if (rc) return rc;
    krr::PlainArgs a{};
    a.P = make_params(mass, spin, options);
    a.Y0 = d_Y0;
    a.n = n;
    a.o = to_outputs(&dev);
    KRR_CUDA(launch_plain(precision, options, a, c->stream));
    rc = copy_results_back(c, n, &dev, out);
    if (rc) return rc;
    KRR_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (runtime_s) runtime_s[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return KRR_OK;
}

int krr_disk_shading(int device, double mass, double spin, int32_t prograde, double r_in, double r_out,
                     double emissivity_index, int32_t redshift_power, const double* d_event_Y, const uint8_t* d_hit,
                     int64_t n, double* d_g, double* d_intensity, double* d_r_hit, void* stream) {
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  if (!(std::isfinite(r_in) && std::isfinite(r_out) && 0.0 < r_in && r_in < r_out))
    return fail(KRR_ERR_INVALID, "need 0 < r_in < r_out, got r_in=%g, r_out=%g", r_in, r_out);
  if (!std::isfinite(emissivity_index)) return fail(KRR_ERR_INVALID, "emissivity_index must be finite");
  if (redshift_power != 3 && redshift_power != 4)
    return fail(KRR_ERR_INVALID, "redshift_power must be 3 or 4, got %d", redshift_power);
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0");
  if (n == 0) return KRR_OK;
  if (!d_event_Y || !d_hit || !d_g || !d_intensity || !d_r_hit) return fail(KRR_ERR_INVALID, "device buffers must not be NULL");
  KRR_CUDA(cudaSetDevice(device));
  KRR_CUDA(krr::disk_shading(mass, spin * mass, prograde != 0, r_in, r_out, emissivity_index, redshift_power, d_event_Y,
                             d_hit, n, d_g, d_intensity, d_r_hit, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_trig_eval(int device, int32_t which, const double* d_theta, const double* d_delta, int64_t n, double* d_sin,
                  double* d_cos, void* stream) {
  if (which < 0 || which > 2) return fail(KRR_ERR_INVALID, "which must be 0, 1 or 2, got %d", which);
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0");
  if (n == 0) return KRR_OK;
  if (!d_theta || !d_sin || !d_cos || (which != 0 && !d_delta))
    return fail(KRR_ERR_INVALID, "device buffers must not be NULL (d_delta may be NULL only for which 0)");
  KRR_CUDA(cudaSetDevice(device));
  KRR_CUDA(krr::trig_eval(which, d_theta, d_delta, n, d_sin, d_cos, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_escape_directions(int device, double mass, double spin, double r_surface, const double* d_Y,
                          const int64_t* d_state, int64_t n, double* d_theta, double* d_phi, void* stream) {
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0");
  if (!(r_surface > 0.0)) return fail(KRR_ERR_INVALID, "r_surface must be > 0, got %g", r_surface);
  if (n == 0) return KRR_OK;
  if (!d_Y || !d_state || !d_theta || !d_phi) return fail(KRR_ERR_INVALID, "device buffers must not be NULL");
  krr_options o{};
  o.rtol = 1e-6;
  o.atol = 1e-8;
  o.step_size = 0.01;
  o.max_steps = 1;
  o.lambda_max = 1.0;
  o.h_min = 1e-12;
  o.h_max = 1.0;
  o.escape_radius = r_surface;
  const krr::Params P = make_params(mass, spin, &o);
  KRR_CUDA(cudaSetDevice(device));
  KRR_CUDA(krr::escape_directions(P, r_surface, d_Y, reinterpret_cast<const long long*>(d_state), n, d_theta, d_phi,
                                  static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_camera_states(int device, double mass, double spin, const krr_camera* camera, const double* alpha,
                      const double* beta, int64_t n, double* Y0) {
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  krr::Frame F{};
  rc = make_frame(mass, spin, camera, F);
  if (rc) return rc;
  const bool grid = alpha == nullptr && beta == nullptr;
  if (!grid && (!alpha || !beta)) return fail(KRR_ERR_INVALID, "alpha and beta must both be given or both be NULL");
  long long rows = n;
  if (grid) {
    rc = validate_grid(camera);
    if (rc) return rc;
    rows = camera->resolution * camera->resolution;
  } else {
    if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0");
    for (int64_t i = 0; i < n; ++i)
      if (!((alpha[i] * alpha[i] + beta[i] * beta[i]) / (camera->radius * camera->radius) < 1.0))
        return fail(KRR_ERR_INVALID, "image points with alpha^2 + beta^2 >= radius^2 are not directions on the observer's sky");
  }
  if (!Y0 && rows > 0) return fail(KRR_ERR_INVALID, "Y0 must not be NULL");
  if (rows == 0) return KRR_OK;
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  KRR_CUDA(c->buf[B_Y0].ensure((size_t)rows * 8 * sizeof(double)));
  KRR_CUDA(c->buf[B_ERR].ensure(16));
  KRR_CUDA(cudaMemsetAsync(c->buf[B_ERR].p, 0, 16, c->stream));
  double* d_a = nullptr;
  double* d_b = nullptr;
  if (!grid) {
    KRR_CUDA(c->buf[B_AB].ensure((size_t)rows * 2 * sizeof(double)));
    d_a = static_cast<double*>(c->buf[B_AB].p);
    d_b = d_a + rows;
    KRR_CUDA(cudaMemcpyAsync(d_a, alpha, (size_t)rows * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KRR_CUDA(cudaMemcpyAsync(d_b, beta, (size_t)rows * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  KRR_CUDA(krr::camera_states(F, camera->fov, camera->resolution, d_a, d_b, rows, static_cast<double*>(c->buf[B_Y0].p),
                              static_cast<int*>(c->buf[B_ERR].p), c->stream));
  int err = 0;
  KRR_CUDA(cudaMemcpyAsync(&err, c->buf[B_ERR].p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  KRR_CUDA(cudaMemcpyAsync(Y0, c->buf[B_Y0].p, (size_t)rows * 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  KRR_CUDA(cudaStreamSynchronize(c->stream));
  if (err) return fail(KRR_ERR_NOT_NULL, "tetrad projection is not null to 1e-10 (or no null momentum exists)");
  return KRR_OK;
}

int krr_list_variants(int device, int32_t precision, const krr_options* options, krr_variant_info* out,
                      int32_t max_out, int32_t* count) {
  int rc = validate_options(options);
  if (rc) return rc;
  rc = check_precision(precision, options);
  if (rc) return rc;
  if (!count) return fail(KRR_ERR_INVALID, "count must not be NULL");
  int n = 0;
  const krr::Variant* vs = variants_for(precision, options, &n);
  *count = n;
  if (!out) return KRR_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(KRR_ERR_NO_DEVICE, "no CUDA device available");
  KRR_CUDA(cudaSetDevice(device));
  for (int i = 0; i < n && i < max_out; ++i) {
    out[i].block = vs[i].block;
    out[i].min_blocks = vs[i].min_blocks;
    out[i].registers = vs[i].registers();
    out[i].blocks_per_sm = vs[i].occupancy();
  }
  return KRR_OK;
}

size_t krr_workspace_size(int32_t n_images, int64_t retrace_photons) { return work_bytes(n_images, retrace_photons); }

int krr_analytic_classes(double mass, double spin, double rtol, double horizon_epsilon, const double* Y0, int64_t n,
                         uint8_t* out) {
  int rc = validate_spacetime(mass, spin);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!Y0 || !out))) return fail(KRR_ERR_INVALID, "Y0 and out must hold n >= 0 rows");
  if (!(rtol > 0.0) || !(horizon_epsilon >= 0.0)) return fail(KRR_ERR_INVALID, "rtol must be > 0 and horizon_epsilon >= 0");
  const double a = spin * mass;
  const double r_capture = outer_horizon(mass, a) + horizon_epsilon;
  const double band = krr::risk_band(mass, rtol);
  for (int64_t i = 0; i < n; ++i) out[i] = (uint8_t)krr::radial_risk(mass, a, r_capture, Y0 + 8 * i, band);
  return KRR_OK;
}

int krr_trace_images_device(int device, const krr_image* images, int32_t n_images, const double* d_Y0,
                            const krr_launch* launch, const krr_result* d_out, void* workspace, size_t workspace_bytes,
                            void* stream, krr_stats* stats) {
  std::vector<krr::Image> ims;
  long long total = 0;
  int rc = build_images(images, n_images, ims, total);
  if (rc) return rc;
  if (!d_out || !d_out->Y || !d_out->state || !workspace) return fail(KRR_ERR_INVALID, "Y, state and workspace must not be NULL");
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  return run_images(c, images, ims, total, d_Y0, launch, d_out, workspace, workspace_bytes,
                    static_cast<cudaStream_t>(stream), stats);
}

int krr_plan_create(int device, const krr_image* images, int32_t n_images, const double* d_Y0, const krr_launch* launch,
                    const krr_result* d_out, void* workspace, size_t workspace_bytes, krr_plan** plan) {
  if (!plan) return fail(KRR_ERR_INVALID, "plan must not be NULL");
  *plan = nullptr;
  std::vector<krr::Image> ims;
  long long total = 0;
  int rc = build_images(images, n_images, ims, total);
  if (rc) return rc;
  if (!d_out || !d_out->Y || !d_out->state || !workspace) return fail(KRR_ERR_INVALID, "Y, state and workspace must not be NULL");
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  auto pl = std::make_unique<krr_plan>();
  pl->device = device;
  rc = prepare_pipeline(device, images, n_images, total, d_Y0, launch, d_out, workspace, workspace_bytes, pl->p);
  if (rc) return rc;
  // The caller may still be filling `workspace` (or the outputs) on a stream of its own -- e.g.
  // the asynchronous zero fill of a freshly allocated buffer: wait for the device before the
  // upload, which goes through this library's stream and is ordered after nothing else.
  KRR_CUDA(cudaDeviceSynchronize());
  KRR_CUDA(cudaMemcpyAsync(pl->p.w.images, ims.data(), ims.size() * sizeof(krr::Image), cudaMemcpyHostToDevice, c->stream));
  KRR_CUDA(cudaStreamSynchronize(c->stream));
  KRR_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e = enqueue_pipeline(pl->p, c->stream, nullptr, nullptr, nullptr);
  cudaGraph_t graph = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return fail(KRR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e3 = cudaGraphInstantiate(&exec, graph, 0);
  if (e3 != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(KRR_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e3));
  }
  pl->graph = graph;
  pl->exec = exec;
  *plan = pl.release();
  return KRR_OK;
}

int krr_plan_launch(krr_plan* plan, void* stream) {
  if (!plan) return fail(KRR_ERR_INVALID, "plan must not be NULL");
  KRR_CUDA(cudaSetDevice(plan->device));
  KRR_CUDA(cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_plan_stats(krr_plan* plan, void* stream, krr_stats* stats) {
  if (!plan) return fail(KRR_ERR_INVALID, "plan must not be NULL");
  KRR_CUDA(cudaSetDevice(plan->device));
  return finish_pipeline(plan->p, static_cast<cudaStream_t>(stream), stats, nullptr, nullptr, nullptr);
}

int krr_plan_destroy(krr_plan* plan) {
  if (!plan) return KRR_OK;
  cudaSetDevice(plan->device);
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  delete plan;
  return KRR_OK;
}

// The lensing workspace: step sizes (n, cap), checkpoints (n, cap / K + 1, 6), landed final
// states (n, 16), the stage tape's chunk table (n, cap / STAGE_CHUNK + 1) int32, staged flags (n),
// the chunk counter, then the pool: every whole chunk that fits in the bytes that remain.  Every
// offset is a multiple of 256 B (the bulk copies into the pool need 16 B alignment).
struct LensLayout {
  size_t h, ck, rec, tab, staged, counter, pool;
};
static LensLayout lens_layout(int64_t n, int32_t cap, int32_t K) {
  LensLayout l{};
  size_t o = 0;
  l.h = o;
  o += round256((size_t)n * cap * 8);
  l.ck = o;
  o += round256((size_t)n * (cap / K + 1) * 6 * 8);
  l.rec = o;
  o += round256((size_t)n * 16 * 8);
  l.tab = o;
  o += round256((size_t)n * (cap / krr::STAGE_CHUNK + 1) * 4);
  l.staged = o;
  o += round256((size_t)n);
  l.counter = o;
  o += 256;
  l.pool = o;
  return l;
}
static constexpr size_t kStageChunkBytes = (size_t)krr::STAGE_CHUNK * krr::STEP_REC * 8;

size_t krr_lensing_workspace_size(int64_t n, int32_t tape_capacity, int32_t checkpoint_every) {
  if (n < 0 || tape_capacity < 1 || checkpoint_every < 1) return 0;
  return lens_layout(n, tape_capacity, checkpoint_every).pool;
}

size_t krr_lensing_workspace_size_staged(int64_t n, int32_t tape_capacity, int32_t checkpoint_every,
                                         int64_t stage_steps) {
  if (n < 0 || tape_capacity < 1 || checkpoint_every < 1 || stage_steps < 0) return 0;
  const size_t base = lens_layout(n, tape_capacity, checkpoint_every).pool;
  if (stage_steps == 0 || n == 0) return base;
  const size_t chunks = (size_t)((stage_steps + krr::STAGE_CHUNK - 1) / krr::STAGE_CHUNK) + (size_t)n;
  return base + chunks * kStageChunkBytes;
}

static int lens_launch(const krr_lens_params* p, int64_t n, krr::LensLaunch& L, size_t workspace_bytes) {
  if (!p) return fail(KRR_ERR_INVALID, "params must not be NULL");
  int rc = validate_spacetime(p->mass, p->spin);
  if (!rc) rc = validate_options(&p->options);
  if (rc) return rc;
  if (p->options.method != 0 || p->options.dtype != 0 || p->options.disk_plane)
    return fail(KRR_ERR_UNSUPPORTED, "the lensing adjoint integrates with rk45 in float64 without events");
  if (p->checkpoint_every < 1 || p->checkpoint_every > 64)
    return fail(KRR_ERR_INVALID, "checkpoint_every must lie in [1, 64], got %d", p->checkpoint_every);
  if (p->tape_capacity < 1) return fail(KRR_ERR_INVALID, "tape_capacity must be >= 1");
  if (n < 0) return fail(KRR_ERR_INVALID, "n must be >= 0");
  if (workspace_bytes < krr_lensing_workspace_size(n, p->tape_capacity, p->checkpoint_every))
    return fail(KRR_ERR_INVALID, "workspace too small for the tape");
  krr_camera cam{p->radius, p->inclination_deg, p->phi_deg, 1.0, 2};
  krr::Frame F{};
  rc = make_frame(p->mass, p->spin, &cam, F);
  if (rc) return rc;
  L.P = make_params(p->mass, p->spin, &p->options);
  L.spin = p->spin;
  L.mass = p->mass;
  L.r_o = F.r_o;
  L.th_o = F.th_o;
  L.ph_o = F.ph_o;
  L.K = p->checkpoint_every;
  L.cap = p->tape_capacity;
  L.n = n;
  return KRR_OK;
}

int krr_lensing_adjoint(int device, const krr_lens_params* params, const double* d_alpha, const double* d_beta,
                        int64_t n, double* d_theta, double* d_phi, double* d_jac, int64_t* d_state, int64_t* d_n_steps,
                        int32_t* d_status, void* workspace, size_t workspace_bytes, void* stream) {
  krr::LensLaunch L{};
  int rc = lens_launch(params, n, L, workspace_bytes);
  if (rc) return rc;
  if (n == 0) return KRR_OK;
  if (!d_alpha || !d_beta || !d_theta || !d_phi || !d_jac || !d_state || !d_n_steps || !d_status || !workspace)
    return fail(KRR_ERR_INVALID, "device buffers must not be NULL");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(KRR_ERR_INVALID, "the workspace must be 256-byte aligned (as cudaMalloc returns it)");
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  L.aux = c->lens_aux;
  L.ev_fork = c->lens_fork;
  L.ev_join = c->lens_join;
  L.alpha = d_alpha;
  L.beta = d_beta;
  L.theta = d_theta;
  L.phi = d_phi;
  L.jac = d_jac;
  L.state = reinterpret_cast<long long*>(d_state);
  L.n_steps = reinterpret_cast<long long*>(d_n_steps);
  L.status = d_status;
  char* w = static_cast<char*>(workspace);
  const LensLayout lay = lens_layout(n, L.cap, L.K);
  L.tape_h = reinterpret_cast<double*>(w + lay.h);
  L.tape_ck = reinterpret_cast<double*>(w + lay.ck);
  L.final_rec = reinterpret_cast<double*>(w + lay.rec);
  L.chunk_tab = reinterpret_cast<int*>(w + lay.tab);
  L.staged = reinterpret_cast<unsigned char*>(w + lay.staged);
  L.pool_next = reinterpret_cast<unsigned long long*>(w + lay.counter);
  L.pool = reinterpret_cast<double*>(w + lay.pool);
  L.pool_chunks = (long long)((workspace_bytes - lay.pool) / kStageChunkBytes);
  KRR_CUDA(krr::lensing_adjoint(L, false, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_lensing_tape_usage(const krr_lens_params* params, int64_t n, const void* workspace, size_t workspace_bytes,
                           int64_t* staged_rays, int64_t* chunks_used, int64_t* chunks_total, void* stream) {
  krr::LensLaunch L{};
  int rc = lens_launch(params, n, L, workspace_bytes);
  if (rc) return rc;
  if (!staged_rays || !chunks_used || !chunks_total) return fail(KRR_ERR_INVALID, "outputs must not be NULL");
  const LensLayout lay = lens_layout(n, L.cap, L.K);
  *chunks_total = (int64_t)((workspace_bytes - lay.pool) / kStageChunkBytes);
  *staged_rays = 0;
  *chunks_used = 0;
  if (n == 0) return KRR_OK;
  if (!workspace) return fail(KRR_ERR_INVALID, "workspace must not be NULL");
  const char* w = static_cast<const char*>(workspace);
  std::vector<unsigned char> flags((size_t)n);
  unsigned long long used = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  KRR_CUDA(cudaMemcpyAsync(flags.data(), w + lay.staged, (size_t)n, cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(&used, w + lay.counter, sizeof(used), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaStreamSynchronize(s));
  int64_t k = 0;
  for (unsigned char f : flags) k += f ? 1 : 0;
  *staged_rays = k;
  *chunks_used = (int64_t)std::min<unsigned long long>(used, (unsigned long long)*chunks_total);
  return KRR_OK;
}

int krr_lensing_replay(int device, const krr_lens_params* params, const double* d_alpha, const double* d_beta,
                       int64_t n, const int64_t* d_state, const int64_t* d_n_steps, double* d_theta, double* d_phi,
                       int32_t* d_status, const void* workspace, size_t workspace_bytes, void* stream) {
  krr::LensLaunch L{};
  int rc = lens_launch(params, n, L, workspace_bytes);
  if (rc) return rc;
  if (n == 0) return KRR_OK;
  if (!d_alpha || !d_beta || !d_theta || !d_phi || !d_state || !d_n_steps || !d_status || !workspace)
    return fail(KRR_ERR_INVALID, "device buffers must not be NULL");
  KRR_CUDA(cudaSetDevice(device));
  L.alpha = d_alpha;
  L.beta = d_beta;
  L.theta = d_theta;
  L.phi = d_phi;
  L.state = const_cast<long long*>(reinterpret_cast<const long long*>(d_state));
  L.n_steps = const_cast<long long*>(reinterpret_cast<const long long*>(d_n_steps));
  L.status = d_status;
  L.tape_h = const_cast<double*>(static_cast<const double*>(workspace));
  KRR_CUDA(krr::lensing_adjoint(L, true, static_cast<cudaStream_t>(stream)));
  return KRR_OK;
}

int krr_bisect_edges(int device, const krr_edge_case* cases, int32_t n_cases, const int32_t* item_case,
                     const double* cos_phi, const double* sin_phi, double* lo, double* hi, int64_t* failures,
                     int64_t n_items, int32_t iterations, int32_t precision, krr_stats* stats) {
  if (!cases || n_cases < 1) return fail(KRR_ERR_INVALID, "need at least one case");
  if (n_items < 0 || iterations < 0) return fail(KRR_ERR_INVALID, "n_items and iterations must be >= 0");
  if (n_items > 0 && (!item_case || !cos_phi || !sin_phi || !lo || !hi))
    return fail(KRR_ERR_INVALID, "item_case, cos_phi, sin_phi, lo and hi must not be NULL");
  std::vector<krr::EdgeCase> ec(n_cases);
  for (int k = 0; k < n_cases; ++k) {
    const krr_edge_case& c = cases[k];
    int rc = validate_spacetime(c.mass, c.spin);
    if (!rc) rc = validate_options(&c.options);
    if (!rc) rc = check_precision(precision, &c.options);
    if (rc) return rc;
    if (c.options.method != 0 || c.options.disk_plane)
      return fail(KRR_ERR_UNSUPPORTED, "the edge bisection integrates with rk45 and no events");
    krr_camera cam{c.radius, c.inclination_deg, c.phi_deg, 1.0, 2};
    rc = make_frame(c.mass, c.spin, &cam, ec[k].F);
    if (rc) return rc;
    ec[k].P = make_params(c.mass, c.spin, &c.options);
    ec[k].c_alpha = c.centre_alpha;
    ec[k].c_beta = c.centre_beta;
  }
  for (int64_t i = 0; i < n_items; ++i) {
    const int c = item_case[i];
    if (c < 0 || c >= n_cases) return fail(KRR_ERR_INVALID, "item_case[%lld] = %d out of range", (long long)i, c);
    if (!(std::isfinite(lo[i]) && std::isfinite(hi[i]) && std::isfinite(cos_phi[i]) && std::isfinite(sin_phi[i])))
      return fail(KRR_ERR_INVALID, "brackets and directions must be finite");
    // Every bisection point lies between the bracket ends: both must be directions on the sky.
    const double r2 = cases[c].radius * cases[c].radius;
    for (double rho : {lo[i], hi[i]}) {
      const double al = cases[c].centre_alpha + rho * cos_phi[i], be = cases[c].centre_beta + rho * sin_phi[i];
      if (!((al * al + be * be) / r2 < 1.0))
        return fail(KRR_ERR_INVALID, "image points with alpha^2 + beta^2 >= radius^2 are not directions on the sky");
    }
  }
  if (n_items == 0) return KRR_OK;
  Context* ctx = nullptr;
  int rc = get_context(device, &ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KRR_CUDA(cudaSetDevice(device));
  // Queue order: the cases' items dealt round robin, so that every warp holds items of every
  // tolerance, and the cheap ones, ending early, lend their lanes to the expensive ones.  That
  // needs the cases' parameters in shared memory (krr::edge_params_in_smem); with more cases
  // the items keep their order, and a warp's lanes mostly share a case.
  const bool interleave = krr::edge_params_in_smem(n_cases);
  std::vector<long long> order((size_t)n_items);
  for (int64_t i = 0; i < n_items; ++i) order[(size_t)i] = i;
  if (interleave) {
    std::vector<long long> start((size_t)n_cases + 1, 0), fill((size_t)n_cases, 0);
    for (int64_t i = 0; i < n_items; ++i) start[(size_t)item_case[i] + 1] += 1;
    for (int k = 0; k < n_cases; ++k) start[(size_t)k + 1] += start[(size_t)k];
    std::vector<long long> by_case((size_t)n_items);
    for (int64_t i = 0; i < n_items; ++i) {
      const int k = item_case[i];
      by_case[(size_t)(start[(size_t)k] + fill[(size_t)k]++)] = i;
    }
    size_t n = 0;
    for (long long r = 0; n < (size_t)n_items; ++r)
      for (int k = 0; k < n_cases; ++k)
        if (start[(size_t)k] + r < start[(size_t)k + 1]) order[n++] = by_case[(size_t)(start[(size_t)k] + r)];
  }
  const size_t nb8 = (size_t)n_items * 8, nb4 = (size_t)n_items * 4;
  const size_t bytes = 512 + round256((size_t)n_cases * sizeof(krr::EdgeCase)) + 6 * round256(nb8) + round256(nb4);
  KRR_CUDA(ctx->buf[B_AB].ensure(bytes));
  char* base = static_cast<char*>(ctx->buf[B_AB].p);
  krr::Queue* d_q = reinterpret_cast<krr::Queue*>(base);
  size_t off = 512;
  auto take = [&](size_t n) { char* p = base + off; off += round256(n); return p; };
  auto* d_cases = reinterpret_cast<krr::EdgeCase*>(take((size_t)n_cases * sizeof(krr::EdgeCase)));
  auto* d_item = reinterpret_cast<int*>(take(nb4));
  auto* d_cos = reinterpret_cast<double*>(take(nb8));
  auto* d_sin = reinterpret_cast<double*>(take(nb8));
  auto* d_lo = reinterpret_cast<double*>(take(nb8));
  auto* d_hi = reinterpret_cast<double*>(take(nb8));
  auto* d_fail = reinterpret_cast<long long*>(take(nb8));
  auto* d_order = reinterpret_cast<long long*>(take(nb8));
  const cudaStream_t s = ctx->stream;
  KRR_CUDA(cudaMemsetAsync(d_q, 0, sizeof(krr::Queue), s));
  KRR_CUDA(cudaMemcpyAsync(d_cases, ec.data(), ec.size() * sizeof(krr::EdgeCase), cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_item, item_case, nb4, cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_cos, cos_phi, nb8, cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_sin, sin_phi, nb8, cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_lo, lo, nb8, cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_hi, hi, nb8, cudaMemcpyHostToDevice, s));
  KRR_CUDA(cudaMemcpyAsync(d_order, order.data(), nb8, cudaMemcpyHostToDevice, s));
  krr::EdgeArgs a{};
  a.cases = d_cases;
  a.item_case = d_item;
  a.cos_phi = d_cos;
  a.sin_phi = d_sin;
  a.lo = d_lo;
  a.hi = d_hi;
  a.failures = d_fail;
  a.order = d_order;
  a.n_cases = n_cases;
  a.n_items = n_items;
  a.iterations = iterations;
  a.q = d_q;
  a.refill_threshold = 1;
  KRR_CUDA(cudaEventRecord(ctx->ev0, s));
  KRR_CUDA(precision == KRR_PREC_REFERENCE ? krr::ref_bisect(a, s) : krr::fast_bisect(precision == KRR_PREC_MIXED, a, s));
  KRR_CUDA(cudaEventRecord(ctx->ev1, s));
  krr::Queue q{};
  KRR_CUDA(cudaMemcpyAsync(&q, d_q, sizeof(q), cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(lo, d_lo, nb8, cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaMemcpyAsync(hi, d_hi, nb8, cudaMemcpyDeviceToHost, s));
  if (failures) KRR_CUDA(cudaMemcpyAsync(failures, d_fail, nb8, cudaMemcpyDeviceToHost, s));
  KRR_CUDA(cudaStreamSynchronize(s));
  float ms = 0.0f;
  KRR_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->photons = (uint64_t)n_items * (uint64_t)iterations;
    stats->retired = q.retired;
    stats->attempts = q.attempts - q.discarded;  // the sequential bisection's attempts
    stats->accepted = q.accepted;
    stats->lane_slots = q.lane_iters;
    stats->busy_slots = q.busy_iters;             // every attempt run, discarded ones included
    stats->kernel_ms = ms;
    stats->speculative = q.speculative;
    stats->discarded_attempts = q.discarded;
  }
  if (q.error) return fail(KRR_ERR_NOT_NULL, "tetrad projection is not null to 1e-10 (or no null momentum exists)");
  if (q.retired != (unsigned long long)n_items)
    return fail(KRR_ERR_CUDA, "work-queue inconsistency: %llu items retired of %lld", q.retired, (long long)n_items);
  return KRR_OK;
}

int krr_trace_images(int device, const krr_image* images, int32_t n_images, const double* Y0, const krr_launch* launch,
                     const krr_result* out, krr_stats* stats) {
  std::vector<krr::Image> ims;
  long long total = 0;
  int rc = build_images(images, n_images, ims, total);
  if (rc) return rc;
  if (!out || !out->Y || !out->state) return fail(KRR_ERR_INVALID, "Y and state must not be NULL");
  Context* c = nullptr;
  rc = get_context(device, &c);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(c->mu);
  KRR_CUDA(cudaSetDevice(device));
  const bool overlapped = total >= 2 * kChunkPhotons && !(launch && (launch->retrace || launch->plain));
  const double* d_Y0 = nullptr;
  if (Y0 && !overlapped) {
    rc = upload_y0(c, Y0, total, &d_Y0);
    if (rc) return rc;
  }
  krr_result dev;
  rc = device_results(c, total, out, images[0].options.disk_plane != 0, &dev);
  if (rc) return rc;
  const size_t wbytes = work_bytes(n_images, (launch && launch->retrace) ? total : 0);
  KRR_CUDA(c->buf[B_QUEUE].ensure(wbytes));
  if (overlapped)
    return run_images_overlapped(c, images, ims, total, Y0, launch, &dev, out, c->buf[B_QUEUE].p, wbytes, stats);
  rc = run_images(c, images, ims, total, d_Y0, launch, &dev, c->buf[B_QUEUE].p, wbytes, c->stream, stats);
  if (rc) return rc;
  rc = copy_results_back(c, total, &dev, out);
  if (rc) return rc;
  KRR_CUDA(cudaStreamSynchronize(c->stream));
  return KRR_OK;
}

}  // extern "C"
