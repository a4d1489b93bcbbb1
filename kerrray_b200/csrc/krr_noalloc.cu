// krr_trace_images_noalloc: the batched persistent trace for callers that cannot allocate
// device memory.
//
// Some callers must not call cudaMalloc or any allocating routine on the path they run: a
// host application with its own device-memory pool (a renderer or a serving process that
// budgets every byte up front and forbids allocations after start-up), or a plug-in whose host
// framework owns all device memory.  This entry point takes the caller's inputs and outputs and
// keeps the launch's scratch -- the work-queue counters and the image descriptors -- in a fixed
// array in this library's device image, so it allocates nothing.  The array is sized for
// KRR_NOALLOC_MAX_IMAGES images; every GPU that loads the library holds it (the queue plus 128
// descriptors of 368 B: about 47 KB) until the process exits.
//
// The call is synchronous: it uploads the descriptors from a host stack buffer, reads the
// counters back and synchronises the stream.  It therefore cannot run inside a stream capture,
// and refuses a stream that is capturing.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/kerrray_cuda.h"
#include "krr_host.h"
#include "krr_launch.h"

namespace {

constexpr size_t kQueueBytes = (sizeof(krr::Queue) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kQueueBytes + (size_t)KRR_NOALLOC_MAX_IMAGES * sizeof(krr::Image);

// The launch scratch: queue counters first, then the image descriptors.  In host code this
// name is only a stand-in for the device array; its device address comes from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current), looked up once per
// device on the first call.
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return krr_host::fail(KRR_ERR_INVALID, "device %d out of range", device);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return krr_host::fail(KRR_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return KRR_OK;
}

}  // namespace

extern "C" int krr_trace_images_noalloc(int device, const krr_image* images, int32_t n_images, const double* d_Y0,
                                        const krr_launch* launch, const krr_result* d_out, void* stream,
                                        krr_stats* stats) {
  using namespace krr_host;
  if (!images || n_images < 1) return fail(KRR_ERR_INVALID, "need at least one image");
  if (n_images > KRR_NOALLOC_MAX_IMAGES)
    return fail(KRR_ERR_INVALID, "krr_trace_images_noalloc takes at most %d images (got %d); use krr_trace_images_device",
                KRR_NOALLOC_MAX_IMAGES, n_images);
  if (!d_out || !d_out->Y || !d_out->state) return fail(KRR_ERR_INVALID, "Y and state must not be NULL");
  if (launch && (launch->plain || launch->retrace))
    return fail(KRR_ERR_UNSUPPORTED, "krr_trace_images_noalloc runs the persistent kernel only, without the re-trace");
  const int32_t precision = launch ? launch->precision : KRR_PREC_FAST64;
  // Descriptors are built in a fixed host buffer: no heap allocation either.
  krr::Image ims[KRR_NOALLOC_MAX_IMAGES];
  long long total = 0;
  for (int k = 0; k < n_images; ++k) {
    const krr_image& im = images[k];
    int rc = validate_spacetime(im.mass, im.spin);
    if (!rc) rc = validate_options(&im.options);
    if (!rc) rc = make_frame(im.mass, im.spin, &im.camera, ims[k].F);
    if (!rc) rc = validate_grid(&im.camera);
    if (rc) return rc;
    if (im.options.method != images[0].options.method || im.options.dtype != images[0].options.dtype)
      return fail(KRR_ERR_UNSUPPORTED, "all images of one launch must share method and dtype");
    rc = pixel_range(im, &ims[k].first, &ims[k].count);
    if (rc) return rc;
    ims[k].P = make_params(im.mass, im.spin, &im.options);
    ims[k].fov = im.camera.fov;
    ims[k].res = im.camera.resolution;
    ims[k].offset = total;
    total += ims[k].count;
  }
  int rc = check_precision(precision, &images[0].options);
  if (rc) return rc;
  int count = 0;
  const krr::Variant* vs = variants_for(precision, &images[0].options, &count);
  const int idx = (launch && launch->variant > 0) ? launch->variant : 0;
  if (!vs || idx >= count) return fail(KRR_ERR_INVALID, "launch variant %d out of range [0, %d)", idx, count);
  if (cudaSetDevice(device) != cudaSuccess) return fail(KRR_ERR_NO_DEVICE, "cannot select device %d", device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &capturing) != cudaSuccess || capturing != cudaStreamCaptureStatusNone)
    return fail(KRR_ERR_UNSUPPORTED, "krr_trace_images_noalloc synchronises its stream and cannot run during a stream capture");
  void* scratch = nullptr;
  rc = scratch_address(device, &scratch);
  if (rc) return rc;
  krr::Queue* d_q = static_cast<krr::Queue*>(scratch);
  krr::Image* d_images = reinterpret_cast<krr::Image*>(static_cast<unsigned char*>(scratch) + kQueueBytes);
  cudaError_t e = cudaMemcpyAsync(d_images, ims, (size_t)n_images * sizeof(krr::Image), cudaMemcpyHostToDevice, s);
  // The counters keep the previous call's values: clear them before every launch.
  if (e == cudaSuccess) e = cudaMemsetAsync(d_q, 0, sizeof(krr::Queue), s);
  // The kernel writes the disk-event outputs only for rays that hit the disk: clear them first,
  // as the workspace entry point does.
  if (e == cudaSuccess && d_out->event_Y) e = cudaMemsetAsync(d_out->event_Y, 0, (size_t)total * 8 * sizeof(double), s);
  if (e == cudaSuccess && d_out->event_hit) e = cudaMemsetAsync(d_out->event_hit, 0, (size_t)total, s);
  if (e != cudaSuccess) return fail(KRR_ERR_CUDA, "scratch upload: %s", cudaGetErrorString(e));
  const int occ = vs[idx].occupancy();
  if (occ < 1) return fail(KRR_ERR_CUDA, "persistent kernel variant %d cannot be resident", idx);
  krr::PersistArgs a{};
  a.images = d_images;
  a.n_images = n_images;
  a.total = total;
  a.Y0 = d_Y0;
  a.o = to_outputs(d_out);
  a.q = d_q;
  a.refill_threshold = (launch && launch->refill_threshold > 0) ? (launch->refill_threshold < 32 ? launch->refill_threshold : 32) : 1;
  a.grid = sm_count_of(device) * ((launch && launch->blocks_per_sm > 0 && launch->blocks_per_sm < occ) ? launch->blocks_per_sm : occ);
  a.block = vs[idx].block;
  e = vs[idx].run(a, s);
  if (e != cudaSuccess) return fail(KRR_ERR_CUDA, "persistent kernel launch: %s", cudaGetErrorString(e));
  krr::Queue q;
  std::memset(&q, 0, sizeof(q));
  e = cudaMemcpyAsync(&q, d_q, sizeof(q), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(KRR_ERR_CUDA, "persistent kernel: %s", cudaGetErrorString(e));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->photons = (uint64_t)total;
    stats->retired = q.retired;
    stats->attempts = q.attempts;
    stats->accepted = q.accepted;
    stats->lane_slots = q.lane_iters;
    stats->busy_slots = q.busy_iters;
  }
  if (q.error) return fail(KRR_ERR_NOT_NULL, "tetrad projection is not null to 1e-10 (or no null momentum exists)");
  if (q.retired != (unsigned long long)total)
    return fail(KRR_ERR_CUDA, "work-queue inconsistency: %llu photons retired of %lld", q.retired, total);
  return KRR_OK;
}
