// Kernels in the reference's operation order.  This translation unit is compiled with
// -fmad=false: every product and sum is rounded separately, as in KerrRay's Numba kernel
// (fastmath=False, src/kerrray/raytracing/backends/numba_kernel.py:466).
#include "krr_launch.h"

namespace krr {

cudaError_t ref_plain(bool dtype32, bool rk4, const PlainArgs& a, int block, cudaStream_t s) {
  if (dtype32) return rk4 ? run_plain<RefMode<float>, true>(a, block, s) : run_plain<RefMode<float>, false>(a, block, s);
  return rk4 ? run_plain<RefMode<double>, true>(a, block, s) : run_plain<RefMode<double>, false>(a, block, s);
}

const Variant* ref_variants(bool dtype32, bool rk4, int* count) {
  static const Variant v64[] = {make_variant<RefMode<double>, false, 128, 1>()};
  static const Variant v64rk4[] = {make_variant<RefMode<double>, true, 128, 1>()};
  static const Variant v32[] = {make_variant<RefMode<float>, false, 128, 1>()};
  static const Variant v32rk4[] = {make_variant<RefMode<float>, true, 128, 1>()};
  *count = 1;
  if (dtype32) return rk4 ? v32rk4 : v32;
  return rk4 ? v64rk4 : v64;
}

cudaError_t ref_bisect(const EdgeArgs& a, cudaStream_t s) { return run_bisect<RefMode<double>, 128, 1>(a, s); }

// Eight warps per block: at the reference order's register count one block fills an SM's
// register file, so the critical photons of the mixed pipeline hold SMs of their own.
const Variant* ref_wide_variant() {
  static const Variant v = make_variant<RefMode<double>, false, 256, 1>();
  return &v;
}

// Warp-aggregated append of the flagged lanes' global indices to list (count in q->flagged).
__device__ __forceinline__ void append_flagged(bool flag, long long g, long long* list, Queue* q) {
  constexpr unsigned FULL = 0xffffffffu;
  const unsigned mask = __ballot_sync(FULL, flag);
  if (mask) {
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(&q->flagged, (unsigned long long)__popc(mask));
    base = __shfl_sync(FULL, base, leader);
    if (flag) list[base + __popc(mask & ((1u << lane) - 1u))] = g;
  }
}

__global__ void k_risk_prepass(const Image* __restrict__ images, int n_images, long long total,
                               const double* __restrict__ Y0, unsigned char* __restrict__ risk,
                               long long* __restrict__ list, Queue* q, long long* __restrict__ near_list,
                               Queue* q_near) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  bool critical = false, near = false;
  if (g < total) {
    const int img = find_image(images, n_images, g);
    const Params& P = images[img].P;
    double y0[8];
    photon_source(images, img, Y0, g, y0, q);
    const int cls = radial_risk(P.mass, P.a, P.r_capture, y0, risk_band(P.mass, P.rtol),
                                near_list ? near_band(P.mass) : 0.0);
    risk[g] = (unsigned char)cls;
    critical = cls == RISK_CRITICAL;
    near = cls == RISK_NEAR;
  }
  append_flagged(critical, g, list, q);
  if (near_list) append_flagged(near, g, near_list, q_near);
}

__global__ void k_check_risk(const Image* __restrict__ images, int n_images, long long total,
                             const unsigned char* __restrict__ risk, const long long* __restrict__ state,
                             long long* __restrict__ list, Queue* q, int recheck) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  bool flag = false;
  if (g < total) {
    const int cls = risk[g];
    const long long st = state[g];
    if (cls == RISK_ESCAPE || cls == RISK_NEAR) flag = st != ESCAPED;
    else if (cls == RISK_CAPTURE) flag = st != CAPTURED;
    else if (cls == RISK_RECHECK) flag = recheck != 0;
  }
  append_flagged(flag, g, list, q);
}

cudaError_t risk_prepass(const Image* images, int n_images, long long total, const double* Y0, unsigned char* risk,
                         long long* list, Queue* q, long long* near_list, Queue* q_near, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  const int block = 256;  // a multiple of 32: the append is warp-aggregated
  k_risk_prepass<<<(unsigned)((total + block - 1) / block), block, 0, s>>>(images, n_images, total, Y0, risk, list, q,
                                                                          near_list, q_near);
  return cudaGetLastError();
}

cudaError_t check_risk(const Image* images, int n_images, long long total, const unsigned char* risk,
                       const long long* state, long long* list, Queue* q, bool recheck, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  const int block = 256;
  k_check_risk<<<(unsigned)((total + block - 1) / block), block, 0, s>>>(images, n_images, total, risk, state, list, q,
                                                                        recheck ? 1 : 0);
  return cudaGetLastError();
}

__global__ void k_flag_boundary(const Image* __restrict__ images, int n_images, long long total,
                                const long long* __restrict__ state, long long* __restrict__ list, Queue* q) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  bool flag = false;
  if (g < total) {
    const Image& im = images[find_image(images, n_images, g)];
    const long long n = im.res;
    const long long p = g - im.offset + im.first;  // pixel of the image's grid
    const long long i = p / n, j = p - (p / n) * n;
    const long long s = state[g];
    flag = !(s == ESCAPED || s == CAPTURED);
    for (int di = -1; di <= 1 && !flag; ++di) {
      for (int dj = -1; dj <= 1 && !flag; ++dj) {
        const long long ii = i + di, jj = j + dj;
        if ((di == 0 && dj == 0) || ii < 0 || ii >= n || jj < 0 || jj >= n) continue;
        const long long q = ii * n + jj - im.first;  // the neighbour's row of this launch, if traced in it
        if (q < 0 || q >= im.count) continue;
        flag = state[im.offset + q] != s;
      }
    }
  }
  append_flagged(flag, g, list, q);
}

cudaError_t flag_boundary(const Image* images, int n_images, long long total, const long long* state, long long* list,
                          Queue* q, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  const int block = 256;  // a multiple of 32: the append is warp-aggregated
  k_flag_boundary<<<(unsigned)((total + block - 1) / block), block, 0, s>>>(images, n_images, total, state, list, q);
  return cudaGetLastError();
}

// Camera kernel: one image point per thread.
__global__ void k_camera_states(Frame F, double fov, long long res, const double* __restrict__ alpha,
                                const double* __restrict__ beta, long long n, double* __restrict__ Y0, int* err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a, b;
  if (alpha) {
    a = alpha[i];
    b = beta[i];
  } else {
    pixel_alpha_beta(fov, res, i, a, b);
  }
  double y0[8];
  if (camera_state(F, a, b, y0) != 0 && err) atomicCAS(err, 0, 6);
#pragma unroll
  for (int c = 0; c < 8; ++c) Y0[i * 8 + c] = y0[c];
}

cudaError_t camera_states(const Frame& F, double fov, long long res, const double* alpha, const double* beta,
                          long long n, double* Y0, int* err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int block = 256;
  k_camera_states<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(F, fov, res, alpha, beta, n, Y0, err);
  return cudaGetLastError();
}

}  // namespace krr
