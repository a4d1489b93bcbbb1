// Fast kernels: FP64 (Fast64) and FP32 stages with FP64 accumulation (Mixed).  Their FMAs are
// written out in the source; the translation unit is compiled with -fmad=false so the compiler
// fuses nothing else and every launch variant (register cap) computes identical results.
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

// The mixed re-trace of the few rays an FP32 overflow ended early (MixedSat: an overflowing
// trial step is a rejection, as in FP64).
const Variant* mixed_sat_variant() {
  static const Variant v = make_variant<MixedSat, false, 128, 4>();
  return &v;
}

cudaError_t fast_bisect(bool mixed, const EdgeArgs& a, cudaStream_t s) {
  return mixed ? run_bisect<Mixed, 128, 1>(a, s) : run_bisect<Fast64, 128, 3>(a, s);
}

}  // namespace krr
