// Kernels with FMA contraction: FP64 (Fast64) and FP32 stages with FP64 accumulation (Mixed).
#include "krr_launch.h"

namespace krr {

cudaError_t fast_plain(bool mixed, bool rk4, const PlainArgs& a, int block, cudaStream_t s) {
  if (mixed) {
    if (rk4) return cudaErrorNotSupported;
    return run_plain<Mixed, false>(a, block, s);
  }
  return rk4 ? run_plain<Fast64, true>(a, block, s) : run_plain<Fast64, false>(a, block, s);
}

cudaError_t fast_persistent(bool mixed, bool rk4, const PersistArgs& a, cudaStream_t s) {
  if (mixed) {
    if (rk4) return cudaErrorNotSupported;
    return run_persistent<Mixed, false>(a, s);
  }
  return rk4 ? run_persistent<Fast64, true>(a, s) : run_persistent<Fast64, false>(a, s);
}

int fast_occupancy(bool mixed, bool rk4, bool persistent, int block) {
  if (persistent) {
    if (mixed) return rk4 ? 0 : persistent_occupancy<Mixed, false>(block);
    return rk4 ? persistent_occupancy<Fast64, true>(block) : persistent_occupancy<Fast64, false>(block);
  }
  if (mixed) return rk4 ? 0 : plain_occupancy<Mixed, false>(block);
  return rk4 ? plain_occupancy<Fast64, true>(block) : plain_occupancy<Fast64, false>(block);
}

}  // namespace krr
