// Kernels of the per-ray hot path, instantiated by krr_ref.cu (reference operation order,
// compiled with -fmad=false) and krr_fast.cu (FMA contraction; FP64 and FP32/FP64 mixed).
//
//   k_trace_plain       one photon per thread from an initial-state array or an image's camera
//                       (optionally through an index list: the FP64 re-trace of flagged
//                       pixels), until termination;
//   k_trace_persistent  a persistent grid over many images: each warp pulls photon indices
//                       from a device work queue, builds the photon from its image descriptor
//                       (camera at a finite observer distance) or from an initial-state array,
//                       and refills lanes as photons terminate.
#pragma once

#include "krr_device.cuh"
#include "krr_camera.cuh"
#include "krr_radial.cuh"

namespace krr {

// Which image a global photon index belongs to (images are contiguous ranges, offsets ascending).
__device__ __forceinline__ int find_image(const Image* __restrict__ im, int n_images, long long g) {
  int lo = 0, hi = n_images - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (im[mid].offset <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Scratch of a launch (device memory, zeroed before the launch).
struct Queue {
  unsigned long long head;        // next unclaimed global photon index
  unsigned long long retired;     // photons written back (every photon exactly once)
  unsigned long long attempts;    // step attempts, summed over rays
  unsigned long long accepted;    // accepted steps, summed over rays
  unsigned long long lane_iters;  // warp iterations x 32 (lane slots offered)
  unsigned long long busy_iters;  // lane slots that advanced a running photon
  int error;                      // KRR error code raised on the device, or 0
  int pad;
  unsigned long long flagged;     // photons appended to the re-trace list
  unsigned long long t_first;     // globaltimer (ns) of the first block's start (PDL_STAMP), from ~0
  unsigned long long t_last;      // globaltimer (ns) of the last block's end (PDL_STAMP)
  unsigned long long speculative; // edge bisection: photons traced ahead of their bracket
  unsigned long long discarded;   // edge bisection: attempts of speculative photons not needed
};

// Programmatic dependent launch (sm_90+) of the persistent kernel, as bits of its `pdl`
// argument: PDL_TRIGGER lets the next kernel of the stream launch (if it was launched as a
// programmatic dependent) as soon as every block of this one has started; PDL_WAIT makes this
// kernel, launched as such a dependent, wait at its exit for the kernel before it to complete
// (so later work of the stream sees both); PDL_STAMP records the kernel's start and end times.
enum : int { PDL_TRIGGER = 1, PDL_WAIT = 2, PDL_STAMP = 4 };

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Initial state of global photon g: a row of Y0, or the camera pixel of its image (pixel
// first + (g - offset) of the image's grid).
__device__ __forceinline__ void photon_source(const Image* __restrict__ images, int img,
                                              const double* __restrict__ Y0, long long g, double y0[8],
                                              Queue* q) {
  if (Y0) {
#pragma unroll
    for (int c = 0; c < 8; ++c) y0[c] = Y0[g * 8 + c];
  } else {
    const Image& im = images[img];
    if (camera_pixel_state(im, g - im.offset + im.first, y0) != 0 && q) atomicCAS(&q->error, 0, 6);
  }
}

// A photon's initial state and Carter constant, out of line: the camera's reference-order
// divisions and square roots run once per photon and stay out of the step loop's code (the
// mixed kernel: +0.7 %; the fast64 kernel keeps them inline, where the call's frame spills).
static __device__ __noinline__ double photon_start(const Image* __restrict__ images, int img, const double* __restrict__ Y0,
                                            long long g, double y0[8], Queue* q) {
  photon_source(images, img, Y0, g, y0, q);
  return carter_initial(images[img].P, y0);
}

// One photon per thread.  Without images every ray uses P and a row of Y0; with images the
// photon's image supplies the parameters and (when Y0 is null) the camera pixel.  index
// (nullable) maps thread i to global photon index[i].
template <class M, bool RK4>
__global__ void k_trace_plain(Params P, const Image* __restrict__ images, int n_images,
                              const double* __restrict__ Y0, const long long* __restrict__ index, long long n,
                              Outputs o, Queue* q) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned long long n_att = 0, n_acc = 0, n_ret = 0;
  if (i < n) {
    const long long g = index ? index[i] : i;
    double y0[8];
    Ray<M> ry;
    double* ev = o.event_Y ? o.event_Y + g * 8 : nullptr;
    unsigned char* hit = o.event_hit ? o.event_hit + g : nullptr;
    if (images) {
      const int img = find_image(images, n_images, g);
      photon_source(images, img, Y0, g, y0, q);
      const Params& Pi = images[img].P;
      ray_init<M>(Pi, y0, carter_initial(Pi, y0), ry);
      while (ry.state == RUNNING) attempt<M, RK4>(Pi, ry, ev, hit);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) y0[c] = Y0[g * 8 + c];
      ray_init<M>(P, y0, carter_initial(P, y0), ry);
      while (ry.state == RUNNING) attempt<M, RK4>(P, ry, ev, hit);
    }
    ray_store<M>(ry, o, g);
    n_att = (unsigned long long)ry.attempts;
    n_acc = (unsigned long long)ry.n_steps;
    n_ret = 1;
  }
  if (q) {  // warp-aggregated counters (blockDim is a multiple of 32)
    constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      n_att += __shfl_down_sync(FULL, n_att, off);
      n_acc += __shfl_down_sync(FULL, n_acc, off);
      n_ret += __shfl_down_sync(FULL, n_ret, off);
    }
    if ((threadIdx.x & 31u) == 0 && n_ret) {
      atomicAdd(&q->retired, n_ret);
      atomicAdd(&q->attempts, n_att);
      atomicAdd(&q->accepted, n_acc);
    }
  }
}

// MAXT threads per block and MINB resident blocks per SM are the launch bounds: the register
// cap (65536 / (MAXT * MINB)) that trades per-thread registers against resident warps.
// Queue entries are global photon indices, or positions in `index` (a re-trace list) when it
// is given; the number of entries is `total`, or *d_total when that is given (a count written
// on the device by the kernel before, so the launch can sit in a captured graph).
// risk (nullable, one byte per photon, from k_risk_prepass): RISK_CRITICAL photons are skipped
// (retired unwritten: another kernel traces them), and a photon that ends within 1 % of its
// affine or step budget is marked RISK_RECHECK (its class could depend on the last steps).
// flags: TRACE_SPREAD -- a warp holds at most ceil(entries / warps) photons at a time, so a
// short queue is shared by every warp of the grid instead of filling the first warps' lanes;
// TRACE_RESUME -- a photon continues from the result row already in the outputs (its last
// accepted state, affine parameter, counters and drift maxima: a trace that an FP32 overflow
// ended early) with the first step size, instead of starting again at the camera.
// TRACE_SKIP_NEAR -- RISK_NEAR photons are skipped as well (the near-edge kernel traces them).
enum : int { TRACE_SPREAD = 1, TRACE_RESUME = 2, TRACE_SKIP_NEAR = 4 };

template <class M>
__device__ __forceinline__ void resume_from_outputs(const Params& P, const Outputs& o, long long g, Ray<M>& ry) {
  using S = typename M::S;
  using D = typename M::D;
  if (!(o.lam && o.n_steps && o.n_rej)) return;  // nothing to resume from: start again
  const double* Y = o.Y + g * 8;
  ry.y[CT] = (S)Y[0];
  ry.y[CR] = (S)Y[1];
  ry.y[CTH] = (S)Y[2];
  ry.y[CPH] = (S)Y[3];
  ry.y[CPR] = (S)Y[5];
  ry.y[CPTH] = (S)Y[6];
  M::init_rhs(P, ry.y, ry.pt, ry.pph, ry.sh, ry.f, ry.tr);
  ry.lam = o.lam[g];
  ry.n_steps = (int)o.n_steps[g];
  ry.n_rej = (int)o.n_rej[g];
  if (o.max_null) ry.m_null = py_max(ry.m_null, (D)o.max_null[g]);
  if (o.max_q) ry.m_q = (D)o.max_q[g];
  ry.state = classify<M>(P, ry, false);
}

template <class M, bool RK4, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    k_trace_persistent(const Image* __restrict__ images, int n_images, long long total,
                       const double* __restrict__ Y0, Outputs o, Queue* __restrict__ q, int refill_threshold,
                       const long long* __restrict__ index, const unsigned long long* __restrict__ d_total,
                       unsigned char* __restrict__ risk, int flags, int pdl) {
  constexpr unsigned FULL = 0xffffffffu;
  if (pdl & PDL_TRIGGER) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if ((pdl & PDL_STAMP) && threadIdx.x == 0) atomicMin(&q->t_first, global_ns());
  if (d_total) total = (long long)*d_total;
  int cap = 32;
  if (flags & TRACE_SPREAD) {
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    cap = (int)min(32LL, max(1LL, (total + warps - 1) / warps));
  }
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  Ray<M> ry;
  ry.state = FAILURE;
  bool active = false;
  bool drained = false;
  long long g = -1;
  int img = 0;
  // Lane statistics, added when a photon retires (every busy lane slot is one step attempt).
  // 32-bit lane totals, flushed to the queue's 64-bit counters before they could wrap.
  unsigned my_attempts = 0, my_accepted = 0, my_iters = 0;
  auto retire = [&]() {
    ray_store<M>(ry, o, g);
    if (risk && (ry.lam > 0.99 * images[img].P.lambda_max || ry.n_steps > 0.99 * (double)images[img].P.max_steps))
      risk[g] = RISK_RECHECK;
    const unsigned long long ra = (unsigned long long)ry.attempts;
    if (ra >= (1ull << 30) || my_attempts >= (1u << 30)) {
      atomicAdd(&q->attempts, ra + my_attempts);
      atomicAdd(&q->busy_iters, ra + my_attempts);
      atomicAdd(&q->accepted, (unsigned long long)ry.n_steps + my_accepted);
      my_attempts = my_accepted = 0;
    } else {
      my_attempts += (unsigned)ra;
      my_accepted += (unsigned)ry.n_steps;
    }
    atomicAdd(&q->retired, 1ull);
  };
  while (true) {
    const unsigned idle = __ballot_sync(FULL, !active);
    const int n_idle = __popc(idle);
    const int want = min(n_idle, cap - (32 - n_idle));
    if (!drained && want > 0 && (n_idle >= refill_threshold || n_idle == 32)) {
      unsigned long long base = 0;
      const int leader = __ffs(idle) - 1;
      if ((int)lane == leader) base = atomicAdd(&q->head, (unsigned long long)want);
      base = __shfl_sync(FULL, base, leader);
      if (base + (unsigned long long)want >= (unsigned long long)total) drained = true;
      const int rank = __popc(idle & lt_mask);
      if (!active && rank < want) {
        const unsigned long long mine = base + (unsigned long long)rank;
        if (mine < (unsigned long long)total) {
          g = index ? index[mine] : (long long)mine;
          if (risk && (risk[g] == RISK_CRITICAL || ((flags & TRACE_SKIP_NEAR) && risk[g] == RISK_NEAR))) {
            atomicAdd(&q->retired, 1ull);  // traced by the reference-order or the near-edge kernel
          } else {
            img = find_image(images, n_images, g);
            const Image& im = images[img];
            double y0[8];
            double q0;
            if constexpr (M::kMixed) {
              q0 = photon_start(images, img, Y0, g, y0, q);
            } else {
              photon_source(images, img, Y0, g, y0, q);
              q0 = carter_initial(im.P, y0);
            }
            ray_init<M>(im.P, y0, q0, ry);
            if (flags & TRACE_RESUME) resume_from_outputs<M>(im.P, o, g, ry);
            if (ry.state == RUNNING) active = true;
            else retire();
          }
        }
      }
    }
    const unsigned busy = __ballot_sync(FULL, active);
    if (busy == 0) {
      if (drained) break;
      continue;
    }
    my_iters += 1;
    if (active) {
      const Image& im = images[img];
      double* ev = o.event_Y ? o.event_Y + g * 8 : nullptr;
      unsigned char* hit = o.event_hit ? o.event_hit + g : nullptr;
      attempt<M, RK4>(im.P, ry, ev, hit);
      if (ry.state != RUNNING) {
        retire();
        active = false;
      }
    }
  }
  // Per-warp statistics (one atomic per counter per warp).
  unsigned long long w_att = my_attempts, w_acc = my_accepted;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    w_att += __shfl_down_sync(FULL, w_att, off);
    w_acc += __shfl_down_sync(FULL, w_acc, off);
  }
  if (lane == 0) {
    atomicAdd(&q->attempts, w_att);
    atomicAdd(&q->accepted, w_acc);
    atomicAdd(&q->busy_iters, w_att);
    atomicAdd(&q->lane_iters, (unsigned long long)my_iters * 32ull);
  }
  if (pdl & PDL_STAMP) {
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&q->t_last, global_ns());
  }
  if (pdl & PDL_WAIT) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ------------------------------------------------------------------------------------------
// Edge bisection (scripts/study_edge_bisection.py:53-68): for each (case, polar angle phi) the
// image radius rho is bisected between a bracket [lo, hi] (captured at lo, escaped at hi): a
// photon at alpha = c_a + mid cos(phi), beta = c_b + mid sin(phi), mid = (lo + hi) / 2, is
// traced; ESCAPED moves hi to mid, anything else moves lo to mid; a result that is neither
// ESCAPED nor CAPTURED counts as a failure.
//
// One lane owns an item and runs its halvings one after another.  Once the queue is drained,
// a warp's idle lanes trace ahead: a helper takes a node of the bisection tree below an
// owner's current bracket, at depth 1..KRR_EDGE_DEPTH (the brackets the item holds after the
// owner's photon and the next ones, for either outcome), and traces its midpoint while the
// owner's photon is still running.  When the owner's photon ends, the helpers on the outcome's
// side move up one level; the one at depth 1 inherits the item and continues with its photon
// (possibly already ended, which settles one more halving at once); the helpers on the other
// side are discarded.  Every midpoint is 0.5 * (lo + hi) of the bracket the sequential
// bisection would hold there, so the results are the sequential ones bit for bit.  Lanes are
// given to the shallowest untraced nodes first, across the warp's owners with the most work
// left, then across the others.  A warp's lanes share its instructions, so a helper costs
// issue slots only where its warp would otherwise have ended; the host interleaves the items
// of all cases so that every warp holds cheap items, which end early and lend their lanes,
// beside expensive ones.
// ------------------------------------------------------------------------------------------
struct EdgeCase {
  Params P;
  Frame F;
  double c_alpha, c_beta;  // bracket centre in the image plane
};

struct EdgeArgs {
  const EdgeCase* cases;
  const int* item_case;
  const double* cos_phi;
  const double* sin_phi;
  double* lo;
  double* hi;
  long long* failures;
  const long long* order;  // queue position -> item (nullable: identity)
  int n_cases;
  long long n_items;
  int iterations;
  Queue* q;
  int refill_threshold;
  int grid, block;
};

template <class M>
struct EdgeLane {
  Ray<M> ry;
  double lo, hi, mid, cphi, sphi;
  long long fails;
  int it, c;
};

template <class M>
__device__ __forceinline__ void edge_start(const EdgeArgs& a, EdgeLane<M>& L) {
  const EdgeCase& ec = a.cases[L.c];
  L.mid = 0.5 * (L.lo + L.hi);
  const double al = ec.c_alpha + L.mid * L.cphi;
  const double be = ec.c_beta + L.mid * L.sphi;
  double y0[8];
  if (camera_state(ec.F, al, be, y0) != 0) atomicCAS(&a.q->error, 0, 6);
  ray_init<M>(ec.P, y0, carter_initial(ec.P, y0), L.ry);
}

enum : int { EDGE_IDLE = 0, EDGE_OWNER = 1, EDGE_HELPER = 2 };

#ifndef KRR_EDGE_DEPTH
#define KRR_EDGE_DEPTH 4
#endif
// Nodes below an owner's bracket, depth d = 1..KRR_EDGE_DEPTH, path p (d bits, the first step
// in the highest bit; 1 = the photon before escaped): bit (2^d - 2 + p) of a 32-bit mask.
constexpr int EDGE_DEPTH = KRR_EDGE_DEPTH;
static_assert(EDGE_DEPTH >= 1 && EDGE_DEPTH <= 4, "the node masks hold depths 1..4");
__device__ __forceinline__ int edge_node(int d, int p) { return (1 << d) - 2 + p; }

__device__ __forceinline__ int nth_set_bit(unsigned mask, int n) {
  for (int i = 0; i < n; ++i) mask &= mask - 1u;
  return __ffs(mask) - 1;
}

// The cases' step parameters are staged in shared memory when they fit: a warp's lanes hold
// items of different cases, and each parameter load is then one shared-memory access (the
// 184-byte stride, 23 doubles, is odd: no bank conflicts) instead of one global-memory
// wavefront per distinct case.
constexpr size_t kEdgeSmemMax = 46 * 1024;  // within the 48 KB a block gets without opt-in, beside its static slots
__host__ __device__ constexpr bool edge_params_in_smem(int n_cases) {
  return (size_t)n_cases * sizeof(Params) <= kEdgeSmemMax;
}

template <class M, int MAXT, int MINB, bool SMEM>
__global__ void __launch_bounds__(MAXT, MINB) k_bisect_edges(EdgeArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char edge_smem[];
  Params* s_params = reinterpret_cast<Params*>(edge_smem);
  if constexpr (SMEM) {
    static_assert(sizeof(Params) % 8 == 0, "Params is copied in 8-byte words");
    constexpr int words = (int)(sizeof(Params) / 8);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(s_params);
    for (int k = threadIdx.x; k < a.n_cases * words; k += blockDim.x)
      dst[k] = reinterpret_cast<const unsigned long long*>(&a.cases[k / words].P)[k % words];
    __syncthreads();
  }
  auto params = [&](int c) -> const Params& {
    if constexpr (SMEM) return s_params[c];
    else return a.cases[c].P;
  };
  __shared__ int slots[MAXT];  // 32 per warp, indexed by lane
  int* slot = slots + (threadIdx.x & ~31u);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  EdgeLane<M> L;
  L.ry.state = FAILURE;
  L.lo = L.hi = L.mid = L.cphi = L.sphi = 0.0;
  L.fails = 0;
  L.it = L.c = 0;
  int role = EDGE_IDLE, host = 0, depth = 0, path = 0;
  bool drained = false, dirty = true;
  long long g = -1;
  unsigned long long my_attempts = 0, my_accepted = 0, my_spec = 0, my_discarded = 0;
  unsigned my_iters = 0;
  auto finish_item = [&]() {
    a.lo[g] = L.lo;
    a.hi[g] = L.hi;
    if (a.failures) a.failures[g] = L.fails;
    atomicAdd(&a.q->retired, 1ull);
    role = EDGE_IDLE;
  };
  // Settle every owner whose photon has ended, repeatedly: an heir whose photon had ended too
  // settles the next halving in the following pass.
  auto resolve = [&]() {
    while (true) {
      const bool ended = role == EDGE_OWNER && L.ry.state != RUNNING;
      const unsigned em = __ballot_sync(FULL, ended);
      if (em == 0) break;
      dirty = true;
      int want = -1;  // the side the item continues on: 1 escaped, 0 otherwise; -1 item done
      if (ended) {
        my_accepted += (unsigned long long)L.ry.n_steps;
        const int st = L.ry.state;
        if (st != ESCAPED && st != CAPTURED) L.fails += 1;
        if (st == ESCAPED) L.hi = L.mid; else L.lo = L.mid;
        L.it += 1;
        if (L.it < a.iterations) want = (st == ESCAPED) ? 1 : 0;
        slot[lane] = -1;
      }
      __syncwarp();
      const int hl = (role == EDGE_HELPER) ? host : (int)lane;
      const int host_want = __shfl_sync(FULL, want, hl);
      const bool host_ended = role == EDGE_HELPER && ((em >> hl) & 1u);
      const bool on_side = host_ended && host_want >= 0 && ((path >> (depth - 1)) & 1) == host_want;
      const bool heir = on_side && depth == 1;
      if (heir) slot[host] = (int)lane;
      __syncwarp();
      const int my_heir = ended ? slot[lane] : -1;
      const int new_host = host_ended ? slot[host] : -1;
      const int src = heir ? host : (int)lane;
      const double lo_s = __shfl_sync(FULL, L.lo, src);
      const double hi_s = __shfl_sync(FULL, L.hi, src);
      const long long fails_s = __shfl_sync(FULL, L.fails, src);
      const long long g_s = __shfl_sync(FULL, g, src);
      const int it_s = __shfl_sync(FULL, L.it, src);
      if (heir) {  // the item's bracket is this lane's: its midpoint is this photon's
        L.lo = lo_s;
        L.hi = hi_s;
        L.fails = fails_s;
        L.it = it_s;
        g = g_s;
        role = EDGE_OWNER;
      } else if (on_side) {  // one level up, below the heir (or the same owner)
        depth -= 1;
        path &= (1 << depth) - 1;
        if (new_host >= 0) host = new_host;
      } else if (host_ended) {  // the other side: the photon is not needed
        my_discarded += (unsigned long long)L.ry.attempts;
        role = EDGE_IDLE;
      }
      if (ended) {
        if (want < 0) finish_item();
        else if (my_heir >= 0) role = EDGE_IDLE;
        else edge_start<M>(a, L);  // the next halving here (ends at once: next pass)
      }
      __syncwarp();
    }
  };
  while (true) {
    resolve();
    // New items from the queue for idle lanes.
    const unsigned idle = __ballot_sync(FULL, role == EDGE_IDLE);
    const int n_idle = __popc(idle);
    if (!drained && n_idle > 0 && (n_idle >= a.refill_threshold || n_idle == 32)) {
      dirty = true;
      unsigned long long base = 0;
      const int leader = __ffs(idle) - 1;
      if ((int)lane == leader) base = atomicAdd(&a.q->head, (unsigned long long)n_idle);
      base = __shfl_sync(FULL, base, leader);
      if (base + (unsigned long long)n_idle >= (unsigned long long)a.n_items) drained = true;
      if (role == EDGE_IDLE) {
        const unsigned long long mine = base + (unsigned long long)__popc(idle & lt_mask);
        if (mine < (unsigned long long)a.n_items) {
          g = a.order ? a.order[mine] : (long long)mine;
          L.c = a.item_case[g];
          L.lo = a.lo[g];
          L.hi = a.hi[g];
          L.cphi = a.cos_phi[g];
          L.sphi = a.sin_phi[g];
          L.fails = 0;
          L.it = 0;
          role = EDGE_OWNER;
          if (a.iterations > 0) edge_start<M>(a, L);
          else finish_item();
        }
      }
      resolve();
    }
    // Once the queue is drained: idle lanes take the untraced nodes below the owners'
    // brackets, shallowest first, then in lane order of the owners.
    if (drained && dirty) {
      dirty = false;
      const unsigned idle2 = __ballot_sync(FULL, role == EDGE_IDLE);
      if (idle2) {
        slot[lane] = 0;
        __syncwarp();
        if (role == EDGE_HELPER) atomicOr(&slot[host], 1 << edge_node(depth, path));
        __syncwarp();
        const unsigned cover = (unsigned)slot[lane];
        const int rank = (role == EDGE_IDLE) ? __popc(idle2 & lt_mask) : -1;
        // The owners with the most work left (halvings left x rtol^-1/5, the DP5 step count's
        // growth) come first: those at least half the warp's largest, then the others (5 % of
        // the edge study's time, 17 % fewer attempts discarded).
        float work = 0.0f;
        if (role == EDGE_OWNER)
          work = (float)(a.iterations - L.it) * exp2f(-0.2f * __log2f((float)params(L.c).rtol));
        float wmax = work;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) wmax = fmaxf(wmax, __shfl_xor_sync(FULL, wmax, off));
        const bool heavy = work >= 0.5f * wmax;
        int h = -1, hd = 0, hp = 0, base_rank = 0;
#pragma unroll
        for (int pd = 0; pd < 2 * EDGE_DEPTH; ++pd) {
          const int d = pd % EDGE_DEPTH + 1;
          const bool this_pass = (pd < EDGE_DEPTH) == heavy;
          const int width = 1 << d;
          unsigned seg = 0;
          if (role == EDGE_OWNER && this_pass && L.it + d < a.iterations)
            seg = (~cover >> (width - 2)) & (width == 32 ? FULL : ((1u << width) - 1u));
          const int cnt = __popc(seg);
          int incl = cnt;
#pragma unroll
          for (int off = 1; off < 32; off <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, off);
            if ((int)lane >= off) incl += t;
          }
          const int total = __shfl_sync(FULL, incl, 31);
          const bool mine = h < 0 && rank >= base_rank && rank < base_rank + total;
          const int key = mine ? rank - base_rank : -1;
          int j = 0;  // the owner lane: the first with incl > key
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1) {
            const int v = __shfl_sync(FULL, incl, j + step - 1);
            if (v <= key) j += step;
          }
          const int excl_j = __shfl_sync(FULL, incl - cnt, j);
          const unsigned seg_j = __shfl_sync(FULL, seg, j);
          if (mine) {
            h = j;
            hd = d;
            hp = nth_set_bit(seg_j, key - excl_j);
          }
          base_rank += total;
        }
        const int src = (h >= 0) ? h : (int)lane;
        double lo_s = __shfl_sync(FULL, L.lo, src);
        double hi_s = __shfl_sync(FULL, L.hi, src);
        const double cphi_s = __shfl_sync(FULL, L.cphi, src);
        const double sphi_s = __shfl_sync(FULL, L.sphi, src);
        const int c_s = __shfl_sync(FULL, L.c, src);
        const int it_s = __shfl_sync(FULL, L.it, src);
        if (h >= 0) {
          // the brackets along the path from the owner's: escaped halves to [lo, mid]
          for (int k = hd - 1; k >= 0; --k) {
            const double mid = 0.5 * (lo_s + hi_s);
            if ((hp >> k) & 1) hi_s = mid; else lo_s = mid;
          }
          L.lo = lo_s;
          L.hi = hi_s;
          L.cphi = cphi_s;
          L.sphi = sphi_s;
          L.c = c_s;
          L.it = it_s + hd;
          host = h;
          depth = hd;
          path = hp;
          role = EDGE_HELPER;
          my_spec += 1;
          edge_start<M>(a, L);
        }
        __syncwarp();
      }
    }
    const unsigned busy = __ballot_sync(FULL, role != EDGE_IDLE && L.ry.state == RUNNING);
    if (busy == 0) {
      if (drained) break;
      continue;
    }
    my_iters += 1;
    if (role != EDGE_IDLE && L.ry.state == RUNNING) {
      attempt<M, false>(params(L.c), L.ry, nullptr, nullptr);
      my_attempts += 1;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    my_attempts += __shfl_down_sync(FULL, my_attempts, off);
    my_accepted += __shfl_down_sync(FULL, my_accepted, off);
    my_spec += __shfl_down_sync(FULL, my_spec, off);
    my_discarded += __shfl_down_sync(FULL, my_discarded, off);
  }
  if (lane == 0) {
    atomicAdd(&a.q->attempts, my_attempts);
    atomicAdd(&a.q->accepted, my_accepted);
    atomicAdd(&a.q->busy_iters, my_attempts);
    atomicAdd(&a.q->lane_iters, (unsigned long long)my_iters * 32ull);
    atomicAdd(&a.q->speculative, my_spec);
    atomicAdd(&a.q->discarded, my_discarded);
  }
}

template <class M, int MAXT, int MINB, bool SMEM>
cudaError_t run_bisect_as(EdgeArgs a, cudaStream_t s) {
  const size_t smem = SMEM ? (size_t)a.n_cases * sizeof(Params) : 0;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bisect_edges<M, MAXT, MINB, SMEM>, MAXT, smem) !=
          cudaSuccess ||
      nb < 1)
    return cudaErrorLaunchOutOfResources;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Blocks per SM: the most, up to what fits, whose lanes number at most 3/4 of the items, so
  // that lanes which finish take further items from the queue; a study smaller than that keeps
  // every resident block, its idle lanes tracing midpoints ahead.  (The 51,840-item edge study
  // ran 131 ms at 2 blocks per SM, 147 ms at 3 and 181 ms at 1; every bracket the same.)
  int bps = nb;
  for (int b = nb; b >= 1; --b) {
    if (4LL * sms * b * MAXT <= 3LL * a.n_items) {
      bps = b;
      break;
    }
  }
  a.block = MAXT;
  a.grid = sms * bps;
  k_bisect_edges<M, MAXT, MINB, SMEM><<<a.grid, MAXT, smem, s>>>(a);
  return cudaGetLastError();
}

template <class M, int MAXT, int MINB>
cudaError_t run_bisect(EdgeArgs a, cudaStream_t s) {
  if (a.n_items <= 0) return cudaSuccess;
  return edge_params_in_smem(a.n_cases) ? run_bisect_as<M, MAXT, MINB, true>(a, s)
                                        : run_bisect_as<M, MAXT, MINB, false>(a, s);
}

// Flag the pixels whose classification the FP64 re-trace must settle: every photon that did not
// end ESCAPED or CAPTURED, and every pixel with a different code from one of its 8 neighbours
// in the same image (the shadow edge).  Flagged global indices are appended to `list` (at most
// `total` entries; each photon once) and counted in q->flagged.
__global__ void k_flag_boundary(const Image* __restrict__ images, int n_images, long long total,
                                const long long* __restrict__ state, long long* __restrict__ list, Queue* q);

// ------------------------------------------------------------------------------------------
// Launch helpers shared by the two translation units.
// ------------------------------------------------------------------------------------------
struct PlainArgs {
  Params P;
  const Image* images;
  int n_images;
  const double* Y0;
  const long long* index;
  long long n;
  Outputs o;
  Queue* q;
};

struct PersistArgs {
  const Image* images;
  int n_images;
  long long total;
  const double* Y0;
  Outputs o;
  Queue* q;
  int refill_threshold;
  int grid;
  int block;
  const long long* index;             // re-trace list (nullable)
  const unsigned long long* d_total;  // device-side entry count (nullable)
  unsigned char* risk;                // analytic classes (nullable): skip the critical photons
  int flags;                          // TRACE_* bits
  int pdl;                            // PDL_* bits; with PDL_WAIT launched as a programmatic dependent
};

template <class M, bool RK4>
cudaError_t run_plain(const PlainArgs& a, int block, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const long long grid = (a.n + block - 1) / block;
  k_trace_plain<M, RK4><<<(unsigned)grid, block, 0, s>>>(a.P, a.images, a.n_images, a.Y0, a.index, a.n, a.o, a.q);
  return cudaGetLastError();
}

template <class M, bool RK4, int MAXT, int MINB>
cudaError_t run_persistent(const PersistArgs& a, cudaStream_t s) {
  if (a.total <= 0 && !a.d_total) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)a.grid);
  cfg.blockDim = dim3(MAXT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (a.pdl & PDL_WAIT) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_trace_persistent<M, RK4, MAXT, MINB>, a.images, a.n_images, (long long)a.total,
                            a.Y0, a.o, a.q, a.refill_threshold, a.index, a.d_total, a.risk, a.flags, a.pdl);
}

template <class M, bool RK4, int MAXT, int MINB>
int persistent_occupancy() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_persistent<M, RK4, MAXT, MINB>, MAXT, 0) !=
      cudaSuccess)
    return 0;
  return nb;
}

template <class M, bool RK4, int MAXT, int MINB>
int persistent_registers() {
  cudaFuncAttributes attr{};
  if (cudaFuncGetAttributes(&attr, k_trace_persistent<M, RK4, MAXT, MINB>) != cudaSuccess) return 0;
  return attr.numRegs;
}

// A compiled launch shape of the persistent kernel.
struct Variant {
  int block;     // threads per block
  int min_blocks;  // launch-bounds minimum resident blocks per SM (1 = no register cap)
  cudaError_t (*run)(const PersistArgs&, cudaStream_t);
  int (*occupancy)();
  int (*registers)();
};

template <class M, bool RK4, int MAXT, int MINB>
constexpr Variant make_variant() {
  return Variant{MAXT, MINB, &run_persistent<M, RK4, MAXT, MINB>, &persistent_occupancy<M, RK4, MAXT, MINB>,
                 &persistent_registers<M, RK4, MAXT, MINB>};
}

// Analytic classes of every photon (krr_radial.cuh) into risk[]; the critical photons'
// global indices are appended to `list` and counted in q->flagged, and with near_list the
// near-edge photons' to near_list, counted in q_near->flagged.
__global__ void k_risk_prepass(const Image* __restrict__ images, int n_images, long long total,
                               const double* __restrict__ Y0, unsigned char* __restrict__ risk,
                               long long* __restrict__ list, Queue* q, long long* __restrict__ near_list,
                               Queue* q_near);

// After the traces: every non-critical photon whose code is not its analytic class, and with
// `recheck` every photon marked RISK_RECHECK, is appended to `list` and counted in q->flagged.
__global__ void k_check_risk(const Image* __restrict__ images, int n_images, long long total,
                             const unsigned char* __restrict__ risk, const long long* __restrict__ state,
                             long long* __restrict__ list, Queue* q, int recheck);

template <class M, bool RK4>
int plain_occupancy(int block) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_plain<M, RK4>, block, 0) != cudaSuccess) return 0;
  return nb;
}

}  // namespace krr
