"""Benchmark of KerrRay's per-ray hot path on B200.

Workload (one "step"): the batched FP64 sweep -- spins {0, 0.5, 0.9, 0.99} x inclinations
{17, 60, 85} deg x resolutions {128, 256, 512}^2 x rtol {1e-6, 1e-8, 1e-10} (atol = 1e-2 rtol),
observer at r_o = 1000 M, image plane +-8 M, reference defaults otherwise: 108 images,
12,386,304 photons in one persistent launch (camera, Dormand-Prince 5(4) integration and
classification on the device). Metric: rays/s, the whole job over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun the job is N copies of the sweep with the observer turned in azimuth (distinct
images of equal cost), split across the N ranks by predicted cost (kerrray_b200.shard): each
rank traces one sweep's worth on its own GPU (weak scaling; the photons are independent, there
is no data-path collective); the time is the max over ranks.
``--impl reference`` times the CPU restatement of the reference kernel (the oracle, OpenMP over
all host threads) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "rays/s per B200: plain FP64 vs persistent/FP32-mixed at identical mask; %peak"
WORKLOAD = ("batched FP64 sweep: a*{0,0.5,0.9,0.99} x i{17,60,85}deg x res{128,256,512}^2 x "
            "rtol{1e-6,1e-8,1e-10}, atol=1e-2 rtol, r_o=1000 M, +-8 M (108 images)")

# Floating-point operations of the reference algorithm, counted on the oracle with a counting
# scalar type (each add, mul, div, sqrt, sin/cos and pow is one operation; pinned by
# tests/test_oracle_golden.py): per step attempt, per accepted step, per ray.
FLOP_PER_ATTEMPT = 1210
FLOP_PER_ACCEPT = 28
FLOP_PER_RAY = 127


def ordinal(k: int) -> str:
    """1st, 2nd, 3rd, 4th, ..., 11th, 12th, 13th, 21st, ..."""
    k = int(k)
    suffix = "th" if 10 <= k % 100 <= 20 else {1: "st", 2: "nd", 3: "rd"}.get(k % 10, "th")
    return f"{k}{suffix}"

def algorithmic_flops(stats: dict) -> float:
    return FLOP_PER_ATTEMPT * stats["attempts"] + FLOP_PER_ACCEPT * stats["accepted"] + FLOP_PER_RAY * stats["photons"]


WORKLOADS = {
    "sweep": WORKLOAD,
    "sweep128": "the 36 128^2 images of the sweep (a*{0,0.5,0.9,0.99} x i{17,60,85} x rtol{1e-6,1e-8,1e-10})",
    "spin99_1024": "a*=0.99, i=85deg, r_o=1000 M, +-8 M, 1024^2, rtol 1e-6, atol 1e-8",
    "spin99_2048": "a*=0.99, i=85deg, r_o=1000 M, +-8 M, 2048^2, rtol 1e-6, atol 1e-8",
    "bisect": ("batched edge bisection: a*{0,0.5,0.9,0.99} x i{17,60,85}deg x 1440 polar angles x rtol{1e-6,1e-8,"
               "1e-10}, rho in [2, 8] M about the Bardeen centroid / k, 36 halvings, r_o = 1e5 M"),
    "lensing": ("lensing-map adjoint: a*=0.8, i=60deg, r_o=1000 M, 256^2 over +-12 M, escaped rays > 3 px from the "
                "shadow edge, rtol 1e-10, checkpoints every 32 accepted steps"),
}


def workload_specs(K, name: str):
    if name == "sweep":
        return sweep_specs(K)
    if name == "sweep128":
        return sweep_specs(K, resolutions=(128,))
    if name in ("spin99_1024", "spin99_2048"):
        cam = K.Camera(radius=1000.0, inclination_deg=85.0, fov=8.0, resolution=int(name[-4:]))
        integ = K.IntegratorOptions(method="rk45", rtol=1e-6, atol=1e-8)
        return [K.ImageSpec(K.Spacetime(1.0, 0.99), cam, integ, K.TerminationOptions())]
    raise ValueError(name)


def sweep_specs(K, resolutions=(128, 256, 512)):
    specs = []
    for spin in (0.0, 0.5, 0.9, 0.99):
        st = K.Spacetime(1.0, spin)
        for incl in (17.0, 60.0, 85.0):
            for res in resolutions:
                cam = K.Camera(radius=1000.0, inclination_deg=incl, fov=8.0, resolution=res)
                for rtol in (1e-6, 1e-8, 1e-10):
                    integ = K.IntegratorOptions(method="rk45", rtol=rtol, atol=1e-2 * rtol)
                    specs.append(K.ImageSpec(st, cam, integ, K.TerminationOptions()))
    order = K.order_by_cost(specs)
    return [specs[k] for k in order]


# ------------------------------------------------------------------------------------------
# Clocks during the timed region.
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="krr_clocks_", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clocks not sampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


# ------------------------------------------------------------------------------------------
# CPU baseline: the oracle (C++ restatement of the reference kernel) on a bounded sample.
# ------------------------------------------------------------------------------------------
def cpu_sample(specs, stride: int, offset: int = 0):
    """(spec index, pixel indices) pairs of a uniform stride sample over the global photon order."""
    out = []
    base = 0
    for k, s in enumerate(specs):
        n = s.n_rays
        first = (offset - base) % stride
        idx = np.arange(first, n, stride, dtype=np.int64)
        if idx.size:
            out.append((k, idx))
        base += n
    return out


def oracle_options(spec, scale: float = 1.0):
    """The oracle's options for an image spec, with the tolerances scaled by ``scale``."""
    from oracle import oracle as O

    i, t = spec.integ, spec.term
    return O.Options(rtol=i.rtol * scale, atol=i.atol * scale, step_size=i.step_size, max_steps=i.max_steps,
                     lambda_max=i.lambda_max, h_min=i.h_min, h_max=i.h_max, horizon_epsilon=t.horizon_epsilon,
                     escape_radius=t.escape_radius)


def oracle_pixels(spec, pixels: np.ndarray, scale: float = 1.0, threads: int | None = None) -> dict:
    """The oracle (the reference's kernel restated in C++, OpenMP over the host threads) on the
    given pixels of an image: camera states restated in NumPy, then the integration."""
    from oracle import oracle as O

    cam = spec.camera
    a, b = O.pixel_coordinates(cam.fov, cam.resolution)
    y0 = O.initial_states(spec.spacetime.mass, spec.spacetime.spin, cam.radius, cam.inclination_deg, cam.phi_deg,
                          a.ravel()[pixels], b.ravel()[pixels])
    out = O.integrate(spec.spacetime.mass, spec.spacetime.spin, y0, oracle_options(spec, scale),
                      threads=threads or os.cpu_count() or 1)
    out["Y0"] = y0
    return out


def time_cpu_sample(specs, stride: int, offset: int = 0, keep: bool = False):
    """Trace every ``stride``-th photon of the job (from ``offset``) with the oracle on all host
    threads: (rays, seconds, threads[, per-image (pixels, results) when ``keep``])."""
    threads = os.cpu_count() or 1
    n_rays = 0
    kept = []
    t0 = time.perf_counter()
    for k, idx in cpu_sample(specs, stride, offset):
        out = oracle_pixels(specs[k], idx, threads=threads)
        n_rays += idx.size
        if keep:
            kept.append((k, idx, out))
    dt = time.perf_counter() - t0
    return (n_rays, dt, threads, kept) if keep else (n_rays, dt, threads)


def calibrate_stride(specs, target_s: float) -> int:
    """Stride whose sample takes about target_s seconds (probe samples grow until >= 1 s)."""
    total = sum(s.n_rays for s in specs)
    stride = max(total // 3000, 1)
    while True:
        n, dt, _ = time_cpu_sample(specs, stride, 0)
        if dt >= 1.0 or stride == 1:
            break
        stride = max(stride // 4, 1)
    want = max(int(n / max(dt, 1e-6) * target_s), 1)
    return max(total // want, 1)


def cpu_baseline(specs, target_s: float = 15.0, keep: bool = False):
    """The oracle's rays/s on a bounded uniform sample of the job (about ``target_s`` seconds);
    with ``keep``, also the sample's per-image (pixels, oracle results)."""
    from oracle.build import build

    build()
    stride = calibrate_stride(specs, target_s)
    n, dt, threads, kept = time_cpu_sample(specs, stride, 1, keep=True)
    line = {"value": n / dt, "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": f"every {ordinal(stride)} photon of the {len(specs)}-image job ({n} rays, {dt:.1f} s), C++ oracle, "
                      f"OpenMP {threads} threads"}
    return (line, kept) if keep else line


# ------------------------------------------------------------------------------------------
# Parity against the oracle at bench size: termination codes, and terminal directions where
# the escaped rays cross the escape surface.
# ------------------------------------------------------------------------------------------
def surface_directions(K, spec, Y, state) -> np.ndarray:
    """(n, 2) theta, phi where each escaped ray of an image spec (or of a ``(spacetime, r_esc)``
    pair) crosses r = r_esc (device landing, ``krr_escape_directions``); NaN for the other rows.
    ``Y``/``state`` host arrays or device tensors."""
    import torch

    Yt = torch.as_tensor(np.asarray(Y, dtype=np.float64) if not torch.is_tensor(Y) else Y, device="cuda").contiguous()
    St = torch.as_tensor(np.asarray(state, dtype=np.int64) if not torch.is_tensor(state) else state,
                         device="cuda").contiguous()
    st, r_esc = spec if isinstance(spec, tuple) else (spec.spacetime, float(spec.term.escape_radius))
    th, ph = K.escape_directions(st, Yt, St, float(r_esc))
    return torch.stack([th, ph], dim=1).cpu().numpy()


def direction_error(d1: np.ndarray, d2: np.ndarray) -> np.ndarray:
    """The angle (rad) between the directions (theta, phi) of each row on the escape sphere
    (``kerrray_b200.direction_angle``)."""
    from kerrray_b200 import direction_angle

    return direction_angle(d1[:, 0], d1[:, 1], d2[:, 0], d2[:, 1])


def component_error(d1: np.ndarray, d2: np.ndarray) -> np.ndarray:
    """max(|d theta|, |d phi| wrapped into [-pi, pi)) per row (rad): the coordinates' own differences."""
    dth = np.abs(d1[:, 0] - d2[:, 0])
    dph = np.abs(np.remainder(d1[:, 1] - d2[:, 1] + math.pi, 2.0 * math.pi) - math.pi)
    return np.maximum(dth, dph)


# Tolerance scales of the oracle runs that bound its own error at a tolerance: 100x tighter,
# and 5 % either side.
ENVELOPE_SCALES = (0.01, 0.95, 1.05)


def against_oracle(K, spec, pixels: np.ndarray, gpu_state: np.ndarray, gpu_dirs: np.ndarray, oracle: dict,
                   threads: int | None = None) -> dict:
    """GPU results on ``pixels`` of an image against the oracle's on the same pixels.

    Codes must be identical. Terminal states of rays escaped in both are compared on the escape
    surface, by the angle between their directions (``direction_error``; the coordinates' own
    differences are reported beside it); the bar is 10 rtol, or 4x the oracle's own error
    envelope there in the same measure, computed for the
    rays beyond 10 rtol: the larger of its distance to the oracle at a 100x tighter tolerance
    and its spread over tolerances 5 % apart (rtol x 0.95 and x 1.05). Two valid integrations at
    one tolerance differ by their global errors: near the photon orbit these grow far beyond
    rtol, and a ray whose step sequence takes a few very large steps (the reference's
    controller has no step cap) has a global error that changes with any change of the sequence
    -- a tolerance 5 % away, or the FP32 rounding of the mixed stages. Returns the counts and the
    error distribution in units of rtol."""
    ref_state = np.asarray(oracle["state"], dtype=np.int64)
    differ = np.flatnonzero(ref_state != gpu_state)
    ref_dirs = surface_directions(K, spec, oracle["Y"], ref_state)
    both = np.flatnonzero((ref_state == 1) & (gpu_state == 1))
    err = direction_error(gpu_dirs[both], ref_dirs[both])
    comp = component_error(gpu_dirs[both], ref_dirs[both])
    rtol = float(spec.integ.rtol)
    out = {"rays": int(pixels.size), "codes_differ": int(differ.size), "escaped_compared": int(both.size)}
    if both.size:
        out["component_err_over_rtol"] = {"p99": float(np.quantile(comp, 0.99)) / rtol, "max": float(comp.max()) / rtol,
                                          "beyond_10rtol": int((comp > 10 * rtol).sum())}
        over = both[err > 10 * rtol]
        out.update({"err_over_rtol": {"median": float(np.median(err)) / rtol, "p99": float(np.quantile(err, 0.99)) / rtol,
                                      "max": float(err.max()) / rtol},
                    "beyond_10rtol": int(over.size), "beyond_bar": 0})
        if over.size:
            env = np.zeros(over.size)
            for scale in ENVELOPE_SCALES:
                other = oracle_pixels(spec, pixels[over], scale=scale, threads=threads)
                d = direction_error(ref_dirs[over], surface_directions(K, spec, other["Y"], other["state"]))
                env = np.where(np.isnan(d) | np.isnan(env), np.nan, np.maximum(env, d))
            # A ray that one of these integrations does not see escape lies within the
            # tolerance's own ambiguity of the shadow edge: its envelope is unbounded.
            out["envelope_unbounded"] = int((~np.isfinite(env)).sum())
            env = np.where(np.isfinite(env), env, np.inf)
            e_over = err[err > 10 * rtol]
            bad = e_over > 4.0 * env
            out["beyond_bar"] = int(bad.sum())
            finite = env[np.isfinite(env)]
            out["envelope_over_rtol_max"] = float(finite.max()) / rtol if finite.size else None
            if bad.any():
                out["worst_beyond_bar"] = [{"pixel": int(pixels[over][j]), "err_over_rtol": float(e_over[j] / rtol),
                                            "env_over_rtol": float(env[j] / rtol)}
                                           for j in np.argsort(-e_over * bad)[: min(5, int(bad.sum()))]]
    return out


# ------------------------------------------------------------------------------------------
def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import kerrray_b200 as K
    from oracle.build import build

    build()
    specs = sweep_specs(K)
    total = sum(s.n_rays for s in specs)
    stride = calibrate_stride(specs, 8.0)
    for w in range(args.warmup):
        time_cpu_sample(specs, stride * 4, w)
    rays, secs = 0, 0.0
    threads = os.cpu_count() or 1
    for k in range(args.steps):
        n, dt, threads = time_cpu_sample(specs, stride, k)
        rays += n
        secs += dt
    value = rays / secs
    # A step is one bounded sample of the sweep (every stride-th photon, a different offset per
    # step); ms_per_step is that sample's measured time. The whole sweep would take
    # total / value seconds on these cores, reported beside it as an extrapolation.
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "photons": total, "sample_stride": stride,
                   "photons_per_step": rays // max(args.steps, 1),
                   "step": f"every {ordinal(stride)} photon of the sweep (offset = step index), the same rays/s metric",
                   "full_sweep_s_extrapolated": total / value},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads, "kind": "port",
                         "sample": f"every {ordinal(stride)} photon per step ({rays // max(args.steps, 1)} rays/step), "
                                   f"C++ restatement of the reference kernel, OpenMP {threads} threads"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed_steps(sweep, steps: int, stream, flush) -> list[float]:
    """CUDA-event time (ms) of each graph launch; L2 flushed before each, outside the events."""
    import torch

    out = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sweep.run(stats=False)
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


PLAIN_BLOCKS = (32, 64, 128, 256)


def best_plain(K, specs, local: int, stream, flush, steps: int, precision: str = "reference"):
    """A one-thread-per-photon kernel (no work queue) at its fastest block size: each of
    PLAIN_BLOCKS timed once, the fastest again over ``steps`` launches. ``precision``
    "reference" is the plain FP64 kernel in the reference's operation order; "fast64" the same
    launch with the fast FP64 arithmetic. Returns (its DeviceSweep, best ms, block, ms per
    block). The results do not depend on the block size (the arithmetic is per photon)."""
    import torch

    by_block = {}
    for blk in PLAIN_BLOCKS:
        sw = K.DeviceSweep(specs, precision=precision, device=local, launch=K.LaunchConfig(plain=True, block=blk))
        sw.run(stats=False)
        by_block[blk] = min(_timed_steps(sw, 1, stream, flush))
        sw.close()
        del sw
        torch.cuda.empty_cache()
    blk = min(by_block, key=by_block.get)
    sw = K.DeviceSweep(specs, precision=precision, device=local, launch=K.LaunchConfig(plain=True, block=blk))
    sw.run(stats=False)
    best = min([by_block[blk]] + _timed_steps(sw, steps, stream, flush))
    return sw, best, blk, {str(b): round(t, 3) for b, t in by_block.items()}


def escape_surface_errors(K, specs, a, b) -> dict:
    """Terminal directions of two traces of the same images compared where each ray that
    escaped in both crosses the escape surface (their final states are the first accepted
    steps beyond it, which depend on the step sequence): |d theta| and |d phi| in rad."""
    import torch

    dth, dph = [], []
    for k, spec in enumerate(specs):
        lo, hi = int(a.offsets[k]), int(a.offsets[k + 1])
        r_esc = float(spec.term.escape_radius)
        ya, sa = a.tensors["Y"][lo:hi], a.tensors["state"][lo:hi]
        yb, sb = b.tensors["Y"][lo:hi], b.tensors["state"][lo:hi]
        tha, pha = K.escape_directions(spec.spacetime, ya, sa, r_esc)
        thb, phb = K.escape_directions(spec.spacetime, yb, sb, r_esc)
        both = (sa == 1) & (sb == 1)
        dth.append((tha - thb).abs()[both])
        dph.append(torch.remainder(pha - phb + math.pi, 2 * math.pi).sub(math.pi).abs()[both])
    out = {}
    for name, v in (("dtheta", torch.cat(dth)), ("dphi", torch.cat(dph))):
        v = v.double()
        out[name] = {"median": float(v.median()), "p99": float(torch.quantile(v[:10_000_000], 0.99)),
                     "max": float(v.max())}
    out["rays"] = int(sum(x.numel() for x in dth))
    return out


def edge_rms_px(K, spec, state: np.ndarray) -> float:
    """rms distance (px) of the captured-mask edge (the bilinear interpolant's 0.5 level set)
    from Bardeen's exact curve after the finite-distance correction."""
    return float(K.mask_edge_error(spec.spacetime, spec.camera, state == 2)["rms_px"])


def sweep_edge_errors(K, specs, state: np.ndarray, offsets) -> dict:
    """Per-image mask-edge rms against Bardeen (px), summarised per resolution."""
    rows = []
    for k, spec in enumerate(specs):
        rows.append((spec.camera.resolution, edge_rms_px(K, spec, state[int(offsets[k]):int(offsets[k + 1])])))
    out = {}
    for res in sorted({r for r, _ in rows}):
        v = [e for r, e in rows if r == res]
        out[f"{res}^2"] = {"images": len(v), "median_px": float(np.median(v)), "max_px": float(np.max(v))}
    return out


def mixed_vs_plain(K, local: int, stream, flush, name: str = "spin99_1024", oracle_check: bool = True) -> dict:
    """Mixed persistent + FP64 settling of the near-critical pixels against the plain FP64 kernel
    on the a*=0.99, i=85 deg image (rtol 1e-6): rays/s of each pipeline and of the fast64 kernels
    (persistent, and one thread per photon), whether the shadow masks are identical, and --
    against the oracle on every pixel -- the codes and the terminal states on the escape surface."""
    import torch

    specs = workload_specs(K, name)
    spec = specs[0]
    total = spec.n_rays
    tuned, _ = K.autotune(specs, precision="mixed", device=local)

    def mixed_with(retrace: int):
        return K.DeviceSweep(specs, precision="mixed", device=local,
                             launch=K.LaunchConfig(variant=tuned.variant, refill_threshold=tuned.refill_threshold,
                                                   retrace=retrace))

    crit, edge, bare = mixed_with(K.RETRACE_CRITICAL), mixed_with(K.RETRACE_EDGE), mixed_with(0)
    near = mixed_with(K.RETRACE_CRITICAL_NEAR)
    fast = K.DeviceSweep(specs, precision="fast64", device=local, launch=K.autotune(specs, precision="fast64", device=local)[0])
    sweeps = (crit, edge, bare, fast, near)
    for sw in sweeps:
        sw.run()
    t = {k: min(_timed_steps(sw, 3, stream, flush)) for k, sw in zip(("crit", "edge", "bare", "fast", "near"), sweeps)}
    plain, t["plain"], plain_block, plain_by_block = best_plain(K, specs, local, stream, flush, 2)
    fplain, t["fast_plain"], fplain_block, _ = best_plain(K, specs, local, stream, flush, 2, precision="fast64")
    cs, es, bs, ns = crit.stats(), edge.stats(), bare.stats(), near.stats()
    from kerrray_b200 import _lib

    mixed_tflops = algorithmic_flops(bs) / (t["bare"] * 1e-3) / 1e12
    peak32, peak64 = _lib.fma_peak_tflops(local, False), _lib.fma_peak_tflops(local, True)
    ref = plain.tensors["state"]
    esc = (ref == 1) & (crit.tensors["state"] == 1)
    # Terminal states compared where each escaped ray crosses the escape surface: the final
    # states themselves lie at the first accepted step beyond it, which depends on the step
    # sequence (up to ~100 M apart at r = 1000).
    dirs_m = surface_directions(K, spec, crit.tensors["Y"], crit.tensors["state"])
    dirs_p = surface_directions(K, spec, plain.tensors["Y"], plain.tensors["state"])
    esc_np = esc.cpu().numpy()
    d_mp = direction_error(dirs_m[esc_np], dirs_p[esc_np])
    st_plain = ref.cpu().numpy()
    st_mixed = crit.tensors["state"].cpu().numpy()
    st_fast = fast.tensors["state"].cpu().numpy()
    rtol = float(spec.integ.rtol)
    out = {"workload": WORKLOADS[name], "photons": total,
           "mixed_pipeline_rays_s": total / (t["crit"] * 1e-3), "plain_fp64_rays_s": total / (t["plain"] * 1e-3),
           "plain_fp64_block": plain_block, "plain_fp64_ms_by_block": plain_by_block,
           "fast64_plain_rays_s": total / (t["fast_plain"] * 1e-3), "fast64_plain_block": fplain_block,
           "speedup_mixed_vs_plain": t["plain"] / t["crit"],
           "speedup_mixed_vs_fast64_plain": t["fast_plain"] / t["crit"],
           "speedup_mixed_vs_fast64_persistent": t["fast"] / t["crit"],
           "speedup_fast64_persistent_vs_fast64_plain": t["fast_plain"] / t["fast"],
           "mask_identical": bool(torch.equal(crit.tensors["state"], ref)),
           "pixels_differing": int((crit.tensors["state"] != ref).sum().item()),
           "critical": int(cs["critical"]), "rechecked": int(cs["rechecked"]), "critical_ms": cs["critical_ms"],
           "pipeline": "analytic critical set in reference-order FP64 beside the mixed trace, then a re-trace of "
                       "every photon unlike its analytic class",
           "mixed_near_pipeline_rays_s": total / (t["near"] * 1e-3),
           "speedup_mixed_near_vs_plain": t["plain"] / t["near"],
           "mixed_near_mask_identical": bool(torch.equal(near.tensors["state"], ref)),
           "near_edge": int(ns["near_edge"]), "near_critical_ms": ns["critical_ms"],
           "near_pipeline": "the same with the escaping photons within 0.35 M of the critical curve in fast FP64 "
                            "on SMs of their own (exit directions at the oracle's bar)",
           "mixed_kernel_only_rays_s": total / (t["bare"] * 1e-3),
           "mixed_kernel_roofline": {"achieved": mixed_tflops, "unit": "TFLOP/s", "fp32_peak": peak32,
                                     "frac_fp32": mixed_tflops / peak32, "fp64_peak": peak64,
                                     "attempts": int(bs["attempts"]), "accepted": int(bs["accepted"]),
                                     "note": "the reference's algorithmic FLOPs per second of the mixed kernel "
                                             "(stages in FP32, accumulation and error norm in FP64) against the "
                                             "measured FP32 and FP64 FMA peaks"},
           "mixed_edge_retrace_rays_s": total / (t["edge"] * 1e-3),
           "edge_retrace_mask_identical": bool(torch.equal(edge.tensors["state"], ref)),
           "edge_retraced": int(es["retraced"]),
           "fast64_rays_s": total / (t["fast"] * 1e-3),
           "mixed_vs_plain_escape_surface_over_rtol": {"median": float(np.median(d_mp)) / rtol,
                                                      "p99": float(np.quantile(d_mp, 0.99)) / rtol,
                                                      "max": float(d_mp.max()) / rtol,
                                                      "beyond_10rtol": int((d_mp > 10 * rtol).sum())},
           "edge_rms_px_plain": edge_rms_px(K, spec, st_plain),
           "edge_rms_px_mixed": edge_rms_px(K, spec, st_mixed),
           "mixed_launch": {"variant": tuned.variant, "refill_threshold": tuned.refill_threshold}}
    if oracle_check:
        # Every pixel against the oracle (the reference's kernel restated, all host threads).
        pixels = np.arange(total, dtype=np.int64)
        t0 = time.perf_counter()
        ora = oracle_pixels(spec, pixels)
        out["oracle_s"] = time.perf_counter() - t0
        ora_state = np.asarray(ora["state"], dtype=np.int64)
        out["pixels_differing_vs_oracle"] = {"plain_fp64": int((st_plain != ora_state).sum()),
                                             "mixed_pipeline": int((st_mixed != ora_state).sum()),
                                             "fast64": int((st_fast != ora_state).sum())}
        out["mixed_vs_oracle"] = against_oracle(K, spec, pixels, st_mixed, dirs_m, ora)
        st_near = near.tensors["state"].cpu().numpy()
        out["pixels_differing_vs_oracle"]["mixed_near_pipeline"] = int((st_near != ora_state).sum())
        out["mixed_near_vs_oracle"] = against_oracle(K, spec, pixels, st_near,
                                                     surface_directions(K, spec, near.tensors["Y"], near.tensors["state"]),
                                                     ora)
        dirs_f = surface_directions(K, spec, fast.tensors["Y"], fast.tensors["state"])
        out["fast64_vs_oracle"] = against_oracle(K, spec, pixels, st_fast, dirs_f, ora)
        out["plain_vs_oracle"] = against_oracle(K, spec, pixels, st_plain, dirs_p, ora)
    for sw in sweeps + (plain, fplain):
        sw.close()
    return out


def sample_parity(K, specs, sweep, kept) -> dict:
    """The persistent sweep's rows for the CPU baseline's sample against the oracle's results on
    the same photons (codes; terminal states on the escape surface, bar as in against_oracle)."""
    import torch

    tot = {"rays": 0, "codes_differ": 0, "escaped_compared": 0, "beyond_10rtol": 0, "beyond_bar": 0,
           "envelope_unbounded": 0}
    worst = 0.0
    for k, idx, ora in kept:
        rows = torch.as_tensor(int(sweep.offsets[k]) + idx, device=sweep.tensors["state"].device)
        st = sweep.tensors["state"].index_select(0, rows)
        Y = sweep.tensors["Y"].index_select(0, rows)
        dirs = surface_directions(K, specs[k], Y, st)
        r = against_oracle(K, specs[k], idx, st.cpu().numpy(), dirs, ora)
        for key in tot:
            tot[key] += int(r.get(key, 0))
        if "err_over_rtol" in r:
            worst = max(worst, r["err_over_rtol"]["max"])
    tot["err_over_rtol_max"] = worst
    return tot


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import kerrray_b200 as K
    from kerrray_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    _lib.lib()

    from kerrray_b200 import shard

    # N copies of the workload (the observer turned in azimuth), cut into pixel pieces of equal
    # predicted cost and dealt to the ranks: every rank traces one workload's worth.
    specs_all = shard.replicate_specs(workload_specs(K, args.workload), world)
    pieces = shard.shard_pieces(specs_all, rank, world)
    specs = shard.piece_specs(specs_all, pieces)
    total = sum(s.n_rays for s in specs)              # this rank's photons
    job_total = sum(s.n_rays for s in specs_all)      # every rank's
    if args.launch:
        variant, refill = (int(x) for x in args.launch.split(":"))
        tuned = K.LaunchConfig(variant=variant, refill_threshold=refill)
        info = [v for v in K.list_variants(args.precision, specs[0].integ, specs[0].term, local) if v["variant"] == variant]
        tune_report = {"trials": [{**info[0], "refill_threshold": refill, "ms": None}]}
    else:
        tuned, tune_report = K.autotune(specs, precision=args.precision, device=local)
    sweep = K.DeviceSweep(specs, precision=args.precision, device=local, launch=tuned)
    stream = torch.cuda.current_stream(local)
    for _ in range(args.warmup):
        sweep.run(stats=False)
    torch.cuda.synchronize()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2 (126 MB)

    def barrier():
        if world > 1:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        step_ms = _timed_steps(sweep, args.steps, stream, flush)
        torch.cuda.synchronize()
        barrier()
    clock = clocks.summary()
    stats = sweep.stats()
    elapsed_ms = shard.max_over_ranks(float(sum(step_ms)))
    value = job_total * args.steps / (elapsed_ms / 1e3)

    # Roofline of the trace kernel: algorithmic FLOPs per launch over its event-timed duration
    # (each timed graph launch holds this one kernel and two small memsets).
    kernel_ms = statistics.mean(step_ms)
    flops = algorithmic_flops(stats)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    peak64 = _lib.fma_peak_tflops(local, True)

    extra: dict = {}
    summary: dict = {}
    single = world == 1 and not args.kernel_only
    cpu = None
    if single:
        # The oracle on a bounded sample of the same photons: the CPU baseline, and the sweep's
        # parity against the oracle at bench size (codes, terminal states) on those photons.
        if not args.no_cpu:
            cpu, kept = cpu_baseline(specs, keep=True)
            extra["sweep_vs_oracle_sample"] = summary["sweep_vs_oracle_sample"] = sample_parity(K, specs, sweep, kept)
            del kept
        # Plain kernels (one thread per photon, no queue) on the same images: the reference
        # operation order (the plain FP64 baseline) and the fast64 arithmetic.
        plain, t_plain, plain_block, plain_by_block = best_plain(K, specs, local, stream, flush, 1)
        extra["plain_fp64_rays_s"] = total / (t_plain * 1e-3)
        extra["plain_fp64_block"] = plain_block
        extra["plain_fp64_ms_by_block"] = plain_by_block
        extra["persistent_rays_s"] = total / (kernel_ms * 1e-3)
        extra["speedup_persistent_vs_plain"] = t_plain / kernel_ms
        extra["mask_identical_persistent_vs_plain"] = bool(torch.equal(plain.tensors["state"], sweep.tensors["state"]))
        extra["escape_surface_vs_plain"] = escape_surface_errors(K, specs, sweep, plain)
        plain.close()
        del plain
        torch.cuda.empty_cache()
        fplain, t_fplain, fplain_block, _ = best_plain(K, specs, local, stream, flush, 1, precision="fast64")
        extra["fast64_plain_rays_s"] = total / (t_fplain * 1e-3)
        extra["fast64_plain_block"] = fplain_block
        extra["speedup_persistent_vs_fast64_plain"] = t_fplain / kernel_ms
        extra["mask_identical_fast64_plain_vs_persistent"] = bool(torch.equal(fplain.tensors["state"],
                                                                              sweep.tensors["state"]))
        fplain.close()
        del fplain
        torch.cuda.empty_cache()
        summary["sweep"] = {k: extra[k] for k in ("persistent_rays_s", "plain_fp64_rays_s", "fast64_plain_rays_s",
                                                   "speedup_persistent_vs_plain", "speedup_persistent_vs_fast64_plain",
                                                   "mask_identical_persistent_vs_plain")}
        if args.workload == "sweep":
            extra["edge_rms_px_vs_bardeen"] = sweep_edge_errors(K, specs, sweep.tensors["state"].cpu().numpy(),
                                                                sweep.offsets)
        for name in ("spin99_1024", "spin99_2048"):
            m = mixed_vs_plain(K, local, stream, flush, name, oracle_check=not args.no_cpu)
            extra[f"mixed_vs_plain_{name[-4:]}"] = m
            summary[f"mixed_{name[-4:]}"] = {
                "speedup_vs_plain_fp64": m["speedup_mixed_vs_plain"],
                "near_band_speedup_vs_plain_fp64": m["speedup_mixed_near_vs_plain"],
                "near_band_escaped_beyond_10rtol_vs_oracle": m.get("mixed_near_vs_oracle", {}).get("beyond_10rtol"),
                "near_band_escaped_beyond_bar_vs_oracle": m.get("mixed_near_vs_oracle", {}).get("beyond_bar"),
                "speedup_vs_fast64_plain": m["speedup_mixed_vs_fast64_plain"],
                "speedup_vs_fast64_persistent": m["speedup_mixed_vs_fast64_persistent"],
                "mask_identical_vs_plain": m["mask_identical"], "pixels_differing_vs_plain": m["pixels_differing"],
                "pixels_differing_vs_oracle": m.get("pixels_differing_vs_oracle"),
                "escaped_beyond_10rtol_vs_oracle": m.get("mixed_vs_oracle", {}).get("beyond_10rtol"),
                "escaped_beyond_bar_vs_oracle": m.get("mixed_vs_oracle", {}).get("beyond_bar")}
            torch.cuda.empty_cache()
    e2e = None
    if not args.kernel_only:
        # End to end through the public API on every rank: pinned host Y0 in, every result array
        # out, each rank its own share; the job's time is the slowest rank's.
        y0 = torch.empty((total, 8), dtype=torch.float64, pin_memory=True).numpy()
        for k, p in enumerate(pieces):
            sl = slice(int(sweep.offsets[k]), int(sweep.offsets[k + 1]))
            y0[sl] = K.initial_states(specs_all[p.image].camera, specs_all[p.image].spacetime, device=local)[
                p.first:p.first + p.count]
        outs = {name: torch.empty(shape, dtype=dt, pin_memory=True).numpy() for name, shape, dt in (
            ("Y", (total, 8), torch.float64), ("state", (total,), torch.int64), ("n_steps", (total,), torch.int64),
            ("n_rejected", (total,), torch.int64), ("lam", (total,), torch.float64),
            ("max_null_error", (total,), torch.float64), ("max_energy_drift", (total,), torch.float64),
            ("max_lz_drift", (total,), torch.float64), ("max_carter_drift", (total,), torch.float64))}
        outs["event_Y"] = None
        outs["event_hit"] = None
        sweep.close()
        del sweep
        torch.cuda.empty_cache()
        K.trace_images(specs, precision=args.precision, Y0=y0, out=outs, device=local, launch=tuned)
        e2e_steps = max(1, min(args.steps, 3))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            K.trace_images(specs, precision=args.precision, Y0=y0, out=outs, device=local, launch=tuned)
        e2e_s = shard.max_over_ranks((time.perf_counter() - t0) / e2e_steps)
        d2h = sum(a.nbytes for a in outs.values() if a is not None)
        e2e = {"value": job_total / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": int(y0.nbytes),
               "d2h_bytes_per_step": int(d2h)}
        counts = np.bincount(outs["state"], minlength=7)
        extra["state_counts"] = {n: int(c) for n, c in zip(
            ("RUNNING", "ESCAPED", "CAPTURED", "MAX_AFFINE", "FAILURE", "OUT_OF_DOMAIN", "DISK_HIT"), counts)}
    if single and args.workload == "sweep":
        # The other two headline workloads, each with its own roofline and CPU baseline.
        bis = bisect_line(K, argparse.Namespace(steps=3, warmup=3, no_cpu=args.no_cpu, precision="fast64"))
        extra["bisect"] = bis
        summary["bisect"] = {"rays_s": bis["value"], "frac_fp64": bis["roofline"]["frac"],
                             "cpu_rays_s": (bis["cpu_baseline"] or {}).get("value"),
                             "edge_rms_over_rtol_median": {k: v["rms_over_rtol_median"]
                                                           for k, v in bis["edge_error_vs_bardeen"].items()}}
        torch.cuda.empty_cache()
        lens = lensing_line(K, argparse.Namespace(steps=3, warmup=3, no_cpu=args.no_cpu))
        extra["lensing"] = lens
        summary["lensing"] = {"rays_s": lens["value"], "e2e_rays_s": lens["e2e"]["value"],
                              "frac_fp64": (lens["roofline"] or {}).get("frac"),
                              "cpu_rays_s": (lens["cpu_baseline"] or {}).get("value"),
                              "fd_max_rel_h1e-6": lens["fd_check"]["max_rel"],
                              "fd_worst20_max_rel_best_h": lens["fd_check"]["worst20_max_rel_best_h"],
                              "fd_vs_oracle_p999_rel": (lens.get("fd_vs_oracle") or {}).get("p999_rel"),
                              "fit": [lens["gauss_newton"]["spin"], lens["gauss_newton"]["inclination_deg"]]}
    if rank == 0:
        chosen = [t for t in tune_report["trials"] if t["variant"] == tuned.variant
                  and t["refill_threshold"] == tuned.refill_threshold][0]
        line = {
            "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "photons": job_total, "images": len(specs_all),
                       "photons_per_gpu": total, "precision": args.precision,
                       "kernel": "persistent work queue, CUDA-graph launch",
                       "parallelism": (f"shards{world} (the workload replicated per GPU with the observer turned in "
                                       f"azimuth; images cut into pixel pieces of equal predicted cost; no data-path "
                                       f"collective)"),
                       "launch": {**{k: v for k, v in chosen.items() if k != "ms"},
                                  "finalists_full_size_ms": {f"{t['variant']}:{t['refill_threshold']}": t["ms"]
                                                             for t in tune_report.get("final") or []}},
                       "l2": "256 MB buffer written between timed steps (> 126 MB L2)",
                       "summary": summary},
            "e2e": e2e, "gpu_launches": args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64, "traffic": None,
                         "peak_source": "measured FP64 FMA chains on this device (krr_fma_peak)",
                         "algorithmic_flop_per_launch": flops, "kernel_ms": kernel_ms},
            "cpu_baseline": cpu, "clocks": clock,
            "queue": {"attempts": stats["attempts"], "accepted": stats["accepted"],
                      "lane_occupancy": stats["busy_slots"] / max(stats["lane_slots"], 1)},
            **extra,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _line(metric: str, value: float, unit: str, args, ms_per_step: float, config: dict, **rest) -> dict:
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": config, **rest}


def bisect_cases(K, rtols=(1e-6, 1e-8, 1e-10), n_angles: int = 1440, r_o: float = 1.0e5):
    """The 36 cases (12 spacetimes/inclinations x 3 tolerances) of the batched edge bisection."""
    angles = 2.0 * math.pi * np.arange(n_angles) / n_angles
    cases = []
    for rtol in rtols:
        for spin in (0.0, 0.5, 0.9, 0.99):
            for incl in (17.0, 60.0, 85.0):
                cases.append(K.edge_study(K.Spacetime(1.0, spin), incl, r_o, rtol, angles, bracket=(2.0, 8.0)))
    return cases


def bisect_cpu_baseline(K, cases, target_s: float = 15.0) -> dict:
    """The oracle (all host threads) on the first-halving rays (rho = 5 M) of a strided sample of
    the bisection items: rays/s of the same integrations the bisection runs."""
    from oracle import oracle as O

    def run(stride: int):
        n = 0
        t0 = time.perf_counter()
        for c in cases:
            ang = c.angles[::stride]
            rho = 0.5 * (c.r_lo[::stride] + c.r_hi[::stride])
            a = c.centre[0] + rho * np.cos(ang)
            b = c.centre[1] + rho * np.sin(ang)
            integ, term = K.edge_options(c.rtol, c.r_o)
            y0 = O.initial_states(1.0, c.spacetime.spin, c.r_o, c.inclination_deg, 0.0, a, b)
            O.integrate(1.0, c.spacetime.spin, y0, O.Options(rtol=integ.rtol, atol=integ.atol, max_steps=integ.max_steps,
                                                           lambda_max=integ.lambda_max, horizon_epsilon=1e-6,
                                                           escape_radius=c.r_o))
            n += ang.size
        return n, time.perf_counter() - t0

    stride = 1440
    n, dt = run(stride)
    while dt < 1.0 and stride > 1:
        stride = max(1, stride // 8)
        n, dt = run(stride)
    reps = 1
    if stride == 1 and dt < target_s:
        reps = max(1, int(math.ceil(target_s / max(dt, 1e-3))))
    else:
        stride = max(1, int(stride * dt / target_s))
    n = 0
    dt = 0.0
    for _ in range(reps):
        n_k, dt_k = run(stride)
        n += n_k
        dt += dt_k
    return {"value": n / dt, "unit": "rays/s", "cores": os.cpu_count(), "kind": "port",
            "sample": (f"{n} first-halving rays (every {ordinal(stride)} angle of each of the {len(cases)} cases, "
                       f"{reps} pass(es)), {dt:.1f} s")}


def bisect_line(K, args) -> dict:
    """Config 4: every item of every case in one persistent launch; the reference runs one
    integrate_batch per halving (study_edge_bisection.py:53-68)."""
    from kerrray_b200 import _lib

    import dataclasses

    from kerrray_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    all_cases = bisect_cases(K)
    # Under torchrun each rank bisects a contiguous run of the (case, direction) items of equal
    # predicted cost; a direction's bisection depends only on its own history.
    runs = shard.shard_items([c.rtol ** -0.2 for c in all_cases], [c.angles.size for c in all_cases], rank, world)
    cases = [dataclasses.replace(all_cases[k], angles=all_cases[k].angles[f:f + n], r_lo=all_cases[k].r_lo[f:f + n],
                                 r_hi=all_cases[k].r_hi[f:f + n]) for k, f, n in runs]
    n_items = sum(c.angles.size for c in all_cases)
    iterations = 36
    precision = "reference" if args.precision == "reference" else "fast64"
    for _ in range(args.warmup):
        K.bisect_edges(cases, 2, precision=precision, device=local)
    with ClockSampler(local) as clocks:
        kms, walls = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            res, stats = K.bisect_edges(cases, iterations, precision=precision, item_failures=True, device=local)
            walls.append(time.perf_counter() - t0)
            kms.append(stats["kernel_ms"])
    rays = n_items * iterations
    kernel_ms = shard.max_over_ranks(statistics.mean(kms))
    wall_s = shard.max_over_ranks(statistics.mean(walls))
    if world > 1:  # every rank's brackets to every rank, in item order
        import torch.distributed as dist

        parts = [None] * world
        dist.all_gather_object(parts, [(k, f, r) for (k, f, _), r in zip(runs, res)])
        full = [[np.empty(c.angles.size), np.empty(c.angles.size), np.zeros(c.angles.size, np.int64)] for c in all_cases]
        for part in parts:
            for k, f, (r_mid, width, fails) in part:
                for dst, src in zip(full[k], (r_mid, width, fails)):
                    dst[f:f + src.size] = src
        res = [tuple(x) for x in full]
        cases = all_cases
    flops = algorithmic_flops({"attempts": stats["attempts"], "accepted": stats["accepted"], "photons": rays})
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    peak64 = _lib.fma_peak_tflops(0, True)
    from kerrray_b200.bisect import edge_error

    errors = {}
    per_case = []
    # Directions that lost a photon (ended neither ESCAPED nor CAPTURED) steer their bracket
    # wrongly: the a* = 0 cases' two polar directions (alpha = rho cos(pi/2) ~ 1e-16 M) cross
    # the spin axis at every halving, in the reference as here. The edge error is taken over
    # the other directions; the lost photons and directions are counted beside it.
    for c, (r_mid, width, fails) in zip(cases, res):
        ok = fails == 0
        e = edge_error(c, r_mid, keep=ok)
        per_case.append({"spin": c.spacetime.spin, "inclination_deg": c.inclination_deg, "rtol": c.rtol,
                         "rms_M": e["rms_M"], "max_M": e["max_M"], "lost": int(fails.sum()),
                         "lost_directions": int((~ok).sum())})
        key = f"{c.rtol:g}"
        d = errors.setdefault(key, {"rms_M": [], "max_M": [], "lost": 0, "lost_directions": 0, "max_width_M": 0.0})
        d["rms_M"].append(e["rms_M"])
        d["max_M"].append(e["max_M"])
        d["lost"] += int(fails.sum())
        d["lost_directions"] += int((~ok).sum())
        d["max_width_M"] = max(d["max_width_M"], float(np.max(width)))
    summary = {k: {"rms_M_median": float(np.median(v["rms_M"])), "rms_M_max": float(np.max(v["rms_M"])),
                   "max_M": float(np.max(v["max_M"])), "rms_over_rtol_median": float(np.median(v["rms_M"])) / float(k),
                   "lost": v["lost"], "lost_directions": v["lost_directions"], "max_width_M": v["max_width_M"],
                   "over": "directions without a lost photon"} for k, v in errors.items()}
    cpu = None if (args.no_cpu or world > 1) else bisect_cpu_baseline(K, cases)
    return _line("edge-bisection rays/s per B200 (batched, one persistent launch)", rays / (kernel_ms * 1e-3),
                 "rays/s", args, kernel_ms,
                 {"workload": WORKLOADS["bisect"], "items": n_items, "iterations": iterations, "cases": len(cases),
                  "precision": precision, "kernel": "k_bisect_edges (one item per lane, all halvings in registers; idle lanes trace the "
                            "next midpoints ahead, results bit-identical to sequential bisection)",
                  "curve": "edge error against Bardeen's exact curve (polar radius by bisection on its parameter)",
                  "l2": "inputs < 1 MB; the work is FP64 arithmetic in registers"},
                 e2e={"value": rays / wall_s, "unit": "rays/s", "h2d_bytes_per_step": n_items * 36,
                      "d2h_bytes_per_step": n_items * 24},
                 gpu_launches=args.steps,
                 roofline={"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                           "frac": achieved / peak64, "traffic": None,
                           "peak_source": "measured FP64 FMA chains on this device (krr_fma_peak)"},
                 cpu_baseline=cpu, clocks=clocks.summary(), edge_error_vs_bardeen=summary,
                 worst_cases=sorted(per_case, key=lambda d: -d["max_M"])[:6],
                 queue={"attempts": stats["attempts"], "accepted": stats["accepted"],
                        "lane_occupancy": stats["busy_slots"] / max(stats["lane_slots"], 1),
                        "speculative_photons": stats["speculative"],
                        "discarded_attempts": stats["discarded_attempts"],
                        "note": "attempts: the sequential bisection's; discarded attempts (midpoints traced "
                                "ahead on the side not taken) are outside the roofline's work"})


def _init_ranks():
    """(rank, world, local): the process group over NCCL under torchrun, nothing otherwise."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, world, local


def _finish_ranks(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_bisect(args) -> None:
    import kerrray_b200 as K

    rank, world, _ = _init_ranks()
    line = bisect_line(K, args)
    line["n_gpus"] = world
    if rank == 0:
        print(json.dumps(line), flush=True)
    _finish_ranks(world)


# FP64 floating-point operations the lensing kernels execute per accepted step of their rays
# (forward pass with landing and stage records; reverse sweep from the records, two rows, and the
# camera chain), from their FP64 instruction counts in one ncu capture of every 4th ray of this
# workload (dadd + dmul + 2 dfma thread instructions of the launches, divided by the rays'
# 4,414,655 accepted steps; profiles/).
LENS_FLOP_PER_STEP = 3485


def _fd_error(jac: np.ndarray, fd: np.ndarray) -> np.ndarray:
    """|J - FD| relative to max(|FD|, the column's RMS over the rays): entries near zero are
    measured against their column's scale, where FD round-off (~eps |x| / h) sits."""
    return np.abs(jac - fd) / np.maximum(np.abs(fd), np.sqrt(np.mean(fd**2, axis=0, keepdims=True)))


def _fd_replay(A, sub, a, b, spin: float, incl: float, h: float) -> np.ndarray:
    """Central differences of the recorded map (the controller held fixed) in (alpha, beta, a*, i)."""
    fd = np.zeros((a.numel(), 2, 4))
    for p_ in range(4):
        outs = []
        for sgn in (1.0, -1.0):
            d = [0.0] * 4
            d[p_] = sgn * h
            th, ph = A.replay(sub, a + d[0], b + d[1], spin + d[2], incl + d[3])
            outs.append(np.stack([th.cpu().numpy(), ph.cpu().numpy()], axis=1))
        fd[:, :, p_] = (outs[0] - outs[1]) / (2 * h)
    return fd


def lensing_cpu_baseline(K, a_np: np.ndarray, b_np: np.ndarray, spin: float, incl: float, r_o: float,
                         target_s: float = 12.0) -> tuple[dict, dict]:
    """The reference's way to this Jacobian: central differences (h = 1e-6) of its own
    integration, 8 oracle traces per ray at the same rtol 1e-10, timed on all host threads on a
    strided sample of the rays. The FD traces are landed on the escape surface on the device
    (untimed) and returned with the sample for the comparison with the adjoint."""
    from oracle import oracle as O

    opts = O.Options(rtol=1e-10, atol=1e-12, escape_radius=r_o)
    h = 1e-6
    threads = os.cpu_count() or 1

    def traces(idx):
        outs = []
        for p_ in range(4):
            for sgn in (1.0, -1.0):
                d = np.zeros(4)
                d[p_] = sgn * h
                s_ = spin + d[2]
                y0 = O.initial_states(1.0, s_, r_o, incl + d[3], 0.0, a_np[idx] + d[0], b_np[idx] + d[1])
                outs.append((s_, O.integrate(1.0, s_, y0, opts, threads=threads)))
        return outs

    stride = max(1, a_np.size // 64)
    t0 = time.perf_counter()
    traces(np.arange(0, a_np.size, stride))
    dt = time.perf_counter() - t0
    n_probe = a_np[::stride].size
    want = max(16, int(n_probe * target_s / max(dt, 1e-3)))
    stride = max(1, a_np.size // want)
    idx = np.arange(0, a_np.size, stride)
    t0 = time.perf_counter()
    outs = traces(idx)
    dt = time.perf_counter() - t0
    fd = np.zeros((idx.size, 2, 4))
    for p_ in range(4):
        dirs = []
        for sgn in (0, 1):
            s_, o = outs[2 * p_ + sgn]
            dirs.append(surface_directions(K, (K.Spacetime(1.0, s_), r_o), o["Y"], o["state"]))
        fd[:, :, p_] = (dirs[0] - dirs[1]) / (2 * h)
    line = {"value": idx.size / dt, "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": ((f"every {ordinal(stride)} of the {a_np.size} rays" if stride > 1 else f"all {a_np.size} rays") +
                       f" ({idx.size} rays, {dt:.1f} s): central differences "
                       f"(h = 1e-6) of the oracle's integration, 8 traces per ray at rtol 1e-10, OpenMP {threads} "
                       f"threads")}
    return line, {"idx": idx, "fd": fd}


def lensing_line(K, args) -> dict:
    """Config 5: forward pass with tape + reverse sweep for ~50k rays; FD checks; Gauss-Newton
    fit of (a*, i) from (0.5, 50 deg) to the map at (0.8, 60 deg)."""
    import torch

    from kerrray_b200 import _lib
    from kerrray_b200 import adjoint as A

    from kerrray_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    spin, incl, r_o = 0.8, 60.0, 1000.0
    alpha, beta = K.edge_distant_rays(spin, incl, device=local)
    stride = max(1, int(getattr(args, "lens_stride", 1)))
    if stride > 1:  # every stride-th ray (a smaller case of the same kernels, for profiling)
        alpha, beta = alpha[::stride].contiguous(), beta[::stride].contiguous()
    n_job = alpha.numel()
    # Under torchrun each rank maps a contiguous share of the rays (independent, equal cost).
    share = shard.split_range(n_job, rank, world)
    alpha, beta = alpha[share].contiguous(), beta[share].contiguous()
    n = alpha.numel()
    stream = torch.cuda.current_stream(local)
    # One tape for every call (the step sizes, checkpoints and the default stage pool), as a
    # caller that maps repeatedly keeps it.
    ws = torch.empty(A.workspace_bytes(n), dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        res = K.lensing_map(alpha, beta, spin, incl, workspace=ws, device=local)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms = []
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = K.lensing_map(alpha, beta, spin, incl, workspace=ws, device=local)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    kernel_ms = shard.max_over_ranks(statistics.mean(ms))
    # The same map with the rays ordered by the previous map's step counts, as the fit runs it.
    ms_hint = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        K.lensing_map(alpha, beta, spin, incl, workspace=ws, order=res.n_steps, device=local)
        e1.record(stream)
        e1.synchronize()
        ms_hint.append(e0.elapsed_time(e1))
    res = K.lensing_map(alpha, beta, spin, incl, workspace=ws, device=local)  # the tape of the default order
    ok = int(((res.status == 0) & (res.state == 1)).sum().item())
    tape = A.tape_usage(res, device=local)
    steps = res.n_steps.double()
    total_steps = float(steps.sum().item())
    # End to end: pinned host alpha, beta in; theta, phi and the Jacobian out.
    a_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    b_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    a_host.copy_(alpha.cpu())
    b_host.copy_(beta.cpu())
    th_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    ph_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    jac_host = torch.empty((n, 2, 4), dtype=torch.float64, pin_memory=True)
    walls = []
    for it in range(1 + max(1, args.steps)):  # the first, untimed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a_d = a_host.to(f"cuda:{local}", non_blocking=True)
        b_d = b_host.to(f"cuda:{local}", non_blocking=True)
        r = K.lensing_map(a_d, b_d, spin, incl, workspace=ws, device=local)
        th_host.copy_(r.theta, non_blocking=True)
        ph_host.copy_(r.phi, non_blocking=True)
        jac_host.copy_(r.jac, non_blocking=True)
        torch.cuda.synchronize()
        if it:
            walls.append(time.perf_counter() - t0)
        del r
    e2e = {"value": n_job / shard.max_over_ranks(statistics.mean(walls)), "unit": "rays/s",
           "h2d_bytes_per_step": 2 * 8 * n_job, "d2h_bytes_per_step": (2 + 8) * 8 * n_job}
    if world > 1:  # every rank's accepted steps (the roofline's work)
        import torch.distributed as dist

        t = torch.tensor([total_steps], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t)
        total_steps = float(t.item())
    checks = not getattr(args, "kernel_only", False) and world == 1
    fd_check, cpu, fd_vs_oracle, fit, fit_s = None, None, None, None, None
    # FD of the recorded map on a strided sample of >= 8k rays (h = 1e-6); the 20 worst rays
    # again at h = 1e-5 and 1e-7: an error that falls with another h is the FD's, not the adjoint's.
    idx = torch.arange(0, n, max(1, n // 8192), device=alpha.device) if checks else None
    if checks:
        fd_check, cpu, fd_vs_oracle, fit, fit_s = _lensing_checks(K, A, args, alpha, beta, idx, res, spin, incl, r_o)
    mag = K.magnification(res.jac)
    peak64 = _lib.fma_peak_tflops(0, True)
    roofline = None
    if LENS_FLOP_PER_STEP is not None:
        achieved = LENS_FLOP_PER_STEP * total_steps / (kernel_ms * 1e-3) / 1e12
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                    "frac": achieved / peak64, "traffic": None,
                    "work": f"{LENS_FLOP_PER_STEP} FP64 FLOP per accepted step (the kernels' FP64 instruction "
                            f"counts from ncu, dfma = 2) x {int(total_steps)} accepted steps",
                    "peak_source": "measured FP64 FMA chains on this device (krr_fma_peak)"}
    gn = None if fit is None else {"start": [0.5, 50.0], "target": [spin, incl], "spin": fit["spin"],
                                   "inclination_deg": fit["inclination_deg"], "iterations": len(fit["history"]) - 1,
                                   "map_evaluations": fit["evaluations"], "final_cost": fit["history"][-1]["cost"],
                                   "seconds": fit_s}
    return _line("lensing-map adjoint rays/s per B200 (forward with tape + reverse sweep, 4 parameters)",
                 n_job / (kernel_ms * 1e-3), "rays/s", args, kernel_ms,
                 {"workload": WORKLOADS["lensing"] + (f" (every {ordinal(stride)} ray)" if stride > 1 else ""),
                  "rays": n_job, "rays_per_gpu": n, "checkpoint_every": 32,
                  "kernel": ("k_lensing_forward (one ray per thread) + k_lensing_reverse_staged (two threads per "
                             "ray, from the stage records) + k_lensing_reverse (checkpoint recomputation, for rays "
                             "the stage pool could not hold), for each half of the rays, the halves on two streams"),
                  "ray_order": ("increasing impact parameter hypot(alpha, beta), the default; by the previous "
                                "map's step counts (as the fit runs it): "
                                f"{shard.max_over_ranks(statistics.mean(ms_hint)):.3f} ms per map"),
                  "stage_tape": {"rays_from_records": tape["staged_rays"], "chunks_used": tape["chunks_used"],
                                 "chunks_held": tape["chunks_total"], "bytes_per_step": 240},
                  "l2": ("tape in HBM (one workspace for every call), written once by the forward pass and read "
                         "once by the reverse sweep: step sizes (n x 8192 x 8 B) and 240 B of stage records per "
                         "accepted step")},
                 e2e=e2e, gpu_launches=(6 if n > 256 else 3) * args.steps,  # 3 kernels per half of the rays
                 roofline=roofline, cpu_baseline=cpu, clocks=clocks.summary(),
                 rays_ok=ok, accepted_steps={"mean": float(steps.mean().item()), "max": int(steps.max().item()),
                                             "total": int(total_steps)},
                 fd_check=fd_check, fd_vs_oracle=fd_vs_oracle, gauss_newton=gn,
                 magnification={"median": float(mag.median().item()), "max": float(mag.max().item())})


def _lensing_checks(K, A, args, alpha, beta, idx, res, spin, incl, r_o):
    """The lensing line's checks: FD of the recorded map, the CPU baseline with FD of the
    oracle, and the Gauss-Newton fit."""
    import torch

    sub = A.lensing_map(alpha[idx], beta[idx], spin, incl)
    fd = _fd_replay(A, sub, alpha[idx], beta[idx], spin, incl, 1e-6)
    jac = sub.jac.cpu().numpy()
    err = _fd_error(jac, fd)
    worst = np.argsort(-err.reshape(err.shape[0], -1).max(axis=1))[:20]
    by_h = {"1e-6": float(err[worst].max())}
    best = err[worst].reshape(worst.size, -1).max(axis=1)
    for h in (1e-5, 1e-7):
        w = torch.as_tensor(idx.cpu().numpy()[worst], device=alpha.device)
        sub_w = A.lensing_map(alpha[w], beta[w], spin, incl)
        e_h = _fd_error(sub_w.jac.cpu().numpy(), _fd_replay(A, sub_w, alpha[w], beta[w], spin, incl, h))
        by_h[f"{h:g}"] = float(e_h.max())
        best = np.minimum(best, e_h.reshape(worst.size, -1).max(axis=1))
    fd_check = {"rays": int(idx.numel()), "h": 1e-6, "max_rel": float(err.max()), "median_rel": float(np.median(err)),
                "worst20_max_rel_by_h": by_h, "worst20_max_rel_best_h": float(best.max()),
                "metric": "|J - FD| / max(|FD|, column RMS), FD of the recorded map"}
    cpu, fd_vs_oracle = None, None
    if not args.no_cpu:
        cpu, ref = lensing_cpu_baseline(K, alpha.cpu().numpy(), beta.cpu().numpy(), spin, incl, r_o)
        ridx = torch.as_tensor(ref["idx"], device=alpha.device)
        jr = A.lensing_map(alpha[ridx], beta[ridx], spin, incl).jac.cpu().numpy()
        e_ref = _fd_error(jr, ref["fd"])
        per_ray = np.nanmax(e_ref.reshape(e_ref.shape[0], -1), axis=1)
        fd_vs_oracle = {"rays": int(ridx.numel()), "h": 1e-6, "max_rel": float(np.nanmax(e_ref)),
                        "p999_rel": float(np.nanquantile(per_ray, 0.999)), "median_rel": float(np.nanmedian(e_ref)),
                        "note": "the oracle's controller is live: a ray whose +-h traces take different step "
                                "sequences has a jump in its FD; the recorded-map check holds the controller fixed",
                        "metric": "|J - FD| / max(|FD|, column RMS), FD of the oracle's adaptive integration, "
                                  "each trace landed on the escape surface"}
    t0 = time.perf_counter()
    fit = K.fit_spin_inclination(alpha, beta, res.theta, res.phi, p0=(0.5, 50.0), iterations=20)
    torch.cuda.synchronize()
    fit_s = time.perf_counter() - t0
    return fd_check, cpu, fd_vs_oracle, fit, fit_s


def run_lensing(args) -> None:
    import kerrray_b200 as K

    rank, world, _ = _init_ranks()
    line = lensing_line(K, args)
    line["n_gpus"] = world
    if rank == 0:
        print(json.dumps(line), flush=True)
    _finish_ranks(world)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="sweep")
    ap.add_argument("--precision", choices=("reference", "fast64", "mixed"), default="fast64")
    ap.add_argument("--launch", default="", help="VARIANT:REFILL launch shape instead of the autotuner's choice")
    ap.add_argument("--lens-stride", type=int, default=1, help="lensing workload: every k-th ray only")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the device launches only (no plain-kernel, end-to-end or CPU legs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "bisect":
        run_bisect(args)
    elif args.workload == "lensing":
        run_lensing(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
