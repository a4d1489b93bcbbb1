"""Benchmark of KerrRay's per-ray hot path on B200.

Workload (one "step"): the batched FP64 sweep -- spins {0, 0.5, 0.9, 0.99} x inclinations
{17, 60, 85} deg x resolutions {128, 256, 512}^2 x rtol {1e-6, 1e-8, 1e-10} (atol = 1e-2 rtol),
observer at r_o = 1000 M, image plane +-8 M, reference defaults otherwise: 108 images,
12,386,304 photons in one persistent launch (camera, Dormand-Prince 5(4) integration and
classification on the device). Metric: rays/s, the whole job over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank traces the full sweep on its own GPU (weak scaling; the photons are
independent, there is no data-path collective); the time is the max over ranks.
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


def algorithmic_flops(stats: dict) -> float:
    return FLOP_PER_ATTEMPT * stats["attempts"] + FLOP_PER_ACCEPT * stats["accepted"] + FLOP_PER_RAY * stats["photons"]


WORKLOADS = {
    "sweep": WORKLOAD,
    "sweep128": "the 36 128^2 images of the sweep (a*{0,0.5,0.9,0.99} x i{17,60,85} x rtol{1e-6,1e-8,1e-10})",
    "spin99_1024": "a*=0.99, i=85deg, r_o=1000 M, +-8 M, 1024^2, rtol 1e-6, atol 1e-8",
}


def workload_specs(K, name: str):
    if name == "sweep":
        return sweep_specs(K)
    if name == "sweep128":
        return sweep_specs(K, resolutions=(128,))
    if name == "spin99_1024":
        cam = K.Camera(radius=1000.0, inclination_deg=85.0, fov=8.0, resolution=1024)
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


def time_cpu_sample(specs, stride: int, offset: int = 0) -> tuple[int, float, int]:
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    n_rays = 0
    t0 = time.perf_counter()
    for k, idx in cpu_sample(specs, stride, offset):
        s = specs[k]
        a, b = O.pixel_coordinates(s.camera.fov, s.camera.resolution)
        y0 = O.initial_states(s.spacetime.mass, s.spacetime.spin, s.camera.radius, s.camera.inclination_deg,
                              s.camera.phi_deg, a.ravel()[idx], b.ravel()[idx])
        O.integrate(s.spacetime.mass, s.spacetime.spin, y0,
                    O.Options(rtol=s.integ.rtol, atol=s.integ.atol), threads=threads)
        n_rays += idx.size
    return n_rays, time.perf_counter() - t0, threads


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


def cpu_baseline(specs, target_s: float = 15.0) -> dict:
    from oracle.build import build

    build()
    stride = calibrate_stride(specs, target_s)
    n, dt, threads = time_cpu_sample(specs, stride, 1)
    return {"value": n / dt, "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": f"every {stride}th photon of the 108-image sweep ({n} rays, {dt:.1f} s), C++ oracle, "
                      f"OpenMP {threads} threads"}


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
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "photons": total, "sample_stride": stride},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads, "kind": "port",
                         "sample": f"every {stride}th photon per step ({rays // max(args.steps, 1)} rays/step), "
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


def mixed_vs_plain(K, local: int, stream, flush) -> dict:
    """Mixed persistent + FP64 re-trace against the plain FP64 kernel on the 1024^2, a*=0.99,
    i=85 deg image (rtol 1e-6): rays/s of each and whether the two shadow masks are identical."""
    import torch

    specs = workload_specs(K, "spin99_1024")
    total = specs[0].n_rays
    tuned, _ = K.autotune(specs, precision="mixed", device=local)
    mixed = K.DeviceSweep(specs, precision="mixed", device=local,
                          launch=K.LaunchConfig(variant=tuned.variant, refill_threshold=tuned.refill_threshold,
                                                retrace=True))
    fast = K.DeviceSweep(specs, precision="fast64", device=local, launch=K.autotune(specs, precision="fast64", device=local)[0])
    plain = K.DeviceSweep(specs, precision="reference", device=local, launch=K.LaunchConfig(plain=True))
    for sw in (mixed, fast, plain):
        sw.run()
    t_mixed = min(_timed_steps(mixed, 3, stream, flush))
    t_fast = min(_timed_steps(fast, 3, stream, flush))
    t_plain = min(_timed_steps(plain, 2, stream, flush))
    ms = mixed.stats()
    same = bool(torch.equal(mixed.tensors["state"], plain.tensors["state"]))
    differ = int((mixed.tensors["state"] != plain.tensors["state"]).sum().item())
    esc = (plain.tensors["state"] == 1) & (mixed.tensors["state"] == 1)
    rel = ((mixed.tensors["Y"] - plain.tensors["Y"]).abs() / plain.tensors["Y"].abs().clamp_min(1.0)).amax(dim=1)
    out = {"workload": WORKLOADS["spin99_1024"], "photons": total,
           "mixed_retrace_rays_s": total / (t_mixed * 1e-3), "fast64_rays_s": total / (t_fast * 1e-3),
           "plain_fp64_rays_s": total / (t_plain * 1e-3), "speedup_mixed_vs_plain": t_plain / t_mixed,
           "mask_identical": same, "pixels_differing": differ, "retraced": int(ms["retraced"]),
           "escaped_max_rel_dY_vs_plain": float(rel[esc].max().item()),
           "escaped_median_rel_dY_vs_plain": float(rel[esc].median().item()),
           "mixed_launch": {"variant": tuned.variant, "refill_threshold": tuned.refill_threshold}}
    for sw in (mixed, fast, plain):
        sw.close()
    return out


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

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    _lib.lib()

    specs = workload_specs(K, args.workload)
    total = sum(s.n_rays for s in specs)
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
    elapsed_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([elapsed_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = world * total * args.steps / (elapsed_ms / 1e3)

    # Roofline of the trace kernel: algorithmic FLOPs per launch over its event-timed duration
    # (each timed graph launch holds this one kernel and two small memsets).
    kernel_ms = statistics.mean(step_ms)
    flops = algorithmic_flops(stats)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    peak64 = _lib.fma_peak_tflops(local, True)

    extra = {}
    e2e = None
    if rank == 0 and not args.kernel_only:
        # Plain FP64 (one thread per photon, reference operation order) on the same images.
        plain = K.DeviceSweep(specs, precision="reference", device=local, launch=K.LaunchConfig(plain=True))
        plain.run(stats=False)
        t_plain = min(_timed_steps(plain, 1, stream, flush))
        extra["plain_fp64_rays_s"] = total / (t_plain * 1e-3)
        extra["persistent_rays_s"] = total / (kernel_ms * 1e-3)
        extra["speedup_persistent_vs_plain"] = t_plain / kernel_ms
        extra["mask_identical_persistent_vs_plain"] = bool(torch.equal(plain.tensors["state"], sweep.tensors["state"]))
        plain.close()
        del plain
        torch.cuda.empty_cache()
        extra["mixed_vs_plain_1024"] = mixed_vs_plain(K, local, stream, flush)
        torch.cuda.empty_cache()
        # End to end through the public API: pinned host Y0 in, every result array out.
        y0 = torch.empty((total, 8), dtype=torch.float64, pin_memory=True).numpy()
        for k, s in enumerate(specs):
            sl = slice(int(sweep.offsets[k]), int(sweep.offsets[k + 1]))
            y0[sl] = K.initial_states(s.camera, s.spacetime, device=local)
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
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            K.trace_images(specs, precision=args.precision, Y0=y0, out=outs, device=local, launch=tuned)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        d2h = sum(a.nbytes for a in outs.values() if a is not None)
        e2e = {"value": world * total / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": int(y0.nbytes),
               "d2h_bytes_per_step": int(d2h)}
        counts = np.bincount(outs["state"], minlength=7)
        extra["state_counts"] = {n: int(c) for n, c in zip(
            ("RUNNING", "ESCAPED", "CAPTURED", "MAX_AFFINE", "FAILURE", "OUT_OF_DOMAIN", "DISK_HIT"), counts)}

    cpu = cpu_baseline(specs) if (rank == 0 and world == 1 and not args.no_cpu and not args.kernel_only) else None
    if rank == 0:
        chosen = [t for t in tune_report["trials"] if t["variant"] == tuned.variant
                  and t["refill_threshold"] == tuned.refill_threshold][0]
        line = {
            "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "photons": total, "images": len(specs),
                       "precision": args.precision, "kernel": "persistent work queue, CUDA-graph launch",
                       "parallelism": f"replicas{world}",
                       "launch": {k: v for k, v in chosen.items() if k != "ms"},
                       "l2": "256 MB buffer written between timed steps (> 126 MB L2)"},
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
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the device launches only (no plain-kernel, end-to-end or CPU legs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
