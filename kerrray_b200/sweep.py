"""Many images in one persistent launch.

An image is what ``compute_shadow`` (``src/kerrray/raytracing/shadow.py:179-211``) traces:
a spacetime, a camera and the integrator/termination options. :func:`trace_images` puts any
number of them (different spins, inclinations, resolutions and tolerances) into one device
work queue: the persistent kernel builds each photon from its image's camera on the device,
integrates it and writes its result row; warps refill lanes from the queue as photons
terminate (``krr_trace_images``). Images are queued in the order given;
:func:`order_by_cost` sorts them most-expensive-first so the tail of the launch is short.

:class:`DeviceSweep` keeps the result arrays in device memory (torch tensors) and launches
through ``krr_trace_images_device`` on the current torch stream -- the form the benchmark
times with its inputs already resident.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Any, Sequence

import numpy as np

from kerrray_b200 import _lib
from kerrray_b200.camera import Camera
from kerrray_b200.types import BatchResult, TerminationState

__all__ = ["ImageSpec", "SweepResult", "DeviceSweep", "LaunchConfig", "order_by_cost", "trace_images", "RETRACE_EDGE",
           "RETRACE_CRITICAL", "RETRACE_CRITICAL_NEAR", "analytic_classes", "escape_directions", "trig_eval"]

RETRACE_EDGE = 1
RETRACE_CRITICAL = 2
RETRACE_CRITICAL_NEAR = 3


def escape_directions(spacetime, Y, state, r_surface: float):
    """(theta, phi) where each escaped ray crosses r = r_surface (``krr_escape_directions``), for
    device tensors ``Y`` (n x 8, float64) and ``state`` (n, int64); NaN where not ESCAPED. Two
    integrations of the same rays are comparable there whatever steps they took."""
    import torch

    if Y.device.type != "cuda" or Y.dtype != torch.float64 or state.dtype != torch.int64:
        raise ValueError("Y must be a float64 and state an int64 CUDA tensor")
    n = int(state.numel())
    Y, state = Y.contiguous(), state.contiguous()
    theta = torch.empty(n, dtype=torch.float64, device=Y.device)
    phi = torch.empty(n, dtype=torch.float64, device=Y.device)
    stream = torch.cuda.current_stream(Y.device).cuda_stream
    _lib.check(_lib.lib().krr_escape_directions(Y.device.index, float(spacetime.mass), float(spacetime.spin),
                                                float(r_surface), Y.data_ptr(), state.data_ptr(), n,
                                                theta.data_ptr(), phi.data_ptr(), stream))
    return theta, phi


def direction_angle(theta1, phi1, theta2, phi2) -> np.ndarray:
    """The angle (rad) between the directions (theta1, phi1) and (theta2, phi2) on the escape
    sphere, per ray: 2 asin(|u1 - u2| / 2) of their unit vectors, well conditioned for small
    angles. Next to a pole phi alone is ill-conditioned (a displacement d on the sky moves phi by
    d / sin theta), so this, not max(|d theta|, |d phi|), measures how far two integrations of a
    ray landed apart. NaN where either direction is NaN (a ray not escaped)."""
    t1, p1, t2, p2 = (np.asarray(x, dtype=np.float64) for x in (theta1, phi1, theta2, phi2))

    def unit(t, p):
        st = np.sin(t)
        return np.stack([st * np.cos(p), st * np.sin(p), np.cos(t)], axis=-1)

    chord = np.linalg.norm(unit(t1, p1) - unit(t2, p2), axis=-1)
    return 2.0 * np.arcsin(np.minimum(1.0, 0.5 * chord))


def trig_eval(which: int, theta, delta=None):
    """The step kernels' sine and cosine forms at the angles of the float64 CUDA tensor ``theta``
    (``krr_trig_eval``): 0 the FP32 sine/cosine of an FP64 angle (mixed accepted states), 1 the
    FP32 shift by ``delta`` from theta's FP32-rounded sine/cosine (mixed stages), 2 the FP64 shift
    by ``delta`` (fast64 stages). Returns (sin, cos) as float64 tensors, NaN where a shift declines."""
    import torch

    if theta.device.type != "cuda" or theta.dtype != torch.float64:
        raise ValueError("theta must be a float64 CUDA tensor")
    theta = theta.contiguous()
    if delta is not None:
        if delta.device != theta.device or delta.dtype != torch.float64 or delta.numel() != theta.numel():
            raise ValueError("delta must be a float64 tensor on theta's device, with theta's length")
        delta = delta.contiguous()
    n = int(theta.numel())
    s = torch.empty(n, dtype=torch.float64, device=theta.device)
    c = torch.empty(n, dtype=torch.float64, device=theta.device)
    stream = torch.cuda.current_stream(theta.device).cuda_stream
    _lib.check(_lib.lib().krr_trig_eval(theta.device.index, int(which), theta.data_ptr(),
                                        None if delta is None else delta.data_ptr(), n, s.data_ptr(),
                                        c.data_ptr(), stream))
    return s, c


def analytic_classes(spacetime, y0: np.ndarray, rtol: float, horizon_epsilon: float = 1e-6) -> np.ndarray:
    """Analytic class of each initial state (``krr_analytic_classes``): 0 escapes, 1 is captured,
    2 lies within the critical band of the boundary (or is not classified)."""
    y0 = np.ascontiguousarray(np.asarray(y0, dtype=np.float64))
    if y0.ndim != 2 or y0.shape[1] != 8:
        raise ValueError(f"Y0 must have shape (n, 8), got {y0.shape}")
    out = np.empty(len(y0), dtype=np.uint8)
    _lib.check(_lib.lib().krr_analytic_classes(float(spacetime.mass), float(spacetime.spin), float(rtol),
                                               float(horizon_epsilon), _lib.ptr(y0), len(y0), _lib.ptr(out)))
    return out


@dataclass(frozen=True)
class ImageSpec:
    """One image of a batched launch, or with ``pixels = (first, count)`` the pixels
    ``first .. first + count - 1`` of its grid (row-major): a share of an image for one GPU."""

    spacetime: Any
    camera: Camera
    integ: Any
    term: Any
    events: Any = None
    pixels: tuple[int, int] | None = None

    def __post_init__(self) -> None:
        if self.pixels is not None:
            first, count = (int(x) for x in self.pixels)
            if count < 1 or first < 0 or first + count > self.camera.n_rays:
                raise ValueError(f"pixel range {self.pixels} lies outside the image's {self.camera.n_rays} pixels")
            object.__setattr__(self, "pixels", (first, count))

    @property
    def n_rays(self) -> int:
        return self.camera.n_rays if self.pixels is None else self.pixels[1]

    @property
    def whole(self) -> bool:
        """True when the entry traces every pixel of its image."""
        return self.pixels is None or self.pixels == (0, self.camera.n_rays)

    def as_struct(self) -> _lib.KrrImage:
        first, count = (0, 0) if self.pixels is None else self.pixels
        return _lib.KrrImage(mass=float(self.spacetime.mass), spin=float(self.spacetime.spin),
                             camera=self.camera.as_struct(), options=_lib.options_struct(self.integ, self.term, self.events),
                             first_pixel=first, pixel_count=count)


@dataclass(frozen=True)
class LaunchConfig:
    """Launch shape of the persistent kernel (0 = library default)."""

    block: int = 0            # threads per block of the plain kernel
    blocks_per_sm: int = 0    # resident blocks per SM (0 = as many as fit)
    refill_threshold: int = 0  # idle lanes before a warp refills (0 = 1)
    plain: bool = False       # one thread per photon instead of the work queue
    variant: int = 0          # compiled launch shape of the persistent kernel
    # Settle the pixels a mixed trace could classify differently with the reference-order FP64
    # kernel: 0 off; 1 (RETRACE_EDGE) afterwards, every pixel not ESCAPED or CAPTURED or unlike a
    # neighbour; 2 (RETRACE_CRITICAL) the photons near the critical curve (analytic classes from
    # the radial potential) beside the main trace, then every photon unlike its class;
    # 3 (RETRACE_CRITICAL_NEAR) that and, for a mixed trace, the escaping photons within 0.35 M of
    # the critical curve in fast FP64 (their exit directions then meet the oracle's bar too).
    retrace: int = 0
    critical_sms: int = 0     # RETRACE_CRITICAL: SMs of the reference-order kernel (0: library default)


def order_by_cost(specs: Sequence[ImageSpec]) -> list[int]:
    """Indices of ``specs`` most expensive first (steps grow like rtol^(-1/5); rays like res^2)."""
    cost = [s.n_rays * (1.0 / s.integ.rtol) ** 0.2 for s in specs]
    return sorted(range(len(specs)), key=lambda k: -cost[k])


def _images(specs: Sequence[ImageSpec]):
    if not specs:
        raise ValueError("need at least one image")
    arr = (_lib.KrrImage * len(specs))()
    for k, s in enumerate(specs):
        arr[k] = s.as_struct()
    offsets = np.zeros(len(specs) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([s.n_rays for s in specs])
    return arr, offsets


def _launch(precision: str, cfg: LaunchConfig | None) -> _lib.KrrLaunch:
    if precision not in _lib.PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_lib.PRECISIONS)}, got {precision!r}")
    cfg = cfg or LaunchConfig()
    return _lib.KrrLaunch(precision=_lib.PRECISIONS[precision], block=cfg.block, blocks_per_sm=cfg.blocks_per_sm,
                          refill_threshold=cfg.refill_threshold, plain=int(cfg.plain), variant=cfg.variant,
                          retrace=int(cfg.retrace), critical_sms=int(cfg.critical_sms))


@dataclass
class SweepResult:
    """Flat per-photon results of a batched launch; image ``k`` owns rows ``offsets[k]:offsets[k+1]``."""

    specs: list[ImageSpec]
    offsets: np.ndarray
    arrays: dict[str, np.ndarray]
    stats: dict[str, Any]
    runtime_s: float = 0.0
    dtype32: bool = False

    def rows(self, k: int) -> slice:
        return slice(int(self.offsets[k]), int(self.offsets[k + 1]))

    def result(self, k: int) -> BatchResult:
        sl = self.rows(k)
        a = self.arrays
        Y = a["Y"][sl]
        ev = a.get("event_Y")
        return BatchResult(
            Y=Y.astype(np.float32) if self.dtype32 else Y, state=a["state"][sl], n_steps=a["n_steps"][sl],
            lam=a["lam"][sl], max_null_error=a["max_null_error"][sl], max_energy_drift=a["max_energy_drift"][sl],
            max_lz_drift=a["max_lz_drift"][sl], max_carter_drift=a["max_carter_drift"][sl], runtime_s=self.runtime_s,
            event_Y=None if ev is None else (ev[sl].astype(np.float32) if self.dtype32 else ev[sl]),
            event_hit=None if a.get("event_hit") is None else a["event_hit"][sl].astype(bool),
            n_rejected=a["n_rejected"][sl],
        )

    def state_image(self, k: int) -> np.ndarray:
        if not self.specs[k].whole:
            raise ValueError(f"entry {k} is a pixel range, not a whole image")
        return self.arrays["state"][self.rows(k)].reshape(self.specs[k].camera.shape)

    def shadow_image(self, k: int):
        """Image ``k`` as a :class:`~kerrray_b200.shadow.ShadowImage` (``.save(path)`` writes the
        reference's ``.npz``, format version 1; ``shadow.py:119-176``)."""
        from kerrray_b200.shadow import ShadowImage

        spec = self.specs[k]
        if not spec.whole:
            raise ValueError(f"entry {k} is a pixel range, not a whole image")
        return ShadowImage.from_result(spec.spacetime, spec.camera, self.result(k))

    def captured(self, k: int) -> np.ndarray:
        return self.state_image(k) == int(TerminationState.CAPTURED)


def _host_arrays(total: int, disk: bool) -> dict[str, np.ndarray | None]:
    return {
        "Y": np.empty((total, 8), np.float64), "state": np.empty(total, np.int64), "n_steps": np.empty(total, np.int64),
        "n_rejected": np.empty(total, np.int64), "lam": np.empty(total, np.float64),
        "max_null_error": np.empty(total, np.float64), "max_energy_drift": np.empty(total, np.float64),
        "max_lz_drift": np.empty(total, np.float64), "max_carter_drift": np.empty(total, np.float64),
        "event_Y": np.zeros((total, 8), np.float64) if disk else None,
        "event_hit": np.zeros(total, np.uint8) if disk else None,
    }


def trace_images(specs: Sequence[ImageSpec], *, precision: str = "fast64", launch: LaunchConfig | None = None,
                 device: int = 0, Y0: np.ndarray | None = None, out: dict[str, np.ndarray] | None = None) -> SweepResult:
    """Trace every pixel of every image in one persistent launch; results in host arrays.

    ``Y0`` (optional, ``(total, 8)``) replaces the cameras as the photon source (rows in image
    order). ``out`` (optional) supplies preallocated host arrays (e.g. pinned memory).
    """
    import time

    t0 = time.perf_counter()
    specs = list(specs)
    images, offsets = _images(specs)
    total = int(offsets[-1])
    disk = any(bool(getattr(s.events, "disk_plane", False)) for s in specs if s.events is not None)
    arrays = out if out is not None else _host_arrays(total, disk)
    y0 = None
    if Y0 is not None:
        y0 = np.ascontiguousarray(np.asarray(Y0, dtype=np.float64))
        if y0.shape != (total, 8):
            raise ValueError(f"Y0 must have shape ({total}, 8), got {y0.shape}")
    res = _lib.result_struct(arrays)
    stats = _lib.KrrStats()
    lc = _launch(precision, launch)
    rc = _lib.lib().krr_trace_images(device, images, len(specs), _lib.ptr(y0), ctypes.byref(lc), ctypes.byref(res),
                                     ctypes.byref(stats))
    _lib.check(rc)
    dtype32 = any(str(getattr(s.integ, "dtype", "float64")) == "float32" for s in specs)
    return SweepResult(specs=specs, offsets=offsets, arrays=arrays, stats=stats.as_dict(),
                       runtime_s=time.perf_counter() - t0, dtype32=dtype32)


class DeviceSweep:
    """A batched launch whose results stay in device memory (torch tensors on ``cuda:device``).

    Build once, then call :meth:`run` repeatedly on the current torch stream. With
    ``graph=True`` (default) the whole launch sequence is captured once as a CUDA graph
    (``krr_plan_create``) and each run replays it; ``run(stats=False)`` only enqueues. With
    ``graph=False`` each run goes through ``krr_trace_images_device`` and reports the trace
    kernel's CUDA-event time (``kernel_ms``).
    """

    def __init__(self, specs: Sequence[ImageSpec], *, precision: str = "fast64", launch: LaunchConfig | None = None,
                 device: int = 0, Y0=None, minimal: bool = False, graph: bool = True) -> None:
        import torch

        self.specs = list(specs)
        self.images, self.offsets = _images(self.specs)
        self.total = int(self.offsets[-1])
        self.device = device
        self.config = launch or LaunchConfig()
        self.launch = _launch(precision, self.config)
        dev = torch.device("cuda", device)
        n = self.total
        f64, i64 = torch.float64, torch.int64
        self.tensors = {"Y": torch.empty((n, 8), dtype=f64, device=dev), "state": torch.empty(n, dtype=i64, device=dev)}
        if not minimal:
            for name in ("n_steps", "n_rejected"):
                self.tensors[name] = torch.empty(n, dtype=i64, device=dev)
            for name in ("lam", "max_null_error", "max_energy_drift", "max_lz_drift", "max_carter_drift"):
                self.tensors[name] = torch.empty(n, dtype=f64, device=dev)
        self.Y0 = Y0
        ws = int(_lib.lib().krr_workspace_size(len(self.specs), n if self.config.retrace else 0))
        self.workspace = torch.zeros(max(ws, 256), dtype=torch.uint8, device=dev)
        self._res = _lib.result_struct(self.tensors, device=True)
        self.plan = None
        if graph:
            handle = ctypes.c_void_p()
            y0 = None if self.Y0 is None else self.Y0.data_ptr()
            _lib.check(_lib.lib().krr_plan_create(device, self.images, len(self.specs), y0, ctypes.byref(self.launch),
                                                  ctypes.byref(self._res), self.workspace.data_ptr(),
                                                  self.workspace.numel(), ctypes.byref(handle)))
            self.plan = handle

    def run(self, stats: bool = True) -> dict[str, Any] | None:
        import torch

        stream = torch.cuda.current_stream(self.device).cuda_stream
        st = _lib.KrrStats()
        if self.plan is not None:
            _lib.check(_lib.lib().krr_plan_launch(self.plan, stream))
            if not stats:
                return None
            _lib.check(_lib.lib().krr_plan_stats(self.plan, stream, ctypes.byref(st)))
            return st.as_dict()
        y0 = None if self.Y0 is None else self.Y0.data_ptr()
        rc = _lib.lib().krr_trace_images_device(self.device, self.images, len(self.specs), y0, ctypes.byref(self.launch),
                                                ctypes.byref(self._res), self.workspace.data_ptr(),
                                                self.workspace.numel(), stream, ctypes.byref(st))
        _lib.check(rc)
        return st.as_dict()

    def stats(self) -> dict[str, Any]:
        """Counters of the last graph launch (synchronises the current stream)."""
        import torch

        if self.plan is None:
            raise RuntimeError("stats() reads a captured plan; build the sweep with graph=True")
        st = _lib.KrrStats()
        _lib.check(_lib.lib().krr_plan_stats(self.plan, torch.cuda.current_stream(self.device).cuda_stream,
                                             ctypes.byref(st)))
        return st.as_dict()

    def result(self, k: int) -> BatchResult:
        """Image ``k``'s rows of the device results, copied to host arrays."""
        names = ("n_steps", "n_rejected", "lam", "max_null_error", "max_energy_drift", "max_lz_drift",
                 "max_carter_drift")
        if any(n not in self.tensors for n in names):
            raise ValueError("a minimal sweep keeps only Y and state; build it with minimal=False")
        lo, hi = int(self.offsets[k]), int(self.offsets[k + 1])
        host = {n: t[lo:hi].cpu().numpy() for n, t in self.tensors.items()}
        return BatchResult(Y=host["Y"], state=host["state"], n_steps=host["n_steps"], n_rejected=host["n_rejected"],
                           lam=host["lam"], max_null_error=host["max_null_error"],
                           max_energy_drift=host["max_energy_drift"], max_lz_drift=host["max_lz_drift"],
                           max_carter_drift=host["max_carter_drift"], runtime_s=0.0)

    def shadow_image(self, k: int):
        """Image ``k`` from the device buffers as a :class:`~kerrray_b200.shadow.ShadowImage`
        (``.save(path)`` writes the reference's ``.npz``, format version 1)."""
        from kerrray_b200.shadow import ShadowImage

        spec = self.specs[k]
        if not spec.whole:
            raise ValueError(f"entry {k} is a pixel range, not a whole image")
        return ShadowImage.from_result(spec.spacetime, spec.camera, self.result(k))

    def close(self) -> None:
        if self.plan is not None:
            _lib.lib().krr_plan_destroy(self.plan)
            self.plan = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
