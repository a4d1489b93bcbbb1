"""ctypes binding of ``libkerrray_cuda.so`` (the C ABI of ``include/kerrray_cuda.h``).

The library is loaded from the package directory; a missing library or a missing CUDA device
raises :class:`BackendUnavailable` (the reference's exception for an unusable backend,
``src/kerrray/raytracing/backends/base.py:49``). There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import math
import threading
from pathlib import Path
from typing import Any

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libkerrray_cuda.so"

KRR_OK, KRR_ERR_INVALID, KRR_ERR_NO_DEVICE, KRR_ERR_CUDA, KRR_ERR_TIMEOUT, KRR_ERR_UNSUPPORTED, KRR_ERR_NOT_NULL = range(7)
PRECISIONS = {"reference": 0, "fast64": 1, "mixed": 2}

# Every symbol the header declares (checked by the CPU test suite).
EXPORTS = (
    "krr_last_error", "krr_abi_version", "krr_device_count", "krr_max_attempts", "krr_integrate_batch",
    "krr_integrate_batch_device", "krr_camera_states", "krr_trace_images", "krr_workspace_size",
    "krr_trace_images_device", "krr_fma_peak", "krr_list_variants", "krr_trace_images_noalloc",
    "krr_plan_create", "krr_plan_launch", "krr_plan_stats", "krr_plan_destroy", "krr_bisect_edges",
    "krr_lensing_workspace_size", "krr_lensing_workspace_size_staged", "krr_lensing_adjoint",
    "krr_lensing_tape_usage", "krr_lensing_replay", "krr_analytic_classes",
    "krr_escape_directions", "krr_trig_eval", "krr_disk_shading",
)


class BackendUnavailable(RuntimeError):
    """Raised when the ``cuda`` backend cannot be used here (no library, driver or device)."""


class KrrOptions(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int32), ("dtype", ctypes.c_int32),
        ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("step_size", ctypes.c_double),
        ("lambda_max", ctypes.c_double), ("h_min", ctypes.c_double), ("h_max", ctypes.c_double),
        ("max_steps", ctypes.c_int64),
        ("horizon_epsilon", ctypes.c_double), ("escape_radius", ctypes.c_double),
        ("disk_plane", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("r_in", ctypes.c_double), ("r_out", ctypes.c_double),
    ]


class KrrResult(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in (
        "Y", "state", "n_steps", "n_rejected", "lam", "max_null_error", "max_energy_drift", "max_lz_drift",
        "max_carter_drift", "event_Y", "event_hit")]


class KrrCamera(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_double), ("inclination_deg", ctypes.c_double), ("phi_deg", ctypes.c_double),
                ("fov", ctypes.c_double), ("resolution", ctypes.c_int64)]


class KrrImage(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("spin", ctypes.c_double), ("camera", KrrCamera), ("options", KrrOptions),
                ("first_pixel", ctypes.c_int64), ("pixel_count", ctypes.c_int64)]


class KrrEdgeCase(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("spin", ctypes.c_double), ("radius", ctypes.c_double),
                ("inclination_deg", ctypes.c_double), ("phi_deg", ctypes.c_double), ("options", KrrOptions),
                ("centre_alpha", ctypes.c_double), ("centre_beta", ctypes.c_double)]


class KrrLaunch(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("block", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("refill_threshold", ctypes.c_int32), ("plain", ctypes.c_int32), ("variant", ctypes.c_int32),
                ("retrace", ctypes.c_int32), ("critical_sms", ctypes.c_int32)]


class KrrVariantInfo(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("min_blocks", ctypes.c_int32), ("registers", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32)]


class KrrStats(ctypes.Structure):
    _fields_ = [("photons", ctypes.c_uint64), ("retired", ctypes.c_uint64), ("attempts", ctypes.c_uint64),
                ("accepted", ctypes.c_uint64), ("lane_slots", ctypes.c_uint64), ("busy_slots", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("retraced", ctypes.c_uint64), ("retrace_attempts", ctypes.c_uint64),
                ("retrace_ms", ctypes.c_double), ("critical", ctypes.c_uint64), ("rechecked", ctypes.c_uint64),
                ("critical_ms", ctypes.c_double), ("speculative", ctypes.c_uint64),
                ("discarded_attempts", ctypes.c_uint64), ("near_edge", ctypes.c_uint64),
                ("near_edge_attempts", ctypes.c_uint64)]

    def as_dict(self) -> dict[str, Any]:
        return {name: getattr(self, name) for name, _ in self._fields_}


_LOCK = threading.Lock()
_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load the library once (raises BackendUnavailable when it is missing)."""
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not LIB_PATH.exists():
            raise BackendUnavailable(
                f"backend 'cuda' is unavailable: {LIB_PATH.name} is not built (run python -m kerrray_b200.build)")
        try:
            L = ctypes.CDLL(str(LIB_PATH))
        except OSError as exc:
            raise BackendUnavailable(f"backend 'cuda' is unavailable: cannot load {LIB_PATH.name}: {exc}") from exc
        vp, i32, i64, dp = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        L.krr_last_error.restype = ctypes.c_char_p
        L.krr_last_error.argtypes = []
        L.krr_abi_version.restype = ctypes.c_int
        L.krr_device_count.restype = ctypes.c_int
        L.krr_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.krr_max_attempts.restype = ctypes.c_int
        L.krr_max_attempts.argtypes = [ctypes.POINTER(KrrOptions), ctypes.POINTER(ctypes.c_int64)]
        L.krr_integrate_batch.restype = ctypes.c_int
        L.krr_integrate_batch.argtypes = [ctypes.c_int, dp, dp, vp, i64, ctypes.POINTER(KrrOptions), i32,
                                          ctypes.POINTER(KrrResult), ctypes.POINTER(ctypes.c_double)]
        L.krr_integrate_batch_device.restype = ctypes.c_int
        L.krr_integrate_batch_device.argtypes = [ctypes.c_int, dp, dp, vp, vp, i64, ctypes.POINTER(KrrOptions), i32,
                                                 ctypes.POINTER(KrrResult), vp]
        L.krr_camera_states.restype = ctypes.c_int
        L.krr_camera_states.argtypes = [ctypes.c_int, dp, dp, ctypes.POINTER(KrrCamera), vp, vp, i64, vp]
        L.krr_trace_images.restype = ctypes.c_int
        L.krr_trace_images.argtypes = [ctypes.c_int, ctypes.POINTER(KrrImage), i32, vp, ctypes.POINTER(KrrLaunch),
                                       ctypes.POINTER(KrrResult), ctypes.POINTER(KrrStats)]
        L.krr_workspace_size.restype = ctypes.c_size_t
        L.krr_workspace_size.argtypes = [i32, i64]
        L.krr_analytic_classes.restype = ctypes.c_int
        L.krr_analytic_classes.argtypes = [dp, dp, dp, dp, vp, i64, vp]
        L.krr_disk_shading.restype = ctypes.c_int
        L.krr_disk_shading.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int32, dp, dp, dp, ctypes.c_int32, vp, vp, i64,
                                       vp, vp, vp, vp]
        L.krr_trig_eval.restype = ctypes.c_int
        L.krr_trig_eval.argtypes = [ctypes.c_int, ctypes.c_int32, vp, vp, i64, vp, vp, vp]
        L.krr_escape_directions.restype = ctypes.c_int
        L.krr_escape_directions.argtypes = [ctypes.c_int, dp, dp, dp, vp, vp, i64, vp, vp, vp]
        L.krr_trace_images_device.restype = ctypes.c_int
        L.krr_trace_images_device.argtypes = [ctypes.c_int, ctypes.POINTER(KrrImage), i32, vp,
                                              ctypes.POINTER(KrrLaunch), ctypes.POINTER(KrrResult), vp,
                                              ctypes.c_size_t, vp, ctypes.POINTER(KrrStats)]
        L.krr_bisect_edges.restype = ctypes.c_int
        L.krr_bisect_edges.argtypes = [ctypes.c_int, ctypes.POINTER(KrrEdgeCase), i32, vp, vp, vp, vp, vp, vp, i64, i32,
                                       i32, ctypes.POINTER(KrrStats)]
        L.krr_plan_create.restype = ctypes.c_int
        L.krr_plan_create.argtypes = [ctypes.c_int, ctypes.POINTER(KrrImage), i32, vp, ctypes.POINTER(KrrLaunch),
                                      ctypes.POINTER(KrrResult), vp, ctypes.c_size_t, ctypes.POINTER(vp)]
        L.krr_plan_launch.restype = ctypes.c_int
        L.krr_plan_launch.argtypes = [vp, vp]
        L.krr_plan_stats.restype = ctypes.c_int
        L.krr_plan_stats.argtypes = [vp, vp, ctypes.POINTER(KrrStats)]
        L.krr_plan_destroy.restype = ctypes.c_int
        L.krr_plan_destroy.argtypes = [vp]
        L.krr_trace_images_noalloc.restype = ctypes.c_int
        L.krr_trace_images_noalloc.argtypes = [ctypes.c_int, ctypes.POINTER(KrrImage), i32, vp,
                                               ctypes.POINTER(KrrLaunch), ctypes.POINTER(KrrResult), vp,
                                               ctypes.POINTER(KrrStats)]
        L.krr_list_variants.restype = ctypes.c_int
        L.krr_list_variants.argtypes = [ctypes.c_int, i32, ctypes.POINTER(KrrOptions), ctypes.POINTER(KrrVariantInfo),
                                        i32, ctypes.POINTER(ctypes.c_int32)]
        L.krr_fma_peak.restype = ctypes.c_int
        L.krr_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        _LIB = L
        return L


def last_error() -> str:
    msg = lib().krr_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    """Map a status code to the reference's exception types."""
    if rc == KRR_OK:
        return
    msg = last_error()
    if rc in (KRR_ERR_INVALID, KRR_ERR_UNSUPPORTED):
        raise ValueError(msg)
    if rc == KRR_ERR_NO_DEVICE:
        raise BackendUnavailable(f"backend 'cuda' is unavailable: {msg}")
    if rc == KRR_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


def fma_peak_tflops(device: int = 0, fp64: bool = True) -> float:
    """Measured FMA throughput of the device (TFLOP/s, 2 FLOP per FMA)."""
    out = ctypes.c_double(0.0)
    check(lib().krr_fma_peak(device, int(fp64), ctypes.byref(out)))
    return float(out.value)


def device_count() -> int:
    n = ctypes.c_int(0)
    rc = lib().krr_device_count(ctypes.byref(n))
    if rc != KRR_OK:
        return 0
    return int(n.value)


def options_struct(integ: Any, term: Any, events: Any = None) -> KrrOptions:
    """Pack reference-style option objects (duck-typed) into ``krr_options``."""
    method = getattr(integ, "method", "rk45")
    if method == "dop853":
        raise ValueError("method 'dop853' is available in integrate() only; the cuda backend supports 'rk4' and 'rk45'")
    if method not in ("rk45", "rk4"):
        raise ValueError(f"method must be 'rk4' or 'rk45', got {method!r}")
    dtype = str(getattr(integ, "dtype", "float64"))
    h_max = getattr(integ, "h_max", None)
    disk = events is not None and bool(getattr(events, "disk_plane", False))
    return KrrOptions(
        method=0 if method == "rk45" else 1, dtype=1 if dtype == "float32" else 0,
        rtol=float(integ.rtol), atol=float(integ.atol), step_size=float(integ.step_size),
        lambda_max=float(integ.lambda_max), h_min=float(integ.h_min),
        h_max=math.inf if h_max is None else float(h_max), max_steps=int(integ.max_steps),
        horizon_epsilon=float(term.horizon_epsilon), escape_radius=float(term.escape_radius),
        disk_plane=int(disk), reserved=0,
        r_in=float(getattr(events, "r_in", 6.0)) if disk else 0.0,
        r_out=float(getattr(events, "r_out", 20.0)) if disk else 0.0,
    )


def ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


def result_struct(arrays: dict[str, np.ndarray | None], device: bool = False) -> KrrResult:
    """A ``krr_result`` over numpy arrays (host) or torch tensors (device, ``data_ptr``)."""
    r = KrrResult()
    for name, _ in KrrResult._fields_:
        a = arrays.get(name)
        if a is None:
            setattr(r, name, None)
        else:
            setattr(r, name, a.data_ptr() if device else a.ctypes.data)
    return r
