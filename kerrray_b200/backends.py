"""The ``cuda`` backend and the backend registry.

:class:`CudaBackend` implements KerrRay's ``Backend`` protocol
(``src/kerrray/raytracing/backends/base.py:53-68``): ``name`` and
``integrate_batch(st, Y0, integ, term, events=None) -> BatchResult``, plus the optional
``warm_up`` of ``raytracing/backends/numba_backend.py:239-253``. Input checks and their
exceptions follow ``numba_backend.py:78-84, 157-158``: ``Y0`` must be finite with shape
``(N, 8)`` (``ValueError``), ``"dop853"`` raises ``ValueError``, ``dtype="float32"`` returns
``Y`` in float32 with float64 ``lam`` and maxima. The integration itself runs on the GPU
through ``krr_integrate_batch`` of ``libkerrray_cuda.so``; nothing is computed on the CPU.

:func:`get_backend` / :func:`available_backends` mirror ``base.py:85-111`` with the ``cuda``
slot filled. ``"numpy"`` and ``"numba"`` are KerrRay's own CPU backends: they are returned
from an importable ``kerrray`` package and are otherwise unavailable here.
:func:`register_with_kerrray` makes KerrRay's own registry hand out this backend for
``"cuda"`` (``raytrace.backend: cuda`` in a KerrRay config then reaches the GPU).
"""

from __future__ import annotations

import ctypes
import sys
import threading
import time
from typing import Any, Final, Protocol, runtime_checkable

import numpy as np
from numpy.typing import ArrayLike

from kerrray_b200 import _lib
from kerrray_b200._lib import BackendUnavailable
from kerrray_b200.types import STATE_SIZE, BatchResult

__all__ = [
    "BACKEND_NAMES",
    "Backend",
    "BackendUnavailable",
    "CudaBackend",
    "available_backends",
    "get_backend",
    "register_with_kerrray",
]

BACKEND_NAMES: Final[tuple[str, ...]] = ("numpy", "numba", "cuda")


@runtime_checkable
class Backend(Protocol):
    """A batched integrator with the interface of KerrRay's ``integrate_batch``."""

    name: str

    def integrate_batch(self, st: Any, Y0: ArrayLike, integ: Any, term: Any, events: Any = None) -> BatchResult:
        ...


def _validate_batch(Y0: ArrayLike) -> np.ndarray:
    arr = np.array(Y0, dtype=np.float64)
    if arr.ndim != 2 or arr.shape[1] != STATE_SIZE:
        raise ValueError(f"Y0 must have shape (N, {STATE_SIZE}), got {arr.shape}")
    if not np.all(np.isfinite(arr)):
        raise ValueError("Y0 must be finite")
    return np.ascontiguousarray(arr)


def _result_type():
    """KerrRay's ``BatchResult`` when KerrRay is loaded in this process, else this package's."""
    mod = sys.modules.get("kerrray.photons")
    return getattr(mod, "BatchResult", BatchResult) if mod is not None else BatchResult


class CudaBackend:
    """The ``cuda`` backend: KerrRay's per-ray hot path on one B200 (sm_100a).

    Args:
        device: CUDA device ordinal.
        precision: ``"reference"`` (default; the reference's operation order in FP64, or its
            float32 mode when ``integ.dtype == "float32"``), ``"fast64"`` (FP64 with FMA,
            sincos and Newton reciprocals good to 2^-40 relative; for rtol below about 1e-11
            use ``"reference"``) or ``"mixed"`` (FP32 stages with FP64 accumulation, Delta and
            error norm; rk45 only). In the mixed precision the four conservation maxima of the
            result (``max_null_error`` and the E, L_z and Q drifts) are evaluated in FP32 from
            the FP32 copy of each accepted state: they bound that copy's round-off (about 1e-7
            relative), not the drift of the FP64 integration, which ``"fast64"`` and
            ``"reference"`` report.

    Raises:
        BackendUnavailable: When the library, the driver or the device is missing.
    """

    name: Final[str] = "cuda"

    def __init__(self, *, device: int = 0, precision: str = "reference") -> None:
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_lib.PRECISIONS)}, got {precision!r}")
        _lib.lib()
        n = _lib.device_count()
        if n < 1:
            raise BackendUnavailable(f"backend 'cuda' is unavailable: no CUDA device ({_lib.last_error()})")
        if not 0 <= device < n:
            raise ValueError(f"device {device} out of range [0, {n})")
        self.device = int(device)
        self.precision = precision

    def integrate_batch(self, st: Any, Y0: ArrayLike, integ: Any, term: Any, events: Any = None) -> BatchResult:
        """Integrate the states ``Y0`` (N, 8) on the GPU and return a ``BatchResult``."""
        t0 = time.perf_counter()
        opts = _lib.options_struct(integ, term, events)
        y0 = _validate_batch(Y0)
        n = y0.shape[0]
        disk = bool(opts.disk_plane)
        out = {
            "Y": np.empty((n, 8), np.float64), "state": np.empty(n, np.int64), "n_steps": np.empty(n, np.int64),
            "n_rejected": np.empty(n, np.int64), "lam": np.empty(n, np.float64),
            "max_null_error": np.empty(n, np.float64), "max_energy_drift": np.empty(n, np.float64),
            "max_lz_drift": np.empty(n, np.float64), "max_carter_drift": np.empty(n, np.float64),
            "event_Y": np.zeros((n, 8), np.float64) if disk else None,
            "event_hit": np.zeros(n, np.uint8) if disk else None,
        }
        res = _lib.result_struct(out)
        rc = _lib.lib().krr_integrate_batch(self.device, float(st.mass), float(st.spin), _lib.ptr(y0), n,
                                            ctypes.byref(opts), _lib.PRECISIONS[self.precision], ctypes.byref(res),
                                            None)
        _lib.check(rc)
        f32 = opts.dtype == 1
        Y = out["Y"].astype(np.float32) if f32 else out["Y"]
        return _result_type()(
            Y=Y, state=out["state"], n_steps=out["n_steps"], lam=out["lam"],
            max_null_error=out["max_null_error"], max_energy_drift=out["max_energy_drift"],
            max_lz_drift=out["max_lz_drift"], max_carter_drift=out["max_carter_drift"],
            runtime_s=time.perf_counter() - t0,
            event_Y=(out["event_Y"].astype(np.float32) if f32 else out["event_Y"]) if disk else None,
            event_hit=out["event_hit"].astype(bool) if disk else None,
            n_rejected=out["n_rejected"],
        )

    def warm_up(self, st: Any, integ: Any, term: Any) -> float:
        """Load the kernels (one short ray, ``lambda_max = step_size``); return the seconds it took."""
        from kerrray_b200.types import IntegratorOptions

        y0 = np.array([[0.0, 50.0, 0.5 * np.pi, 0.0, -1.0, -1.0, 0.0, 0.0]], dtype=np.float64)
        short = IntegratorOptions(method=integ.method, rtol=integ.rtol, atol=integ.atol, step_size=integ.step_size,
                                  max_steps=integ.max_steps, lambda_max=integ.step_size, h_min=integ.h_min,
                                  dtype=integ.dtype)
        t0 = time.perf_counter()
        self.integrate_batch(st, y0, short, term)
        return time.perf_counter() - t0

    def __repr__(self) -> str:
        return f"CudaBackend(device={self.device}, precision={self.precision!r})"


def _kerrray_backend(name: str):
    try:
        from kerrray.raytracing.backends import base  # type: ignore[import-not-found]
    except ImportError as exc:
        raise BackendUnavailable(f"backend {name!r} is unavailable: KerrRay is not importable ({exc})") from exc
    return _ORIGINAL.get("get_backend", base.get_backend)(name)


def get_backend(name: str):
    """Return the backend called ``name``; ``"cuda"`` is :class:`CudaBackend`.

    Raises:
        BackendUnavailable: When the named backend cannot be used here.
        ValueError: For a name outside :data:`BACKEND_NAMES`.
    """
    if name == "cuda":
        try:
            return CudaBackend()
        except BackendUnavailable:
            raise
        except (OSError, RuntimeError) as exc:
            raise BackendUnavailable(f"backend 'cuda' is unavailable: {exc}") from exc
    if name in ("numpy", "numba"):
        return _kerrray_backend(name)
    raise ValueError(f"unknown backend {name!r}; expected one of {sorted(BACKEND_NAMES)}")


def available_backends() -> dict[str, bool]:
    """``{"numpy": ..., "numba": ..., "cuda": ...}``: whether each backend can be used here."""
    out = {}
    for name in BACKEND_NAMES:
        try:
            get_backend(name)
            out[name] = True
        except BackendUnavailable:
            out[name] = False
    return out


_ORIGINAL: dict[str, Any] = {}
_REG_LOCK = threading.Lock()


def register_with_kerrray() -> bool:
    """Make KerrRay's registry return :class:`CudaBackend` for ``"cuda"``.

    Wraps ``kerrray.raytracing.backends.base.get_backend`` and ``available_backends`` and
    rebinds every module-level reference to them in the loaded ``kerrray`` modules (the tracer,
    shadow and command modules import the name directly). KerrRay's files are not edited.
    Returns False when KerrRay is not importable.
    """
    try:
        from kerrray.raytracing.backends import base  # type: ignore[import-not-found]
    except ImportError:
        return False
    with _REG_LOCK:
        if "get_backend" in _ORIGINAL:
            return True
        orig_get, orig_avail = base.get_backend, base.available_backends
        _ORIGINAL["get_backend"] = orig_get
        _ORIGINAL["available_backends"] = orig_avail

        def get_backend_with_cuda(name: str):
            if name == "cuda":
                try:
                    return CudaBackend()
                except BackendUnavailable as exc:
                    raise base.BackendUnavailable(str(exc)) from exc
            return orig_get(name)

        def available_with_cuda() -> dict[str, bool]:
            out = dict(orig_avail())
            try:
                CudaBackend()
                out["cuda"] = True
            except BackendUnavailable:
                out["cuda"] = False
            return out

        for mod_name, mod in list(sys.modules.items()):
            if mod is None or not mod_name.startswith("kerrray"):
                continue
            if getattr(mod, "get_backend", None) is orig_get:
                mod.get_backend = get_backend_with_cuda
            if getattr(mod, "available_backends", None) is orig_avail:
                mod.available_backends = available_with_cuda
    return True
