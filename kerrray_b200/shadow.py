"""Shadow images: trace every pixel, classify, keep the state map and the captured mask.

Mirrors ``src/kerrray/raytracing/shadow.py:40-211``: :class:`ShadowImage` (fields, counts,
``n_failed``/``n_other``, the compressed ``.npz`` format version 1 with the same keys, so files
round-trip between the two implementations), :func:`state_counts`, :data:`FAILURE_STATES`
and :func:`compute_shadow`. With the ``cuda`` backend the camera, the integration and the
classification of the whole image run in one device launch (``krr_trace_images``); any other
backend object gets the GPU camera states through its ``integrate_batch``.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

from kerrray_b200.camera import Camera, initial_states
from kerrray_b200.rays import DEFAULT_CHUNK_SIZE, ProgressCallback, trace_rays
from kerrray_b200.types import BatchResult, Spacetime, TerminationState

__all__ = ["FAILURE_STATES", "NPZ_FORMAT_VERSION", "ShadowImage", "compute_shadow", "state_counts", "shadow_mask_int8"]

NPZ_FORMAT_VERSION = 1
FAILURE_STATES = (TerminationState.NUMERICAL_FAILURE, TerminationState.OUT_OF_DOMAIN)

_CAMERA_FIELDS = ("radius", "inclination_deg", "phi_deg", "fov", "resolution")
_RESULT_ARRAYS = ("Y", "state", "n_steps", "lam", "max_null_error", "max_energy_drift", "max_lz_drift",
                  "max_carter_drift")
_OPTIONAL_RESULT_ARRAYS = ("event_Y", "event_hit", "n_rejected")


def state_counts(state: NDArray[np.integer]) -> dict[str, int]:
    """Number of rays per ``TerminationState`` name (every member, zeros included)."""
    codes = np.asarray(state)
    return {m.name: int(np.count_nonzero(codes == int(m))) for m in TerminationState}


def shadow_mask_int8(state: NDArray[np.integer]) -> NDArray[np.int8]:
    """int8 mask: 1 captured, 0 escaped, -1 failed (NUMERICAL_FAILURE / OUT_OF_DOMAIN), 2 other."""
    s = np.asarray(state)
    out = np.full(s.shape, 2, dtype=np.int8)
    out[s == int(TerminationState.ESCAPED)] = 0
    out[s == int(TerminationState.CAPTURED)] = 1
    out[(s == int(TerminationState.NUMERICAL_FAILURE)) | (s == int(TerminationState.OUT_OF_DOMAIN))] = -1
    return out


@dataclass
class ShadowImage:
    """A traced image: pixel coordinates, termination map, captured mask and the batch result."""

    alpha: NDArray[np.float64]
    beta: NDArray[np.float64]
    state: NDArray[np.int64]
    captured: NDArray[np.bool_]
    counts: dict[str, int]
    result: Any
    camera: Camera
    spacetime: Any

    @property
    def shape(self) -> tuple[int, int]:
        return self.camera.shape

    @property
    def n_rays(self) -> int:
        return self.camera.n_rays

    @property
    def pixel_size(self) -> float:
        return self.camera.pixel_size

    def count(self, state: TerminationState) -> int:
        return self.counts[state.name]

    @property
    def n_failed(self) -> int:
        return sum(self.count(s) for s in FAILURE_STATES)

    @property
    def n_other(self) -> int:
        settled = self.count(TerminationState.CAPTURED) + self.count(TerminationState.ESCAPED)
        return self.n_rays - settled - self.n_failed

    def save(self, path: Path | str) -> Path:
        """Write the compressed ``.npz`` (format version 1, the reference's keys)."""
        target = Path(path)
        target.parent.mkdir(parents=True, exist_ok=True)
        payload: dict[str, Any] = {
            "format_version": np.int64(NPZ_FORMAT_VERSION), "alpha": self.alpha, "beta": self.beta,
            "image_state": self.state, "captured": self.captured, "mass": np.float64(self.spacetime.mass),
            "spin": np.float64(self.spacetime.spin), "runtime_s": np.float64(self.result.runtime_s),
        }
        for name in _CAMERA_FIELDS:
            payload[f"camera_{name}"] = np.asarray(getattr(self.camera, name))
        for name in _RESULT_ARRAYS:
            payload[f"result_{name}"] = np.asarray(getattr(self.result, name))
        for name in _OPTIONAL_RESULT_ARRAYS:
            value = getattr(self.result, name)
            if value is not None:
                payload[f"result_{name}"] = np.asarray(value)
        np.savez_compressed(target, **payload)
        return target

    @classmethod
    def load(cls, path: Path | str) -> "ShadowImage":
        with np.load(Path(path)) as data:
            version = int(data["format_version"])
            if version != NPZ_FORMAT_VERSION:
                raise ValueError(f"unsupported shadow file version {version} (expected {NPZ_FORMAT_VERSION})")
            camera = Camera(radius=float(data["camera_radius"]), inclination_deg=float(data["camera_inclination_deg"]),
                            phi_deg=float(data["camera_phi_deg"]), fov=float(data["camera_fov"]),
                            resolution=int(data["camera_resolution"]))
            spacetime = Spacetime(mass=float(data["mass"]), spin=float(data["spin"]))
            fields: dict[str, Any] = {name: data[f"result_{name}"] for name in _RESULT_ARRAYS}
            for name in _OPTIONAL_RESULT_ARRAYS:
                key = f"result_{name}"
                fields[name] = data[key] if key in data.files else None
            result = BatchResult(runtime_s=float(data["runtime_s"]), **fields)
            state = np.asarray(data["image_state"], dtype=np.int64)
            return cls(alpha=np.asarray(data["alpha"], dtype=np.float64), beta=np.asarray(data["beta"], dtype=np.float64),
                       state=state, captured=np.asarray(data["captured"], dtype=bool), counts=state_counts(state),
                       result=result, camera=camera, spacetime=spacetime)


def _image_from_result(st, cam: Camera, result) -> ShadowImage:
    alpha, beta = cam.pixel_coordinates()
    state = np.asarray(result.state, dtype=np.int64).reshape(cam.shape)
    return ShadowImage(alpha=alpha, beta=beta, state=state, captured=state == int(TerminationState.CAPTURED),
                       counts=state_counts(state), result=result, camera=cam, spacetime=st)


def compute_shadow(st, cam: Camera, integ, term, *, backend: Any = "cuda", progress: ProgressCallback | None = None,
                   chunk_size: int = DEFAULT_CHUNK_SIZE) -> ShadowImage:
    """Trace every pixel of ``cam`` backwards in ``st`` and classify it."""
    from kerrray_b200.backends import CudaBackend, get_backend
    from kerrray_b200.sweep import ImageSpec, trace_images

    engine = get_backend(backend) if isinstance(backend, str) else backend
    if isinstance(engine, CudaBackend):
        sweep = trace_images([ImageSpec(st, cam, integ, term)], precision=engine.precision, device=engine.device)
        if progress is not None:
            progress(1.0)
        return _image_from_result(st, cam, sweep.result(0))
    Y0 = initial_states(cam, st)
    result = trace_rays(st, Y0, integ, term, backend=engine, progress=progress, chunk_size=chunk_size)
    return _image_from_result(st, cam, result)
