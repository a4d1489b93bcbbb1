"""Shadow images: every pixel of a camera traced, classified and kept with its termination map.

:class:`ShadowImage` carries what KerrRay's ``compute_shadow`` returns (the attributes and
properties of ``raytracing/shadow.py:66-117``), so code written against the reference's class
reads this one. Its per-state counts come from one ``np.bincount`` of the codes.

On disk it is the reference's ``.npz`` format version 1 (``shadow.py:119-176``), so files move
between the two implementations in both directions: flat keys grouped by prefix --
``camera_<field>`` for the camera's five fields and ``result_<field>`` for every per-ray array
of the batch result (the optional ones only when present) -- beside ``format_version``,
``alpha``, ``beta``, ``image_state``, ``captured``, ``mass``, ``spin`` and ``runtime_s``.
Writing walks the result's dataclass fields; reading gathers each group by its prefix.

With the ``cuda`` backend, :func:`compute_shadow` runs the camera, the integration and the
classification of the whole image in one device launch (``krr_trace_images``); any other
backend object integrates the device-computed camera states through its ``integrate_batch``.
"""

from __future__ import annotations

import dataclasses
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
# Codes counted as a failed ray (an RK4 overshoot through the horizon is OUT_OF_DOMAIN, not CAPTURED).
FAILURE_STATES = (TerminationState.NUMERICAL_FAILURE, TerminationState.OUT_OF_DOMAIN)
_SETTLED = (TerminationState.CAPTURED, TerminationState.ESCAPED)
_CAMERA_KEYS = {"radius": float, "inclination_deg": float, "phi_deg": float, "fov": float, "resolution": int}


def state_counts(state: NDArray[np.integer]) -> dict[str, int]:
    """Rays per ``TerminationState`` name, every member listed (zeros included)."""
    codes = np.asarray(state, dtype=np.int64).ravel()
    members = len(TerminationState)
    tally = np.bincount(codes[(codes >= 0) & (codes < members)], minlength=members)
    return {member.name: int(tally[int(member)]) for member in TerminationState}


def shadow_mask_int8(state: NDArray[np.integer]) -> NDArray[np.int8]:
    """int8 mask: 1 captured, 0 escaped, -1 failed (NUMERICAL_FAILURE / OUT_OF_DOMAIN), 2 other."""
    lookup = np.full(len(TerminationState), 2, dtype=np.int8)
    lookup[int(TerminationState.ESCAPED)] = 0
    lookup[int(TerminationState.CAPTURED)] = 1
    lookup[[int(s) for s in FAILURE_STATES]] = -1
    codes = np.asarray(state, dtype=np.int64)
    return np.where((codes >= 0) & (codes < lookup.size), lookup[np.clip(codes, 0, lookup.size - 1)], 2).astype(np.int8)


@dataclass
class ShadowImage:
    """A traced image: pixel coordinates ``alpha``, ``beta`` (H x W, M), the termination code of
    each pixel (``state``), the shadow mask ``captured`` (state == CAPTURED), the pixels per
    state name (``counts``), the batch ``result`` (rays row-major), its ``camera`` and ``spacetime``."""

    alpha: NDArray[np.float64]
    beta: NDArray[np.float64]
    state: NDArray[np.int64]
    captured: NDArray[np.bool_]
    counts: dict[str, int]
    result: Any
    camera: Camera
    spacetime: Any

    @classmethod
    def from_result(cls, spacetime: Any, camera: Camera, result: Any) -> "ShadowImage":
        """The image of ``camera``'s pixels from a batch result in row-major pixel order."""
        alpha, beta = camera.pixel_coordinates()
        state = np.asarray(result.state, dtype=np.int64).reshape(camera.shape)
        return cls(alpha=alpha, beta=beta, state=state, captured=state == int(TerminationState.CAPTURED),
                   counts=state_counts(state), result=result, camera=camera, spacetime=spacetime)

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
        """Pixels whose ray ended in ``state``."""
        return self.counts[TerminationState(state).name]

    @property
    def n_failed(self) -> int:
        """Pixels whose ray failed (``FAILURE_STATES``)."""
        return sum(self.counts[s.name] for s in FAILURE_STATES)

    @property
    def n_other(self) -> int:
        """Pixels that ended neither CAPTURED nor ESCAPED and did not fail."""
        return self.n_rays - sum(self.counts[s.name] for s in _SETTLED + FAILURE_STATES)

    # -- the .npz file ----------------------------------------------------------------------
    def save(self, path: Path | str) -> Path:
        """Write the compressed ``.npz`` (format version 1); returns the path written."""
        target = Path(path)
        target.parent.mkdir(parents=True, exist_ok=True)
        record: dict[str, Any] = {
            "format_version": np.int64(NPZ_FORMAT_VERSION), "alpha": self.alpha, "beta": self.beta,
            "image_state": self.state, "captured": self.captured, "mass": np.float64(self.spacetime.mass),
            "spin": np.float64(self.spacetime.spin), "runtime_s": np.float64(self.result.runtime_s),
        }
        record.update({f"camera_{name}": np.asarray(getattr(self.camera, name)) for name in _CAMERA_KEYS})
        for f in dataclasses.fields(self.result):
            value = getattr(self.result, f.name)
            if f.name != "runtime_s" and value is not None:
                record[f"result_{f.name}"] = np.asarray(value)
        np.savez_compressed(target, **record)
        return target

    @classmethod
    def load(cls, path: Path | str) -> "ShadowImage":
        """Read a file written by :meth:`save` (or by the reference's ``ShadowImage.save``)."""
        with np.load(Path(path)) as archive:
            version = int(archive["format_version"])
            if version != NPZ_FORMAT_VERSION:
                raise ValueError(f"unsupported shadow file version {version} (expected {NPZ_FORMAT_VERSION})")
            groups: dict[str, dict[str, np.ndarray]] = {"camera": {}, "result": {}}
            for key in archive.files:
                prefix, _, name = key.partition("_")
                if prefix in groups and name:
                    groups[prefix][name] = archive[key]
            camera = Camera(**{name: cast(groups["camera"][name]) for name, cast in _CAMERA_KEYS.items()})
            spacetime = Spacetime(mass=float(archive["mass"]), spin=float(archive["spin"]))
            try:
                result = BatchResult(runtime_s=float(archive["runtime_s"]), **groups["result"])
            except TypeError as exc:
                raise ValueError(f"{path}: the batch result is incomplete ({exc})") from exc
            state = np.asarray(archive["image_state"], dtype=np.int64)
            return cls(alpha=np.asarray(archive["alpha"], dtype=np.float64),
                       beta=np.asarray(archive["beta"], dtype=np.float64), state=state,
                       captured=np.asarray(archive["captured"], dtype=bool), counts=state_counts(state),
                       result=result, camera=camera, spacetime=spacetime)


def compute_shadow(st, cam: Camera, integ, term, *, backend: Any = "cuda", progress: ProgressCallback | None = None,
                   chunk_size: int | None = DEFAULT_CHUNK_SIZE) -> ShadowImage:
    """Trace every pixel of ``cam`` backwards in ``st`` and classify it."""
    from kerrray_b200.backends import CudaBackend, get_backend
    from kerrray_b200.sweep import ImageSpec, trace_images

    engine = get_backend(backend) if isinstance(backend, str) else backend
    if isinstance(engine, CudaBackend):
        sweep = trace_images([ImageSpec(st, cam, integ, term)], precision=engine.precision, device=engine.device)
        if progress is not None:
            progress(1.0)
        return ShadowImage.from_result(st, cam, sweep.result(0))
    result = trace_rays(st, initial_states(cam, st), integ, term, backend=engine, progress=progress,
                        chunk_size=chunk_size)
    return ShadowImage.from_result(st, cam, result)
