"""Observer camera: pixel grid on the host, backward null initial states on the GPU.

:class:`Camera` mirrors ``src/kerrray/raytracing/camera.py:99-222`` (fields, validation, the
inclination clamp into ``[1e-3, 180 - 1e-3]`` degrees, the pixel-centre formula
``alpha_j = fov (2j + 1 - n) / n``, ``beta_i = -fov (2i + 1 - n) / n``).
:func:`initial_states` (``camera.py:298-381``) runs the per-pixel tetrad projection and
the null re-normalisation of ``p_t`` in the device kernel ``k_camera_states`` through
``krr_camera_states``; :func:`initial_states_at` does the same for arbitrary image points
(the ``PointCamera`` of ``scripts/study_edge_bisection.py:39-50``).
"""

from __future__ import annotations

import ctypes
import logging
import math
from dataclasses import dataclass

import numpy as np

from kerrray_b200 import _lib

__all__ = ["INCLINATION_EPSILON_DEG", "NULL_CHECK_TOLERANCE", "Camera", "initial_states", "initial_states_at"]

logger = logging.getLogger("kerrray_b200.camera")

INCLINATION_EPSILON_DEG = 1e-3
NULL_CHECK_TOLERANCE = 1e-10


@dataclass(frozen=True)
class Camera:
    """Pinhole camera of a ZAMO at ``(radius, inclination_deg, phi_deg)`` with a square image."""

    radius: float
    inclination_deg: float
    phi_deg: float = 0.0
    fov: float = 12.0
    resolution: int = 64

    def __post_init__(self) -> None:
        radius, inclination, phi, fov = float(self.radius), float(self.inclination_deg), float(self.phi_deg), float(self.fov)
        if not (math.isfinite(radius) and radius > 0.0):
            raise ValueError(f"radius must be a finite number > 0, got {self.radius!r}")
        if not (math.isfinite(inclination) and 0.0 <= inclination <= 180.0):
            raise ValueError(f"inclination_deg must lie in [0, 180], got {self.inclination_deg!r}")
        if not math.isfinite(phi):
            raise ValueError(f"phi_deg must be finite, got {self.phi_deg!r}")
        if not (math.isfinite(fov) and fov > 0.0):
            raise ValueError(f"fov must be a finite number > 0, got {self.fov!r}")
        resolution = self.resolution
        if isinstance(resolution, bool) or not isinstance(resolution, (int, np.integer)):
            raise ValueError(f"resolution must be an integer, got {resolution!r}")
        resolution = int(resolution)
        if resolution < 2 or resolution % 2 != 0:
            raise ValueError(f"resolution must be an even integer >= 2, got {resolution!r}")
        low, high = INCLINATION_EPSILON_DEG, 180.0 - INCLINATION_EPSILON_DEG
        clamped = min(max(inclination, low), high)
        if clamped != inclination:
            logger.warning("Camera inclination_deg = %g lies on the spin axis where the ZAMO tetrad is singular; "
                           "clamped to %g deg", inclination, clamped)
        object.__setattr__(self, "radius", radius)
        object.__setattr__(self, "inclination_deg", clamped)
        object.__setattr__(self, "phi_deg", phi)
        object.__setattr__(self, "fov", fov)
        object.__setattr__(self, "resolution", resolution)

    @property
    def n_rays(self) -> int:
        return self.resolution * self.resolution

    @property
    def shape(self) -> tuple[int, int]:
        return (self.resolution, self.resolution)

    @property
    def pixel_size(self) -> float:
        return 2.0 * self.fov / self.resolution

    @property
    def inclination_rad(self) -> float:
        return math.radians(self.inclination_deg)

    @property
    def phi_rad(self) -> float:
        return math.radians(self.phi_deg)

    def pixel_coordinates(self) -> tuple[np.ndarray, np.ndarray]:
        """Pixel-centre ``(alpha, beta)``, shape ``(H, W)``; row 0 on top (``beta > 0``)."""
        n = self.resolution
        centres = self.fov * (2.0 * np.arange(n, dtype=np.float64) + 1.0 - n) / n
        return np.meshgrid(centres, -centres)

    def as_struct(self) -> _lib.KrrCamera:
        return _lib.KrrCamera(radius=self.radius, inclination_deg=self.inclination_deg, phi_deg=self.phi_deg,
                              fov=self.fov, resolution=self.resolution)


def _ergosphere_warning(st, radius: float, inclination_deg: float) -> None:
    m, a = st.mass, st.a
    r_ergo = m + math.sqrt(m * m - a * a * math.cos(math.radians(inclination_deg)) ** 2)
    if radius <= r_ergo:
        logger.warning("camera radius %g lies inside the ergosphere (r_E(theta_o) = %g): E = -p_t may have either "
                       "sign for the physical photon", radius, r_ergo)


def initial_states(cam: Camera, st, *, reverse: bool = True, device: int = 0) -> np.ndarray:
    """Null photon states for every pixel, shape ``(N, 8)``, row-major over ``(H, W)``.

    ``reverse=True`` (what the tracer integrates) gives backward rays with ``E = -p_t < 0``;
    ``reverse=False`` the physical photon (all four momenta negated, which is exact).

    Raises:
        ValueError: Camera inside the horizon, or ``fov`` too large for ``radius``.
        RuntimeError: The tetrad projection is not null to 1e-10.
    """
    _ergosphere_warning(st, cam.radius, cam.inclination_deg)
    y = np.empty((cam.n_rays, 8), dtype=np.float64)
    cs = cam.as_struct()
    rc = _lib.lib().krr_camera_states(device, float(st.mass), float(st.spin), ctypes.byref(cs), None, None, 0,
                                      y.ctypes.data)
    _lib.check(rc)
    if not reverse:
        y[:, 4:8] = -y[:, 4:8]
    return y


def initial_states_at(st, radius: float, inclination_deg: float, alpha, beta, *, phi_deg: float = 0.0,
                      device: int = 0) -> np.ndarray:
    """Backward null states for arbitrary image points ``(alpha, beta)`` (1-D, same length)."""
    a = np.ascontiguousarray(np.asarray(alpha, dtype=np.float64).ravel())
    b = np.ascontiguousarray(np.asarray(beta, dtype=np.float64).ravel())
    if a.shape != b.shape:
        raise ValueError("alpha and beta must have the same length")
    fov = float(max(np.max(np.abs(a)), np.max(np.abs(b)))) if a.size else 1.0
    cs = _lib.KrrCamera(radius=float(radius), inclination_deg=float(inclination_deg), phi_deg=float(phi_deg),
                        fov=fov if fov > 0 else 1.0, resolution=2)
    y = np.empty((a.size, 8), dtype=np.float64)
    rc = _lib.lib().krr_camera_states(device, float(st.mass), float(st.spin), ctypes.byref(cs), a.ctypes.data,
                                      b.ctypes.data, a.size, y.ctypes.data)
    _lib.check(rc)
    return y
