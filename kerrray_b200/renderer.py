"""Accretion-disk renderer on the GPU (``raytracing/renderer.py:163-262``,
``physics/accretion.py:119-198``, ``physics/redshift.py:131`` of the reference).

:func:`render_disk` traces the camera's backward rays with the disk-plane event on the cuda
backend (``DISK_HIT`` where a ray crosses theta = pi/2 with r_in <= r <= r_out), then shades
the crossings on the device (``krr_disk_shading``): the redshift factor g = nu_obs / nu_em for
a circular equatorial Keplerian emitter, and I_obs = g^n (r / r_in)^-p with n = 3 (``"g3"``)
or 4 (``"g4"``). Other pixels get I_obs = 0 and g = r_hit = NaN. The arrays, their layout,
the errors and the ``.npz`` file are the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np

from kerrray_b200 import _lib
from kerrray_b200.camera import Camera, initial_states
from kerrray_b200.orbits import _mass_and_spin, equatorial_photon_orbit_radius
from kerrray_b200.types import BatchResult, EventOptions, TerminationState

__all__ = ["DiskModel", "DiskImage", "INTENSITY_LAWS", "isco_radius", "keplerian_angular_velocity", "event_options",
           "render_disk", "save_disk_image", "load_disk_image_arrays"]

INTENSITY_LAWS = {"g3": 3, "g4": 4}  # power of g multiplying the emitted intensity
STATE_SIZE = 8


def keplerian_angular_velocity(st: Any, r, prograde: bool = True):
    """Omega = +-sqrt(M) / (r^(3/2) +- |a| sqrt(M)) (Bardeen, Press and Teukolsky 1972, eq. 2.16),
    upper sign prograde (a L_z > 0), times sign(a) with sign(0) = +1 (``photons/orbits.py:281-292``)."""
    mass, a = _mass_and_spin(st)
    s = 1.0 if prograde else -1.0
    sa = -1.0 if a < 0.0 else 1.0
    r = np.asarray(r, dtype=np.float64)
    return s * sa * math.sqrt(mass) / (r ** 1.5 + s * abs(a) * math.sqrt(mass))


def isco_radius(st: Any, prograde: bool = True) -> float:
    """Innermost stable circular orbit (BPT 1972, eq. 2.21; ``photons/orbits.py:336-350``)."""
    mass, a = _mass_and_spin(st)
    s = 1.0 if prograde else -1.0
    chi = abs(a) / mass
    z1 = 1.0 + (1.0 - chi * chi) ** (1.0 / 3.0) * ((1.0 + chi) ** (1.0 / 3.0) + (1.0 - chi) ** (1.0 / 3.0))
    z2 = math.sqrt(3.0 * chi * chi + z1 * z1)
    return mass * (3.0 + z2 - s * math.sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2)))


@dataclass(frozen=True)
class DiskModel:
    """The thin equatorial disk (``physics/accretion.py:DiskModel``): r_in < r_out in units of M,
    emissivity (r / r_in)^-emissivity_index, intensity law ``"g3"`` or ``"g4"``, orbit sense."""

    r_in: float
    r_out: float
    emissivity_index: float = 3.0
    intensity_law: str = "g4"
    prograde: bool = True

    def __post_init__(self) -> None:
        for name in ("r_in", "r_out", "emissivity_index"):
            if not math.isfinite(getattr(self, name)):
                raise ValueError(f"{name} must be finite, got {getattr(self, name)!r}")
        if not (0.0 < self.r_in < self.r_out):
            raise ValueError(f"need 0 < r_in < r_out, got r_in={self.r_in!r}, r_out={self.r_out!r}")
        if self.intensity_law not in INTENSITY_LAWS:
            raise ValueError(f"intensity_law must be one of {sorted(INTENSITY_LAWS)}, got {self.intensity_law!r}")

    @property
    def redshift_power(self) -> int:
        return INTENSITY_LAWS[self.intensity_law]

    @classmethod
    def for_spacetime(cls, st: Any, *, r_in: float | None = None, r_out: float = 20.0, emissivity_index: float = 3.0,
                      intensity_law: str = "g4", prograde: bool = True) -> "DiskModel":
        """The disk for ``st`` (``DiskModel.from_params``): ``r_in=None`` is the ISCO of the orbit
        sense; r_in must exceed the circular photon orbit, below which no circular orbit exists."""
        r_in_v = isco_radius(st, prograde=prograde) if r_in is None else float(r_in)
        r_ph = equatorial_photon_orbit_radius(st, prograde=prograde)
        if not r_in_v > r_ph:
            raise ValueError(f"disk r_in = {r_in_v:.6g} must exceed the circular photon orbit radius r_ph = {r_ph:.6g} "
                             "(no circular gas orbit below it)")
        return cls(r_in=float(r_in_v), r_out=float(r_out), emissivity_index=float(emissivity_index),
                   intensity_law=intensity_law, prograde=bool(prograde))


def event_options(disk: DiskModel) -> EventOptions:
    """The disk-plane event of the batched integrator for this disk."""
    return EventOptions(disk_plane=True, r_in=disk.r_in, r_out=disk.r_out)


@dataclass
class DiskImage:
    """A rendered disk (``raytracing/renderer.py:DiskImage``): arrays in the camera's (H, W) layout."""

    intensity: np.ndarray
    g: np.ndarray
    hit: np.ndarray
    r_hit: np.ndarray
    state: np.ndarray
    alpha: np.ndarray
    beta: np.ndarray
    hit_states: np.ndarray
    result: BatchResult
    camera: Camera
    spacetime: Any
    disk: DiskModel
    backend: str

    @property
    def shape(self) -> tuple[int, int]:
        return self.camera.shape

    @property
    def n_hits(self) -> int:
        return int(np.count_nonzero(self.hit))

    def counts(self) -> dict[str, int]:
        out: dict[str, int] = {}
        for member in TerminationState:
            n = int(np.count_nonzero(self.state == int(member)))
            if n:
                out[member.name] = n
        return out


def render_disk(st: Any, cam: Camera, integ: Any, term: Any, disk: DiskModel, *, backend: Any = None,
                device: int = 0) -> DiskImage:
    """Render ``disk`` seen by ``cam`` in ``st`` (``raytracing/renderer.py:render_disk``): the
    camera rays traced with the disk-plane event on the cuda backend (``backend``: a
    :class:`~kerrray_b200.backends.CudaBackend`, the reference precision by default), the
    crossings shaded on the device."""
    import torch

    from kerrray_b200.backends import CudaBackend

    be = backend if backend is not None else CudaBackend(device=device)
    y0 = initial_states(cam, st, device=be.device)
    result = be.integrate_batch(st, y0, integ, term, events=event_options(disk))
    if result.event_hit is None or result.event_Y is None:
        raise RuntimeError("the backend did not evaluate the disk-plane event")
    n = cam.n_rays
    hit_flat = np.asarray(result.event_hit, dtype=bool)
    ev = torch.tensor(np.asarray(result.event_Y, dtype=np.float64), device=f"cuda:{be.device}")
    hit_dev = torch.tensor(hit_flat.astype(np.uint8), device=f"cuda:{be.device}")
    g_dev = torch.empty(n, dtype=torch.float64, device=ev.device)
    i_dev = torch.empty(n, dtype=torch.float64, device=ev.device)
    r_dev = torch.empty(n, dtype=torch.float64, device=ev.device)
    stream = torch.cuda.current_stream(ev.device).cuda_stream
    _lib.check(_lib.lib().krr_disk_shading(be.device, float(st.mass), float(st.spin), int(disk.prograde), disk.r_in,
                                           disk.r_out, disk.emissivity_index, disk.redshift_power, ev.data_ptr(),
                                           hit_dev.data_ptr(), n, g_dev.data_ptr(), i_dev.data_ptr(), r_dev.data_ptr(),
                                           stream))
    g_flat, i_flat, r_flat = g_dev.cpu().numpy(), i_dev.cpu().numpy(), r_dev.cpu().numpy()
    if np.any(np.isnan(g_flat[hit_flat])):
        raise ValueError("a disk crossing is not equatorial, lies below the circular photon orbit, or has a "
                         "non-positive frequency ratio")
    states_flat = np.full((n, STATE_SIZE), np.nan, dtype=np.float64)
    states_flat[hit_flat] = np.asarray(result.event_Y, dtype=np.float64)[hit_flat]
    shape = cam.shape
    alpha, beta = cam.pixel_coordinates()
    return DiskImage(intensity=i_flat.reshape(shape), g=g_flat.reshape(shape), hit=hit_flat.reshape(shape),
                     r_hit=r_flat.reshape(shape), state=np.asarray(result.state, dtype=np.int64).reshape(shape),
                     alpha=alpha, beta=beta, hit_states=states_flat.reshape(shape + (STATE_SIZE,)), result=result,
                     camera=cam, spacetime=st, disk=disk, backend=getattr(be, "name", "cuda"))


def save_disk_image(path: Path | str, image: DiskImage) -> Path:
    """The reference's ``.npz`` of a rendered disk (``raytracing/renderer.py:save_disk_image``)."""
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    cam, disk, st = image.camera, image.disk, image.spacetime
    np.savez_compressed(target, intensity=image.intensity, g=image.g, hit=image.hit, r_hit=image.r_hit,
                        state=image.state, alpha=image.alpha, beta=image.beta, hit_states=image.hit_states,
                        lam=np.asarray(image.result.lam, dtype=np.float64), n_steps=np.asarray(image.result.n_steps),
                        max_null_error=np.asarray(image.result.max_null_error, dtype=np.float64), mass=st.mass,
                        spin=st.spin, inclination_deg=cam.inclination_deg, camera_radius=cam.radius, fov=cam.fov,
                        resolution=cam.resolution, r_in=disk.r_in, r_out=disk.r_out,
                        emissivity_index=disk.emissivity_index, redshift_power=disk.redshift_power,
                        prograde=disk.prograde)
    return target


def load_disk_image_arrays(path: Path | str) -> dict[str, Any]:
    """A file of :func:`save_disk_image` as a plain dict of arrays and scalars."""
    with np.load(Path(path)) as data:
        return {key: (data[key].item() if data[key].ndim == 0 else data[key]) for key in data.files}
