"""The analytic capture/escape classes of the critical-set re-trace, against the reference's codes.

``krr_analytic_classes`` classifies a photon from its constants of motion (the minimum of the
radial potential R(r) over [r_+ + epsilon, r_0]) and calls it critical when it lies within a
band of the boundary between capture and escape. The mixed-precision pipeline traces the
critical photons in reference-order FP64 and checks every other photon's code against its
class, so the class must be the reference's own code for every non-critical photon. Host
arithmetic only: these run without a GPU.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

K = pytest.importorskip("kerrray_b200")


def _classes(mass: float, spin: float, rtol: float, eps: float, y0: np.ndarray) -> np.ndarray:
    from kerrray_b200 import _lib

    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    out = np.empty(len(y0), dtype=np.uint8)
    _lib.check(_lib.lib().krr_analytic_classes(mass, spin, rtol, eps, _lib.ptr(y0), len(y0), _lib.ptr(out)))
    return out


def _fixture_classes(name: str):
    d = golden(name)
    c = _classes(float(d["mass"]), float(d["spin"]), float(d["integ_rtol"]), float(d["term_horizon_epsilon"]), d["Y0"])
    return d, c


@pytest.mark.parametrize("name", ["shadow64_a0.9_i60", "camera24_rtol1e-8", "schwarzschild_6x6_rtol1e-9", "hmax_none",
                                  "hmax_20", "hmax_3"])
def test_non_critical_classes_are_the_reference_codes(name: str) -> None:
    d, c = _fixture_classes(name)
    state = d["state"].astype(np.int64)
    assert np.all(state[c == 0] == 1), f"{name}: an escaping class the reference captured"
    assert np.all(state[c == 1] == 2), f"{name}: a captured class the reference let escape"
    assert np.count_nonzero(c == 2) <= 0.01 * c.size


def test_sweep_sample_classes() -> None:
    """36 (spin, inclination, rtol) combinations of the 128^2 sweep, rtol 1e-6 .. 1e-10."""
    d = golden("sweep_sample_128")
    for j in range(len(d["spin"])):
        rtol = float(d["rtol"][j])
        c = _classes(1.0, float(d["spin"][j]), rtol, 1e-6, d["Y0"][j])
        state = d["state"][j].astype(np.int64)
        assert np.all(state[c == 0] == 1) and np.all(state[c == 1] == 2), j


def test_critical_pixels_lie_on_the_shadow_edge() -> None:
    """The 64^2 image (a* = 0.9, i = 60 deg, +-8 M): the critical pixels are those nearest
    Bardeen's curve (after the finite-distance scale k), within the band's 2e-3 M."""
    d, c = _fixture_classes("shadow64_a0.9_i60")
    bard = golden("bardeen_curves")
    cam = K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)
    alpha, beta = cam.pixel_coordinates()
    k = float(bard["kscale_0.9_1000"])
    pts = np.stack([alpha.ravel() * k, beta.ravel() * k], axis=1)
    va = np.stack([bard["curve_0.9_60_alpha"], bard["curve_0.9_60_beta"]], axis=1)
    seg = np.roll(va, -1, axis=0) - va
    t = np.clip(((pts[:, None, :] - va[None]) * seg[None]).sum(-1) / (seg**2).sum(-1)[None], 0.0, 1.0)
    dist = np.linalg.norm(pts[:, None, :] - (va[None] + t[..., None] * seg[None]), axis=-1).min(axis=1)
    crit = c == 2
    assert crit.any()
    # Distance to Bardeen's polygon (720 vertices): the critical pixels are the ones nearest the
    # curve, within the band (2e-3 M, first-order) and the polygon's resolution.
    assert np.all(dist[crit] < 3e-3), dist[crit]
    assert np.all(crit[dist < 1e-3])
    assert dist[~crit].min() > dist[crit].max()


def test_axis_and_outward_rays_are_critical() -> None:
    d, c = _fixture_classes("axis_lz0")  # L_z = 0: the ray crosses the axis (OUT_OF_DOMAIN)
    assert np.all(c == 2)
    y = golden("shadow64_a0.9_i60")["Y0"][:8].copy()
    y[:, 5] = -y[:, 5]  # moving outward: not classified
    assert np.all(_classes(1.0, 0.9, 1e-6, 1e-6, y) == 2)


def test_invalid_arguments() -> None:
    from kerrray_b200 import _lib

    y = golden("shadow64_a0.9_i60")["Y0"][:2]
    with pytest.raises(ValueError):
        _classes(1.0, 0.9, 0.0, 1e-6, y)
    with pytest.raises(ValueError):
        _classes(1.0, 1.5, 1e-6, 1e-6, y)
    assert _lib.lib().krr_analytic_classes(1.0, 0.9, 1e-6, 1e-6, None, 0, None) == 0
