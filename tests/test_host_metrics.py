"""Host-side shadow-edge metrics against the reference's own outputs (golden fixtures):
Bardeen curves (``photons/orbits.py:206-273``), critical impact parameters, the
finite-distance factor and the mask-edge extraction and error summary
(``raytracing/boundary.py``). CPU only.

This package computes these differently from the reference (closed-form orbits, the exact
curve instead of a sampled polygon, the exact level set instead of 1/8-pixel marching), so the
pins are: the reference's curve points lie on the exact curve; its polygon lies inside it by no
more than the chord sag; the reference's marched edge lies within its interpolation error of
the exact level set; and the error summary reproduces the reference's numbers on the
reference's own edge and curve.
"""

from __future__ import annotations

import math

import numpy as np

from conftest import golden
import kerrray_b200 as K
from kerrray_b200 import boundary as B
from kerrray_b200 import orbits as O

SPINS = (0.0, 0.5, 0.9, 0.99, 0.8)
INCLINATIONS = (17.0, 60.0, 85.0)


def test_critical_impact_parameters_match_reference() -> None:
    d = golden("bardeen_curves")
    for spin in SPINS:
        st = K.Spacetime(1.0, spin)
        assert np.allclose(O.critical_impact_parameters(st), d[f"bc_{spin:g}"], rtol=1e-13, atol=0)
        assert B.finite_distance_scale(st, 1000.0) == float(d[f"kscale_{spin:g}_1000"])
        assert B.finite_distance_scale(st, 1.0e5) == float(d[f"kscale_{spin:g}_1e5"])
    assert abs(O.critical_impact_parameters(K.Spacetime(1.0, 0.0))[0] - 3.0 * math.sqrt(3.0)) < 1e-14


def test_reference_curve_points_lie_on_the_exact_bardeen_curve() -> None:
    d = golden("bardeen_curves")
    for spin in SPINS:
        st = K.Spacetime(1.0, spin)
        for incl in INCLINATIONS:
            ra, rb = d[f"curve_{spin:g}_{incl:g}_alpha"], d[f"curve_{spin:g}_{incl:g}_beta"]
            curve = O.BardeenCurve(st, incl)
            exact = curve.radii((0.0, 0.0), np.arctan2(rb, ra))
            assert np.max(np.abs(exact - np.hypot(ra, rb))) < 1e-12, (spin, incl)
            # Sampled uniformly in polar angle and ordered by it; the reference's 720-point polygon
            # lies inside the convex curve by at most its chord sag (~1e-4 M here).
            a, b = O.shadow_curve(st, incl, 720)
            phi = np.arctan2(b, a)
            assert a.shape == (720,) and np.all(np.diff(phi) > 0.0)
            assert np.allclose(np.hypot(a, b), curve.radii((0.0, 0.0), phi), rtol=0, atol=1e-13)
            sag = np.hypot(a, b) - B.polygon_radii(ra, rb, (0.0, 0.0), phi)
            assert sag.min() > -1e-12 and sag.max() < 1e-4, (spin, incl, sag.min(), sag.max())
            # The shoelace centroid of the reference's polygon is the reference's; the exact
            # centroid differs from it by the polygon's O(n^-2) error.
            c_ref = d[f"centroid_{spin:g}_{incl:g}"]
            assert np.allclose(B.polygon_centroid(ra, rb), c_ref, atol=1e-12)
            assert np.allclose(curve.centroid(), c_ref, atol=3e-5)


def test_polygon_radii_equal_brute_force_intersection() -> None:
    g = golden("boundary_shadow64")
    ca, cb = g["curve_alpha"], g["curve_beta"]
    phi = np.linspace(-3.0, 9.0, 997)
    centre = (0.3, -0.2)
    qx, qy = ca - centre[0], cb - centre[1]
    ex, ey = np.roll(qx, -1) - qx, np.roll(qy, -1) - qy
    dx, dy = np.cos(phi)[:, None], np.sin(phi)[:, None]
    with np.errstate(all="ignore"):
        den = dx * ey - dy * ex
        t = (qx * ey - qy * ex) / den
        s = (qx * dy - qy * dx) / den
    t = np.where((t > 0) & (s >= -1e-12) & (s <= 1 + 1e-12), t, np.inf).min(axis=1)
    assert np.allclose(B.polygon_radii(ca, cb, centre, phi), t, rtol=0, atol=1e-13)


def _bilinear(field: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """The mask's interpolant at padded grid coordinates (a direct evaluation for the test)."""
    j, i = np.floor(u).astype(int), np.floor(v).astype(int)
    fu, fv = u - j, v - i
    return (field[i, j] * (1 - fu) * (1 - fv) + field[i, j + 1] * fu * (1 - fv) + field[i + 1, j] * (1 - fu) * fv
            + field[i + 1, j + 1] * fu * fv)


def test_mask_edge_extraction_and_error_match_reference() -> None:
    d = golden("shadow64_a0.9_i60")
    g = golden("boundary_shadow64")
    cam = K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)
    alpha, beta = cam.pixel_coordinates()
    captured = d["state"].reshape(cam.shape) == 2
    centre = B.mask_centroid(alpha, beta, captured)
    assert np.array_equal(np.array(centre), g["centre"])
    angles, radii = B.extract_boundary_from_mask(alpha, beta, captured, n_angles=360)
    assert np.array_equal(angles, g["angles"])
    # The edge is the exact 0.5 level set of the bilinear interpolant ...
    px = cam.pixel_size
    field = np.pad(captured.astype(float), 1)
    u = (centre[0] + radii * np.cos(angles) - alpha[0, 0]) / px + 1.0
    v = (beta[0, 0] - centre[1] - radii * np.sin(angles)) / px + 1.0
    assert np.max(np.abs(_bilinear(field, u, v) - 0.5)) < 1e-9
    # ... and the reference's marched edge lies within its linear-interpolation error of it.
    assert np.max(np.abs(radii - g["radii"])) < 0.01 * px
    st = K.Spacetime(1.0, 0.9)
    ref = dict(zip(g["err_keys"].tolist(), g["err_vals"].tolist()))
    keys = ("max", "rms", "mean", "mean_abs", "max_px", "rms_px", "mean_px", "mean_abs_px")
    # On the reference's own edge and curve the summary is the reference's.
    same = B.boundary_error((g["angles"], g["radii"]), (g["curve_alpha"], g["curve_beta"]), centre,
                            pixel_size=px, scale=float(g["scale"]))
    for k in keys:
        assert abs(same[k] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k
    assert abs(same["radius_mean_numeric"] - ref["numeric_radius_mean"]) < 1e-12
    # The exact edge against the exact curve: within 1e-3 px of the reference's figures.
    err = B.mask_edge_error(st, cam, captured)
    for k in keys:
        if k.endswith("_px"):
            assert abs(err[k] - ref[k]) < 1e-3, (k, err[k], ref[k])
    assert err["rms_px"] < 0.5  # the mask edge within half a pixel of Bardeen's curve


def test_winding_prediction_and_initial_states_match_reference() -> None:
    """Closed-form R'' against the study's central differences; equatorial photon states."""
    from kerrray_b200 import validation as V
    from kerrray_b200.types import Spacetime

    d = golden("winding")
    for k, (spin, prograde) in enumerate(zip(d["spins"], d["prograde"])):
        pred = V.winding_rate_prediction(float(spin), bool(prograde))
        assert abs(pred - d["predicted"][k]) <= 1e-7 * pred
        st = Spacetime(1.0, float(spin))
        for j, delta in enumerate(d["deltas"]):
            y = V.equatorial_photon(st, 50.0, float(d["b_c"][k]) * (1 + float(delta)), prograde=bool(prograde))
            assert np.allclose(y, d["Y0"][k][j], rtol=1e-14, atol=0.0)


def test_direction_angle_is_the_angle_on_the_sphere() -> None:
    """direction_angle against the spherical law of cosines where that is well conditioned, the
    small-angle form next to a pole (where phi alone overstates the distance by 1 / sin theta),
    wrapping in phi, and NaN for a ray that did not escape."""
    rng = np.random.default_rng(5)
    t1, p1 = rng.uniform(0.2, 2.9, 500), rng.uniform(-np.pi, np.pi, 500)
    t2, p2 = rng.uniform(0.2, 2.9, 500), rng.uniform(-np.pi, np.pi, 500)
    cos_d = np.cos(t1) * np.cos(t2) + np.sin(t1) * np.sin(t2) * np.cos(p1 - p2)
    ref = np.arccos(np.clip(cos_d, -1.0, 1.0))
    big = ref > 1e-2  # the law of cosines loses digits for small angles
    assert np.allclose(K.direction_angle(t1, p1, t2, p2)[big], ref[big], rtol=1e-12, atol=0)
    th = np.pi - 0.012
    d = K.direction_angle(th, 1.0, th, 1.0 + 1e-4)
    assert abs(d - np.sin(th) * 1e-4) < 1e-12          # 1.2e-6 rad, not 1e-4
    assert abs(K.direction_angle(1.0, np.pi - 1e-7, 1.0, -np.pi + 1e-7) - np.sin(1.0) * 2e-7) < 1e-15
    assert np.isnan(K.direction_angle(np.nan, 0.0, 1.0, 0.0))
