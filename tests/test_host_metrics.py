"""Host-side shadow-edge metrics against the reference's own outputs (golden fixtures):
Bardeen curves (``photons/orbits.py:206-273``), critical impact parameters, the
finite-distance factor and the mask-edge extraction and error summary
(``raytracing/boundary.py``). CPU only."""

from __future__ import annotations

import numpy as np

from conftest import golden
import kerrray_b200 as K
from kerrray_b200 import boundary as B
from kerrray_b200 import orbits as O


def test_bardeen_curves_and_critical_impacts_match_reference() -> None:
    d = golden("bardeen_curves")
    for spin in (0.0, 0.5, 0.9, 0.99, 0.8):
        st = K.Spacetime(1.0, spin)
        assert np.allclose(O.critical_impact_parameters(st), d[f"bc_{spin:g}"], rtol=1e-13, atol=0)
        for incl in (17.0, 60.0, 85.0):
            a, b = O.shadow_curve(st, incl, 720)
            ra, rb = d[f"curve_{spin:g}_{incl:g}_alpha"], d[f"curve_{spin:g}_{incl:g}_beta"]
            assert a.shape == ra.shape and np.max(np.abs(a - ra)) < 1e-11 and np.max(np.abs(b - rb)) < 1e-7
            assert np.allclose(B.polygon_centroid(a, b), d[f"centroid_{spin:g}_{incl:g}"], atol=1e-10)
        assert B.finite_distance_scale(st, 1000.0) == float(d[f"kscale_{spin:g}_1000"])
        assert B.finite_distance_scale(st, 1.0e5) == float(d[f"kscale_{spin:g}_1e5"])


def test_mask_edge_extraction_and_error_match_reference() -> None:
    d = golden("shadow64_a0.9_i60")
    g = golden("boundary_shadow64")
    cam = K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)
    alpha, beta = cam.pixel_coordinates()
    captured = d["state"].reshape(cam.shape) == 2
    centre = B.mask_centroid(alpha, beta, captured)
    assert np.array_equal(np.array(centre), g["centre"])
    angles, radii = B.extract_boundary_from_mask(alpha, beta, captured, n_angles=360)
    assert np.array_equal(angles, g["angles"]) and np.array_equal(radii, g["radii"])
    st = K.Spacetime(1.0, 0.9)
    curve = B.analytic_boundary(st, 60.0, 720)
    err = B.boundary_error((angles, radii), curve, centre, pixel_size=cam.pixel_size,
                           scale=B.finite_distance_scale(st, cam.radius))
    ref = dict(zip(g["err_keys"].tolist(), g["err_vals"].tolist()))
    assert set(err) == set(ref)
    for k, v in ref.items():
        assert abs(err[k] - v) <= 1e-9 * max(1.0, abs(v)), k
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
