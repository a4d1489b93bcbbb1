"""Pin the oracle: the C++ restatement must reproduce the reference's own golden vectors.

The fixtures were written by the reference's ``numba`` backend
(``src/kerrray/raytracing/backends/numba_backend.py:131-207``) and camera
(``raytracing/camera.py:298-381``) through ``tests/golden/make_golden.py``.
The oracle is compiled without contraction and uses the C library's sin, cos
and pow like the Numba build, so agreement is bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TRACE_FIXTURES, golden, golden_options
from oracle import oracle as O

FIELDS = ("Y", "state", "n_steps", "n_rejected", "lam", "max_null_error", "max_energy_drift", "max_lz_drift",
          "max_carter_drift")


@pytest.mark.parametrize("name", TRACE_FIXTURES)
def test_oracle_matches_reference_bit_for_bit(name: str) -> None:
    d = golden(name)
    out = O.integrate(float(d["mass"]), float(d["spin"]), d["Y0"], golden_options(d))
    for field in FIELDS:
        assert np.array_equal(np.asarray(out[field]), np.asarray(d[field]).astype(np.asarray(out[field]).dtype)), field
    if "event_Y" in d:
        assert np.array_equal(out["event_Y"], d["event_Y"]) and np.array_equal(out["event_hit"], d["event_hit"])


def test_oracle_sweep_sample_all_spins_inclinations_tolerances() -> None:
    d = golden("sweep_sample_128")
    for k in range(len(d["spin"])):
        rtol = float(d["rtol"][k])
        out = O.integrate(1.0, float(d["spin"][k]), d["Y0"][k], O.Options(rtol=rtol, atol=1e-2 * rtol))
        assert np.array_equal(out["state"], d["state"][k].astype(np.int64))
        assert np.array_equal(out["n_steps"], d["n_steps"][k].astype(np.int64))
        assert np.array_equal(out["Y"], d["Y"][k])


def test_oracle_camera_matches_reference() -> None:
    d = golden("camera_states")
    for k in range(int(d["n_cameras"])):
        p = lambda n: d[f"c{k}_{n}"]  # noqa: E731
        a, b = O.pixel_coordinates(float(p("camera_fov")), int(p("camera_resolution")))
        assert np.array_equal(a, p("alpha")) and np.array_equal(b, p("beta"))
        y = O.initial_states(float(p("mass")), float(p("spin")), float(p("camera_radius")),
                             float(p("camera_inclination_deg")), float(p("camera_phi_deg")), a, b)
        assert np.array_equal(y, p("Y0"))


def test_oracle_validates_input_like_the_reference() -> None:
    with pytest.raises(ValueError):
        O.integrate(1.0, 0.9, np.ones((2, 7)), O.Options())
    bad = np.ones((1, 8))
    bad[0, 3] = np.nan
    with pytest.raises(ValueError):
        O.integrate(1.0, 0.9, bad, O.Options())
    empty = O.integrate(1.0, 0.9, np.zeros((0, 8)), O.Options())
    assert empty["Y"].shape == (0, 8) and empty["state"].shape == (0,)


def test_flop_count_per_attempt_is_constant() -> None:
    """The reference algorithm does 1210 floating-point operations per DP5(4) attempt."""
    d = golden("shadow64_a0.9_i60")
    c = O.count_flops(1.0, 0.9, d["Y0"][::64], O.Options(rtol=1e-6, atol=1e-8))
    per_attempt = {k: v / c["attempts"] for k, v in c["attempt"].items()}
    assert per_attempt == {"add": 377.0, "mul": 702.0, "div": 111.0, "sqrt": 1.0, "trig": 18.0, "pow": 1.0}
    assert sum(c["accept"].values()) == 28 * c["accepted"]
    assert sum(c["init"].values()) == 127 * c["rays"]


def test_oracle_winding_rays_match_reference() -> None:
    """The winding study's 54 near-critical equatorial rays (rtol 1e-12, escape radius 60 M)."""
    d = golden("winding")
    opts = O.Options(rtol=1e-12, atol=1e-14, max_steps=400_000, escape_radius=60.0)
    for k, spin in enumerate(d["spins"]):
        out = O.integrate(1.0, float(spin), d["Y0"][k], opts)
        assert np.array_equal(out["state"], d["state"][k].astype(np.int64))
        assert np.array_equal(out["n_steps"], d["n_steps"][k].astype(np.int64))
        assert np.array_equal(out["Y"], d["Y"][k])
