"""The accretion-disk renderer against the reference's own render_disk (golden fixture
render_disk24.npz: a* = 0.9, i = 75 deg, fov 25 M, 24 x 24, rtol 1e-8; a prograde g^4 disk from
the ISCO to 20 M and a retrograde g^3 disk to 15 M, numba backend).

CPU: the disk model (ISCO, photon-orbit check, validation) and the shading formula restated in
NumPy against the reference's g and I_obs at its own crossing states. GPU: render_disk end to
end (camera, integration with the disk-plane event, shading on the device)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden

K = pytest.importorskip("kerrray_b200")


def _disk(d, tag):
    return K.DiskModel(r_in=float(d[f"{tag}_r_in"]), r_out=float(d[f"{tag}_r_out"]),
                       emissivity_index=float(d[f"{tag}_emissivity_index"]),
                       intensity_law="g4" if int(d[f"{tag}_redshift_power"]) == 4 else "g3",
                       prograde=bool(d[f"{tag}_prograde"]))


def _shade(st, disk, y):
    """g and I_obs of crossing states y (n x 8) by the closed forms the device kernel uses."""
    m, a = st.mass, st.spin * st.mass
    r, pt, pph = y[:, 1], y[:, 4], y[:, 7]
    s = 1.0 if disk.prograde else -1.0
    om = s * (1.0 if a >= 0 else -1.0) * math.sqrt(m) / (r ** 1.5 + s * abs(a) * math.sqrt(m))
    g_tt, g_tph, g_phph = -(1.0 - 2.0 * m / r), -2.0 * m * a / r, r * r + a * a + 2.0 * m * a * a / r
    ut = 1.0 / np.sqrt(-(g_tt + 2.0 * om * g_tph + om * om * g_phph))
    g = pt / (pt * ut + pph * om * ut)
    inside = (r >= disk.r_in) & (r <= disk.r_out)
    return g, np.where(inside, (r / disk.r_in) ** -disk.emissivity_index * g ** disk.redshift_power, 0.0)


def test_disk_model_and_shading_formula_match_the_reference() -> None:
    d = golden("render_disk24")
    st = K.Spacetime(float(d["mass"]), float(d["spin"]))
    pro = K.DiskModel.for_spacetime(st)
    assert abs(pro.r_in - float(d["pro_r_in"])) <= 1e-14 * pro.r_in and pro.redshift_power == 4
    retro = K.DiskModel.for_spacetime(st, r_out=15.0, emissivity_index=2.5, intensity_law="g3", prograde=False)
    assert abs(retro.r_in - float(d["retro_r_in"])) <= 1e-14 * retro.r_in
    for tag in ("pro", "retro"):
        disk = _disk(d, tag)
        hit = d[f"{tag}_hit"].ravel()
        y = d[f"{tag}_hit_states"].reshape(-1, 8)[hit]
        g, inten = _shade(st, disk, y)
        np.testing.assert_allclose(g, d[f"{tag}_g"].ravel()[hit], rtol=1e-13)
        np.testing.assert_allclose(inten, d[f"{tag}_intensity"].ravel()[hit], rtol=1e-12)
        assert np.all(np.isnan(d[f"{tag}_g"].ravel()[~hit])) and np.all(d[f"{tag}_intensity"].ravel()[~hit] == 0)
    with pytest.raises(ValueError):
        K.DiskModel(r_in=6.0, r_out=5.0)
    with pytest.raises(ValueError):
        K.DiskModel(r_in=6.0, r_out=20.0, intensity_law="g5")
    with pytest.raises(ValueError):  # below the circular photon orbit: no circular gas orbit
        K.DiskModel.for_spacetime(st, r_in=1.5)


def test_oracle_crossings_are_the_reference_crossings() -> None:
    """The oracle (the reference's kernel restated in C++) on the renderer's camera rays with the
    disk-plane event reproduces the reference's crossing states bit for bit."""
    from oracle import oracle as O

    d = golden("render_disk24")
    m, spin = float(d["mass"]), float(d["spin"])
    a, b = O.pixel_coordinates(float(d["camera_fov"]), int(d["camera_resolution"]))
    y0 = O.initial_states(m, spin, float(d["camera_radius"]), float(d["camera_inclination_deg"]), 0.0, a, b)
    for tag in ("pro", "retro"):
        opts = O.Options(rtol=float(d["rtol"]), atol=float(d["atol"]), disk_plane=True, r_in=float(d[f"{tag}_r_in"]),
                         r_out=float(d[f"{tag}_r_out"]))
        out = O.integrate(m, spin, y0, opts, threads=4)
        hit = d[f"{tag}_hit"].ravel()
        assert np.array_equal(out["state"], d[f"{tag}_state"].ravel())
        assert np.array_equal(out["event_hit"].astype(bool), hit)
        assert np.array_equal(out["event_Y"][hit], d[f"{tag}_hit_states"].reshape(-1, 8)[hit])


@pytest.mark.gpu
def test_render_disk_matches_the_reference(tmp_path) -> None:
    d = golden("render_disk24")
    st = K.Spacetime(float(d["mass"]), float(d["spin"]))
    cam = K.Camera(radius=float(d["camera_radius"]), inclination_deg=float(d["camera_inclination_deg"]),
                   fov=float(d["camera_fov"]), resolution=int(d["camera_resolution"]))
    integ = K.IntegratorOptions(method="rk45", rtol=float(d["rtol"]), atol=float(d["atol"]))
    term = K.TerminationOptions()
    for tag in ("pro", "retro"):
        disk = _disk(d, tag)
        img = K.render_disk(st, cam, integ, term, disk)
        assert np.array_equal(img.state, d[f"{tag}_state"]) and np.array_equal(img.hit, d[f"{tag}_hit"])
        # The device's FP64 libm differs from the reference's in the last bits, which the
        # integration carries to ~1e-10 of the crossing states (rtol 1e-8 here).
        hit = img.hit
        np.testing.assert_allclose(img.hit_states[hit], d[f"{tag}_hit_states"][hit], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(img.r_hit[hit], d[f"{tag}_r_hit"][hit], rtol=1e-9)
        np.testing.assert_allclose(img.g[hit], d[f"{tag}_g"][hit], rtol=1e-9)
        np.testing.assert_allclose(img.intensity, d[f"{tag}_intensity"], rtol=1e-8, atol=0)
        # the shading itself: the device's g and I_obs at its own crossing states
        g_own, i_own = _shade(st, disk, img.hit_states[hit])
        np.testing.assert_allclose(img.g[hit], g_own, rtol=1e-13)
        np.testing.assert_allclose(img.intensity[hit], i_own, rtol=1e-12)
        assert np.all(np.isnan(img.g[~hit])) and np.all(img.intensity[~hit] == 0)
        back = K.load_disk_image_arrays(K.save_disk_image(tmp_path / f"{tag}.npz", img))
        assert np.array_equal(back["hit"], img.hit) and back["redshift_power"] == disk.redshift_power
