"""Generate the golden fixtures of the per-ray hot path from the KerrRay reference.

Run where the reference source tree is present (it is read, never modified):
by default the ``reference`` directory beside this repository's root, or the
tree that ``KRR_REFERENCE`` names::

    KRR_REFERENCE=<reference tree> python tests/golden/make_golden.py

Every fixture is produced by the reference's own code: its ``numba`` backend
(``src/kerrray/raytracing/backends/numba_backend.py:131-207``, the FP64 oracle
named for this path), its camera (``raytracing/camera.py:298-381``), its
Bardeen curve (``photons/orbits.py:206-273``), its boundary metrics
(``raytracing/boundary.py``) and its edge bisection
(``scripts/study_edge_bisection.py:53-68``). The outputs are small ``.npz``
files next to this script; the GPU tests and the oracle tests read only those
files, never the reference tree.
"""

from __future__ import annotations

import math
import os
import sys
import time
from pathlib import Path

import numpy as np

REF = Path(os.environ.get("KRR_REFERENCE") or Path(__file__).resolve().parents[3] / "reference")
OUT = Path(__file__).resolve().parent

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/krr_numba_cache")
os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path.insert(0, str(REF / "src"))
sys.path.insert(0, str(REF / "scripts"))

from kerrray.geodesics import EventOptions, IntegratorOptions, TerminationOptions  # noqa: E402
from kerrray.geodesics.initial_conditions import photon_from_constants, tangential_photon  # noqa: E402
from kerrray.geodesics.integrators import max_attempts  # noqa: E402
from kerrray.geometry import Spacetime  # noqa: E402
from kerrray.photons.orbits import critical_impact_parameters, shadow_curve  # noqa: E402
from kerrray.raytracing.backends.numba_backend import NumbaBackend  # noqa: E402
from kerrray.raytracing.boundary import (  # noqa: E402
    analytic_boundary,
    boundary_error,
    extract_boundary_from_mask,
    finite_distance_scale,
    mask_centroid,
    polygon_centroid,
    polygon_radii,
)
from kerrray.raytracing.camera import Camera, initial_states  # noqa: E402

BACKEND = NumbaBackend()


def _integ_fields(integ: IntegratorOptions) -> dict:
    h_max = np.inf if integ.h_max is None else integ.h_max
    return {
        "integ_method": np.array(integ.method),
        "integ_rtol": np.float64(integ.rtol),
        "integ_atol": np.float64(integ.atol),
        "integ_step_size": np.float64(integ.step_size),
        "integ_max_steps": np.int64(integ.max_steps),
        "integ_lambda_max": np.float64(integ.lambda_max),
        "integ_h_min": np.float64(integ.h_min),
        "integ_h_max": np.float64(h_max),
        "integ_dtype": np.array(integ.dtype),
        "integ_max_attempts": np.int64(max_attempts(integ)),
    }


def _run(name: str, st: Spacetime, y0: np.ndarray, integ: IntegratorOptions, term: TerminationOptions,
         events: EventOptions | None = None, extra: dict | None = None) -> dict:
    res = BACKEND.integrate_batch(st, y0, integ, term, events=events)
    payload = {
        "mass": np.float64(st.mass),
        "spin": np.float64(st.spin),
        "Y0": np.asarray(y0, dtype=np.float64),
        "Y": np.asarray(res.Y),
        "state": np.asarray(res.state, dtype=np.int8),
        "n_steps": np.asarray(res.n_steps, dtype=np.int32),
        "n_rejected": np.asarray(res.n_rejected, dtype=np.int32),
        "lam": np.asarray(res.lam),
        "max_null_error": np.asarray(res.max_null_error),
        "max_energy_drift": np.asarray(res.max_energy_drift),
        "max_lz_drift": np.asarray(res.max_lz_drift),
        "max_carter_drift": np.asarray(res.max_carter_drift),
        "term_horizon_epsilon": np.float64(term.horizon_epsilon),
        "term_escape_radius": np.float64(term.escape_radius),
        **_integ_fields(integ),
    }
    if events is not None:
        payload.update({
            "event_disk_plane": np.bool_(events.disk_plane),
            "event_r_in": np.float64(events.r_in),
            "event_r_out": np.float64(events.r_out),
            "event_Y": np.asarray(res.event_Y),
            "event_hit": np.asarray(res.event_hit),
        })
    if extra:
        payload.update(extra)
    np.savez_compressed(OUT / f"{name}.npz", **payload)
    counts = np.bincount(np.asarray(res.state), minlength=7)
    print(f"{name:28s} N={len(y0):5d} states={counts.tolist()} steps mean={np.mean(res.n_steps):.1f}")
    return payload


def _camera_fields(cam: Camera) -> dict:
    return {
        "camera_radius": np.float64(cam.radius),
        "camera_inclination_deg": np.float64(cam.inclination_deg),
        "camera_phi_deg": np.float64(cam.phi_deg),
        "camera_fov": np.float64(cam.fov),
        "camera_resolution": np.int64(cam.resolution),
    }


def main() -> None:
    t0 = time.perf_counter()
    BACKEND.warm_up(Spacetime(1.0, 0.9), IntegratorOptions(), TerminationOptions())

    # 1. The 64 x 64 plain FP64 shadow image (a* = 0.9, i = 60 deg, r_o = 1000 M, +-8 M,
    #    rtol 1e-6, atol 1e-8, reference defaults otherwise).
    st = Spacetime(1.0, 0.9)
    cam = Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)
    integ = IntegratorOptions(method="rk45", rtol=1e-6, atol=1e-8)
    term = TerminationOptions()
    p = _run("shadow64_a0.9_i60", st, initial_states(cam, st), integ, term, extra=_camera_fields(cam))
    alpha, beta = cam.pixel_coordinates()
    captured = p["state"].reshape(cam.shape) == 2
    centre = mask_centroid(alpha, beta, captured)
    angles, radii = extract_boundary_from_mask(alpha, beta, captured, n_angles=360)
    curve = analytic_boundary(st, cam.inclination_deg, 720)
    scale = finite_distance_scale(st, cam.radius)
    err = boundary_error((angles, radii), curve, centre, pixel_size=cam.pixel_size, scale=scale)
    np.savez_compressed(
        OUT / "boundary_shadow64.npz",
        centre=np.array(centre), angles=angles, radii=radii, curve_alpha=curve[0], curve_beta=curve[1],
        scale=np.float64(scale),
        err_keys=np.array(sorted(err)), err_vals=np.array([err[k] for k in sorted(err)]),
    )

    # 2. The reference's own parity case (tests/test_numba_backend.py:92-118): the first
    #    500 pixels of a 24 x 24 image, fov 12, rtol 1e-8, atol 1e-10.
    cam24 = Camera(radius=1000.0, inclination_deg=60.0, fov=12.0, resolution=24)
    _run("camera24_rtol1e-8", st, initial_states(cam24, st)[:500],
         IntegratorOptions(method="rk45", rtol=1e-8, atol=1e-10), term)

    # 3. Budgets (test_numba_backend.py:139-153): max_steps 30 and lambda_max 500.
    cam4 = Camera(radius=1000.0, inclination_deg=60.0, fov=12.0, resolution=4)
    y4 = initial_states(cam4, st)
    _run("budget_max_steps30", st, y4, IntegratorOptions(method="rk45", rtol=1e-8, atol=1e-10, max_steps=30), term)
    _run("budget_lambda500", st, y4, IntegratorOptions(method="rk45", rtol=1e-8, atol=1e-10, lambda_max=500.0), term)

    # 4. Step caps (tests/test_max_step.py:66-75): h_max None / 20 / 3 on 60 camera rays.
    cam16 = Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=16)
    y16 = initial_states(cam16, st)[:60]
    for cap in (None, 20.0, 3.0):
        tag = "none" if cap is None else f"{cap:g}"
        _run(f"hmax_{tag}", st, y16, IntegratorOptions(rtol=1e-6, atol=1e-8, lambda_max=1e4, h_max=cap), term)

    # 5. Schwarzschild limit (test_numba_backend.py:171-177).
    st0 = Spacetime(1.0, 0.0)
    cam6 = Camera(radius=1000.0, inclination_deg=90.0, fov=8.0, resolution=6)
    _run("schwarzschild_6x6_rtol1e-9", st0, initial_states(cam6, st0),
         IntegratorOptions(method="rk45", rtol=1e-9, atol=1e-11), term)

    # 6. Failures at rtol 1e-4 with an unbounded step (scripts/audit/audit_max_step.out:1-13):
    #    the step jumps through the hole to r < 0 or leaves [0, pi] in theta (OUT_OF_DOMAIN).
    #    A 512 x 512 image is traced once; every failed pixel and a strided sample of the
    #    others are kept.
    cam512 = Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=512)
    y512 = initial_states(cam512, st)
    loose = IntegratorOptions(method="rk45", rtol=1e-4, atol=1e-6)
    full = BACKEND.integrate_batch(st, y512, loose, term)
    bad = np.flatnonzero((full.state != 1) & (full.state != 2))
    keep = np.unique(np.concatenate([bad, np.arange(0, len(y512), 997)]))
    _run("failures_512_rtol1e-4", st, y512[keep], loose, term, extra={"pixel_index": keep.astype(np.int64)})

    # 7. h_min failure: a tight tolerance with a large h_min rejects below h_min.
    _run("hmin_failure", st, y4, IntegratorOptions(method="rk45", rtol=1e-12, atol=1e-14, h_min=0.5), term)

    # 8. Axis guard: exact L_z = 0 rays (p_phi == 0) and rays through the polar region.
    ys = []
    for r0, q in ((30.0, 20.0), (50.0, 40.0), (15.0, 5.0)):
        for s_th in (1, -1):
            ys.append(photon_from_constants(st, r0, 0.3, 1.0, 0.0, q, sign_r=-1, sign_theta=s_th))
    _run("axis_lz0", st, np.stack(ys), IntegratorOptions(method="rk45", rtol=1e-8, atol=1e-10, lambda_max=2000.0), term)

    # 9. Spin/inclination/tolerance coverage of the batched sweep: for each of the 36
    #    (spin, inclination, rtol) combinations of the 128 x 128 images, 48 pixels
    #    (24 strided across the image and 24 along the row through the centre).
    rows = []
    for spin in (0.0, 0.5, 0.9, 0.99):
        stc = Spacetime(1.0, spin)
        for incl in (17.0, 60.0, 85.0):
            camc = Camera(radius=1000.0, inclination_deg=incl, fov=8.0, resolution=128)
            y_all = initial_states(camc, stc)
            idx = np.unique(np.concatenate([np.arange(0, 128 * 128, 683)[:24], 64 * 128 + np.arange(8, 120, 5)[:24]]))
            for rtol in (1e-6, 1e-8, 1e-10):
                res = BACKEND.integrate_batch(stc, y_all[idx], IntegratorOptions(method="rk45", rtol=rtol, atol=1e-2 * rtol), term)
                rows.append((spin, incl, rtol, idx, y_all[idx], res))
    np.savez_compressed(
        OUT / "sweep_sample_128.npz",
        spin=np.array([r[0] for r in rows]), incl=np.array([r[1] for r in rows]), rtol=np.array([r[2] for r in rows]),
        pixel_index=np.stack([r[3] for r in rows]), Y0=np.stack([r[4] for r in rows]),
        Y=np.stack([r[5].Y for r in rows]), state=np.stack([r[5].state for r in rows]).astype(np.int8),
        n_steps=np.stack([r[5].n_steps for r in rows]).astype(np.int32),
        n_rejected=np.stack([r[5].n_rejected for r in rows]).astype(np.int32),
        lam=np.stack([r[5].lam for r in rows]),
        max_null_error=np.stack([r[5].max_null_error for r in rows]),
        max_carter_drift=np.stack([r[5].max_carter_drift for r in rows]),
    )
    print("sweep_sample_128             36 combos x", len(rows[0][3]))

    # 10. Working-precision and scheme variants of the backend protocol.
    cam6b = Camera(radius=1000.0, inclination_deg=60.0, fov=12.0, resolution=6)
    _run("float32_6x6", st, initial_states(cam6b, st),
         IntegratorOptions(method="rk45", rtol=1e-6, atol=1e-8, dtype="float32"), TerminationOptions(horizon_epsilon=1e-3))
    far = TerminationOptions(escape_radius=1e6)
    y_rk4 = np.stack([photon_from_constants(st, 15.0, 1.0, 1.0, lz, 4.0, sign_r=1, sign_theta=-1) for lz in (2.0, -3.0, 0.5)])
    _run("rk4_budget", st, y_rk4, IntegratorOptions(method="rk4", step_size=0.05, lambda_max=20.0), far)
    y_disk = np.stack([photon_from_constants(st, 200.0, 1.2, 1.0, lz, 15.0, sign_r=-1, sign_theta=1) for lz in (-6.0, 3.0, 6.0, 9.0)])
    ev = EventOptions(disk_plane=True, r_in=6.0, r_out=30.0)
    for dt in ("float64", "float32"):
        _run(f"disk_{dt}", st, y_disk, IntegratorOptions(method="rk45", rtol=1e-7, atol=1e-9, lambda_max=400.0, dtype=dt), far, events=ev)

    # 11. Camera initial states (raytracing/camera.py:298-381), including the inclination
    #     clamp, an observer azimuth, a far observer and the smallest image.
    cams = [
        (Spacetime(1.0, 0.9), Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)),
        (Spacetime(1.0, 0.99), Camera(radius=1000.0, inclination_deg=85.0, fov=8.0, resolution=16)),
        (Spacetime(1.0, 0.0), Camera(radius=1000.0, inclination_deg=17.0, fov=8.0, resolution=8)),
        (Spacetime(1.0, 0.5), Camera(radius=1.0e5, inclination_deg=0.0, fov=8.0, resolution=4)),
        (Spacetime(1.0, -0.7), Camera(radius=50.0, inclination_deg=120.0, phi_deg=30.0, fov=12.0, resolution=2)),
        (Spacetime(1.0, 0.99), Camera(radius=4.0, inclination_deg=90.0, fov=2.0, resolution=6)),
        (Spacetime(2.0, 0.8), Camera(radius=1000.0, inclination_deg=60.0, fov=24.0, resolution=10)),
    ]
    cam_payload = {}
    for k, (stc, camc) in enumerate(cams):
        cam_payload[f"c{k}_mass"] = np.float64(stc.mass)
        cam_payload[f"c{k}_spin"] = np.float64(stc.spin)
        for key, val in _camera_fields(camc).items():
            cam_payload[f"c{k}_{key}"] = val
        cam_payload[f"c{k}_Y0"] = initial_states(camc, stc)
        a, b = camc.pixel_coordinates()
        cam_payload[f"c{k}_alpha"], cam_payload[f"c{k}_beta"] = a, b
    cam_payload["n_cameras"] = np.int64(len(cams))
    np.savez_compressed(OUT / "camera_states.npz", **cam_payload)
    print("camera_states                ", len(cams), "cameras")

    # 12. Bardeen curves of the twelve (spin, inclination) cases, b_c and k(r_o).
    bard = {}
    for spin in (0.0, 0.5, 0.9, 0.99, 0.8):
        stc = Spacetime(1.0, spin)
        bard[f"bc_{spin:g}"] = np.array(critical_impact_parameters(stc))
        for incl in (17.0, 60.0, 85.0):
            ca, cb = shadow_curve(stc, incl, 720)
            bard[f"curve_{spin:g}_{incl:g}_alpha"], bard[f"curve_{spin:g}_{incl:g}_beta"] = ca, cb
            bard[f"centroid_{spin:g}_{incl:g}"] = np.array(polygon_centroid(ca, cb))
        bard[f"kscale_{spin:g}_1000"] = np.float64(finite_distance_scale(stc, 1000.0))
        bard[f"kscale_{spin:g}_1e5"] = np.float64(finite_distance_scale(stc, 1.0e5))
    np.savez_compressed(OUT / "bardeen_curves.npz", **bard)
    print("bardeen_curves               ", len(bard), "arrays")

    # 13. Edge bisection (scripts/study_edge_bisection.py:53-68) on the numba backend:
    #     a* = 0.9, i = 60 deg, r_o = 1e5 M, rtol 1e-6, 16 directions, 34 halvings of
    #     [0.98, 1.02] x the Bardeen radius about the Bardeen centroid / k.
    from study_edge_bisection import bisect_edge  # noqa: E402

    for spin, rtol in ((0.9, 1e-6), (0.0, 1e-8)):
        stc = Spacetime(1.0, spin)
        incl, r_o, n_dirs, iters = 60.0, 1.0e5, 16, 34
        angles = np.linspace(0.0, 2 * math.pi, n_dirs, endpoint=False) + 0.1
        k = finite_distance_scale(stc, r_o)
        ca, cb = analytic_boundary(stc, incl, 40000)
        c_ana = polygon_centroid(ca, cb)
        r_ana = polygon_radii(ca, cb, c_ana, angles)
        centre_img = (c_ana[0] / k, c_ana[1] / k)
        r_img = r_ana / k
        with np.errstate(all="ignore"):
            r_num, width, failures = bisect_edge(stc, incl, r_o, rtol, centre_img, angles, 0.98 * r_img, 1.02 * r_img,
                                                 iters, BACKEND)
        np.savez_compressed(
            OUT / f"edge_bisection_a{spin:g}_rtol{rtol:g}.npz",
            spin=np.float64(spin), incl=np.float64(incl), r_o=np.float64(r_o), rtol=np.float64(rtol),
            iterations=np.int64(iters), angles=angles, centre_img=np.array(centre_img), r_lo=0.98 * r_img,
            r_hi=1.02 * r_img, r_ana=r_ana, k=np.float64(k), r_num=r_num, width=width, failures=np.int64(failures),
        )
        err = r_num * k - r_ana
        print(f"edge_bisection a={spin} rtol={rtol:g}: rms {np.sqrt(np.mean(err**2)):.2e} M, failures {failures}")

    # 14. Exact checks re-driven on the numba backend with the Schwarzschild validation
    #     settings (configs/schwarzschild.yaml; validation/schwarzschild.py:151-200,
    #     validation/kerr_bisection.py:96-263): rtol 1e-9, atol 1e-11, 15 probes per
    #     iteration, brackets [2.5, 4] M and [4, 7] M, tolerance 1e-6 M.
    st0 = Spacetime(1.0, 0.0)
    integ_v = IntegratorOptions(method="rk45", rtol=1e-9, atol=1e-11)
    term_v = TerminationOptions()
    tang = np.stack([tangential_photon(st0, r) for r in (2.5, 2.9, 3.0 + 1e-3, 3.1, 4.0)])
    _run("tangential_photons_a0", st0, tang, integ_v, term_v)

    # 15. Near-critical winding (scripts/study_winding.py:73-127): the reference's own predicted
    #     rate and its scalar-integrator measurement for the nine (spin, direction) cases, plus the
    #     numba backend on the same initial states (the batch path the cuda backend replaces).
    #     The study imports matplotlib only for its figure; an inert stub stands in for it here.
    import types

    for name in ("matplotlib", "matplotlib.pyplot"):
        stub = types.ModuleType(name)
        stub.use = lambda *a, **k: None
        sys.modules.setdefault(name, stub)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    import study_winding  # noqa: E402
    from kerrray.geodesics.initial_conditions import equatorial_photon  # noqa: E402

    deltas = [1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8]
    cases = [(s, p) for s in (0.0, 0.3, 0.6, 0.9, 0.99) for p in (True, False) if not (s == 0.0 and not p)]
    wind = {"deltas": np.array(deltas), "spins": np.array([c[0] for c in cases]),
            "prograde": np.array([c[1] for c in cases])}
    pred, rate, turns, b_cs, y0s, ys, states, steps = [], [], [], [], [], [], [], []
    integ_w = IntegratorOptions(method="rk45", rtol=1e-12, atol=1e-14, max_steps=400_000)
    term_w = TerminationOptions(horizon_epsilon=1e-6, escape_radius=60.0)
    with np.errstate(all="ignore"):
        for spin, prograde in cases:
            gamma, _, _ = study_winding.predicted_gamma(spin, prograde)
            pred.append(math.log(10) / (2 * math.pi * gamma))
            m = study_winding.measured_rate(spin, prograde, deltas)
            rate.append(m["rate_per_decade"])
            turns.append(m["turns"])
            b_cs.append(m["b_c"])
            stw = Spacetime(1.0, spin)
            y0 = np.stack([equatorial_photon(stw, 50.0, m["b_c"] * (1 + d), prograde=prograde) for d in deltas])
            res = BACKEND.integrate_batch(stw, y0, integ_w, term_w)
            y0s.append(y0)
            ys.append(res.Y)
            states.append(res.state)
            steps.append(res.n_steps)
    wind.update(predicted=np.array(pred), rate_scalar=np.array(rate), turns_scalar=np.array(turns),
                b_c=np.array(b_cs), Y0=np.array(y0s), Y=np.array(ys), state=np.array(states), n_steps=np.array(steps))
    np.savez_compressed(OUT / "winding.npz", **wind)
    for (spin, prograde), p, r in zip(cases, pred, rate):
        print(f"winding a={spin} {'pro' if prograde else 'retro'}: predicted {p:.5f} measured {r:.5f} "
              f"({100 * (r - p) / p:+.3f}%)")
    print(f"done in {time.perf_counter() - t0:.1f} s")


def render_fixture() -> None:
    """The accretion-disk renderer (``raytracing/renderer.py:render_disk``) on the numba backend:
    a* = 0.9, i = 75 deg, r_o = 1000 M, fov 25 M, 24 x 24, rtol 1e-8; the default disk (r_in at
    the prograde ISCO, r_out = 20 M, emissivity index 3, g^4) and a retrograde g^3 disk."""
    from kerrray.physics.accretion import DiskModel, DiskParams
    from kerrray.raytracing.renderer import render_disk

    st = Spacetime(1.0, 0.9)
    cam = Camera(radius=1000.0, inclination_deg=75.0, fov=25.0, resolution=24)
    integ = IntegratorOptions(method="rk45", rtol=1e-8, atol=1e-10)
    term = TerminationOptions()
    out = _camera_fields(cam)
    out.update(mass=np.float64(st.mass), spin=np.float64(st.spin), rtol=np.float64(integ.rtol),
               atol=np.float64(integ.atol))
    for tag, params in (("pro", DiskParams(enabled=True)),
                        ("retro", DiskParams(enabled=True, r_out=15.0, emissivity_index=2.5, intensity_law="g3",
                                             prograde=False))):
        disk = DiskModel.from_params(st, params)
        img = render_disk(st, cam, integ, term, disk, backend=BACKEND)
        out.update({f"{tag}_r_in": np.float64(disk.r_in), f"{tag}_r_out": np.float64(disk.r_out),
                    f"{tag}_emissivity_index": np.float64(disk.emissivity_index),
                    f"{tag}_redshift_power": np.int64(disk.redshift_power), f"{tag}_prograde": np.bool_(disk.prograde),
                    f"{tag}_intensity": img.intensity, f"{tag}_g": img.g, f"{tag}_hit": img.hit,
                    f"{tag}_r_hit": img.r_hit, f"{tag}_state": img.state, f"{tag}_hit_states": img.hit_states})
        print(f"render {tag}: {img.n_hits} hits, r_in {disk.r_in:.6f}, counts {img.counts()}")
    np.savez_compressed(OUT / "render_disk24.npz", **out)


if __name__ == "__main__":
    render_fixture() if "render" in sys.argv[1:] else main()
