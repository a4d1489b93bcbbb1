"""The drop-in boundary through KerrRay's own code (CPU; skipped where the reference tree is absent).

``register_with_kerrray`` makes KerrRay's backend registry (``raytracing/backends/base.py:85-111``)
return this package's ``CudaBackend`` for ``"cuda"``. With no device here the registry must
raise KerrRay's own ``BackendUnavailable`` with this library's reason (not the reference's
stub message) and report ``cuda`` unavailable, also through names that modules imported before
registration (``raytracing/rays.py:27``). With a backend object standing in for the device (the
oracle behind the same ``integrate_batch``), KerrRay's own ``compute_shadow``
(``raytracing/shadow.py:179-211``) must run through the patched name. And shadow files must
move both ways between this package's ``ShadowImage`` and the reference's
(``shadow.py:119-176``).

Each check runs in a child process, so the reference's modules and the registry patch never
enter the test session's own interpreter.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _reference_src() -> Path | None:
    base = os.environ.get("KRR_REFERENCE")
    tree = Path(base) if base else ROOT.parent / "reference"
    src = tree / "src"
    return src if (src / "kerrray" / "raytracing" / "backends" / "base.py").is_file() else None


REF = _reference_src()
pytestmark = pytest.mark.skipif(REF is None, reason="the KerrRay reference tree is not present")


def _run(script: str, tmp_path: Path) -> dict:
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([str(REF), str(ROOT)]), PYTHONDONTWRITEBYTECODE="1",
               NUMBA_CACHE_DIR=str(tmp_path / "numba"), CUDA_VISIBLE_DEVICES="")
    proc = subprocess.run([sys.executable, "-c", textwrap.dedent(script)], env=env, cwd=str(tmp_path),
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-4000:]
    return json.loads(proc.stdout.strip().splitlines()[-1])


def test_kerrray_registry_returns_this_backend_for_cuda(tmp_path: Path) -> None:
    out = _run("""
        import json
        import numpy as np
        import kerrray.raytracing.rays as rays          # binds get_backend before registration
        from kerrray.raytracing.backends import base
        from kerrray.geodesics import IntegratorOptions, TerminationOptions
        from kerrray.geometry import Spacetime
        import kerrray_b200 as K

        out = {"before": base.available_backends()["cuda"]}
        try:
            base.get_backend("cuda")
        except base.BackendUnavailable as exc:
            out["before_msg"] = str(exc)
        out["registered"] = K.register_with_kerrray()
        out["again"] = K.register_with_kerrray()          # idempotent
        out["after"] = base.available_backends()
        try:
            base.get_backend("cuda")
            out["get"] = "returned"
        except base.BackendUnavailable as exc:            # KerrRay's own exception class
            out["get"] = "BackendUnavailable: " + str(exc)
        try:
            rays.trace_rays(Spacetime(1.0, 0.9), np.zeros((1, 8)), IntegratorOptions(), TerminationOptions(),
                            backend="cuda")
            out["trace"] = "returned"
        except base.BackendUnavailable as exc:
            out["trace"] = "BackendUnavailable: " + str(exc)
        out["numpy"] = type(base.get_backend("numpy")).__name__
        print(json.dumps(out))
    """, tmp_path)
    assert out["before"] is False and "D-007" in out["before_msg"]
    assert out["registered"] is True and out["again"] is True
    assert out["after"] == {"numpy": True, "numba": True, "cuda": False}
    for key in ("get", "trace"):
        assert out[key].startswith("BackendUnavailable: backend 'cuda' is unavailable"), out[key]
        assert "D-007" not in out[key]
    assert out["numpy"] == "NumpyBackend"


def test_kerrray_compute_shadow_drives_the_registered_backend(tmp_path: Path) -> None:
    """KerrRay's compute_shadow(backend="cuda") through the patched registry, with the device
    replaced by the oracle behind CudaBackend's interface; the repo's and the reference's
    ShadowImage files load in each other."""
    out = _run("""
        import json
        import numpy as np
        from kerrray.raytracing.backends import base
        import kerrray_b200 as K
        import kerrray_b200.backends as KB
        from oracle import oracle as O

        calls = []

        class OracleStandIn:
            name = "cuda"

            def __init__(self, precision="fast64", device=0):
                pass

            def integrate_batch(self, st, Y0, integ, term, events=None):
                y0 = np.asarray(Y0, dtype=np.float64)
                calls.append(len(y0))
                r = O.integrate(st.mass, st.spin, y0, O.Options(rtol=integ.rtol, atol=integ.atol))
                return K.BatchResult(Y=r["Y"], state=r["state"], n_steps=r["n_steps"], lam=r["lam"],
                                     max_null_error=r["max_null_error"], max_energy_drift=r["max_energy_drift"],
                                     max_lz_drift=r["max_lz_drift"], max_carter_drift=r["max_carter_drift"],
                                     runtime_s=0.0, n_rejected=r["n_rejected"])

        KB.CudaBackend = OracleStandIn
        assert K.register_with_kerrray()
        from kerrray.raytracing.shadow import ShadowImage as RefImage, compute_shadow
        from kerrray.raytracing.camera import Camera
        from kerrray.geodesics import IntegratorOptions, TerminationOptions
        from kerrray.geometry import Spacetime

        st = Spacetime(1.0, 0.9)
        cam = Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=16)
        integ = IntegratorOptions(method="rk45", rtol=1e-6, atol=1e-8)
        img = compute_shadow(st, cam, integ, TerminationOptions(), backend="cuda")
        ref = compute_shadow(st, cam, integ, TerminationOptions(), backend="numba")
        out = {"calls": calls, "same_mask": bool(np.array_equal(img.state, ref.state)),
               "counts": img.counts}
        # reference-written file -> this package; this package's file -> the reference
        mine = K.ShadowImage.load(img.save("ref_written.npz"))
        out["ref_to_mine"] = bool(np.array_equal(mine.state, img.state) and np.array_equal(mine.result.Y, img.result.Y)
                                  and mine.counts == img.counts and mine.camera.resolution == 16
                                  and np.array_equal(mine.result.n_rejected, img.result.n_rejected))
        own = K.ShadowImage.from_result(K.Spacetime(1.0, 0.9), K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0,
                                                                          resolution=16), mine.result)
        back = RefImage.load(own.save("mine_written.npz"))
        out["mine_to_ref"] = bool(np.array_equal(back.state, img.state) and np.array_equal(back.result.Y, img.result.Y)
                                  and back.counts == img.counts and back.camera.inclination_deg == 60.0
                                  and back.result.event_Y is None and np.array_equal(back.alpha, img.alpha))
        with np.load("ref_written.npz") as a, np.load("mine_written.npz") as b:
            out["same_keys"] = sorted(a.files) == sorted(b.files)
        print(json.dumps(out))
    """, tmp_path)
    assert out["calls"] == [256], out["calls"]  # one call for the whole image through the patched name
    assert out["same_mask"], "the oracle stand-in and KerrRay's numba backend disagree on the 16x16 mask"
    assert out["counts"]["CAPTURED"] > 0 and out["counts"]["ESCAPED"] > 0
    assert out["ref_to_mine"] and out["mine_to_ref"] and out["same_keys"]
