"""CPU-only checks of the C ABI and the host logic (no kernel launches).

The library must build for sm_100a, load, export every entry point ``include/kerrray_cuda.h``
declares, and reject invalid arguments with the reference's exception types before touching
a device (``geodesics/integrators.py:98-129``, ``raytracing/camera.py:131-168``,
``raytracing/backends/numba_backend.py:78-84, 157-158``).
"""

from __future__ import annotations

import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, TRACE_FIXTURES, golden
from kerrray_b200 import _lib
from kerrray_b200.build import build
import kerrray_b200 as K


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


def test_library_exports_every_declared_symbol() -> None:
    header = (ROOT / "include" / "kerrray_cuda.h").read_text()
    declared = set(re.findall(r"KRR_API\s+[\w\s\*]+?\b(krr_\w+)\s*\(", header))
    assert declared == set(_lib.EXPORTS)
    lib = _lib.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.krr_abi_version() == 6


def test_library_is_built_for_sm_100a() -> None:
    data = (ROOT / "kerrray_b200" / "libkerrray_cuda.so").read_bytes()
    assert b"sm_100a" in data


@pytest.mark.parametrize("name", TRACE_FIXTURES)
def test_max_attempts_matches_reference(name: str) -> None:
    d = golden(name)
    o = _lib.KrrOptions(method=0 if str(d["integ_method"]) == "rk45" else 1, dtype=0, rtol=float(d["integ_rtol"]),
                        atol=float(d["integ_atol"]), step_size=float(d["integ_step_size"]),
                        lambda_max=float(d["integ_lambda_max"]), h_min=float(d["integ_h_min"]),
                        h_max=float(d["integ_h_max"]), max_steps=int(d["integ_max_steps"]),
                        horizon_epsilon=1e-6, escape_radius=1000.0)
    out = ctypes.c_int64()
    assert _lib.lib().krr_max_attempts(ctypes.byref(o), ctypes.byref(out)) == 0
    assert out.value == int(d["integ_max_attempts"])
    integ = K.IntegratorOptions(method=str(d["integ_method"]), rtol=float(d["integ_rtol"]), atol=float(d["integ_atol"]),
                                step_size=float(d["integ_step_size"]), max_steps=int(d["integ_max_steps"]),
                                lambda_max=float(d["integ_lambda_max"]), h_min=float(d["integ_h_min"]))
    assert K.max_attempts(integ) == int(d["integ_max_attempts"])


def _opts(**kw) -> _lib.KrrOptions:
    base = dict(method=0, dtype=0, rtol=1e-6, atol=1e-8, step_size=0.01, lambda_max=1e4, h_min=1e-12, h_max=math.inf,
                max_steps=100000, horizon_epsilon=1e-6, escape_radius=1000.0, disk_plane=0, reserved=0, r_in=0, r_out=0)
    base.update(kw)
    return _lib.KrrOptions(**base)


@pytest.mark.parametrize("bad", [dict(rtol=0.0), dict(atol=-1.0), dict(step_size=math.nan), dict(h_min=math.inf),
                                 dict(h_max=0.0), dict(max_steps=0), dict(method=7), dict(dtype=3),
                                 dict(horizon_epsilon=-1.0), dict(escape_radius=0.0),
                                 dict(disk_plane=1, r_in=5.0, r_out=1.0)])
def test_invalid_options_rejected_before_any_device_work(bad: dict) -> None:
    y0 = np.ones((1, 8))
    r = _lib.KrrResult()
    rc = _lib.lib().krr_integrate_batch(0, 1.0, 0.5, y0.ctypes.data, 1, ctypes.byref(_opts(**bad)), 0, ctypes.byref(r), None)
    assert rc == _lib.KRR_ERR_INVALID
    assert _lib.last_error()


def test_invalid_spacetime_and_nonfinite_input_rejected() -> None:
    y0 = np.ones((2, 8))
    out = {"Y": np.empty((2, 8)), "state": np.empty(2, np.int64)}
    r = _lib.result_struct(out)
    L = _lib.lib()
    assert L.krr_integrate_batch(0, 1.0, 1.0, y0.ctypes.data, 2, ctypes.byref(_opts()), 0, ctypes.byref(r), None) == 1
    assert L.krr_integrate_batch(0, -1.0, 0.5, y0.ctypes.data, 2, ctypes.byref(_opts()), 0, ctypes.byref(r), None) == 1
    y0[1, 3] = np.inf
    assert L.krr_integrate_batch(0, 1.0, 0.5, y0.ctypes.data, 2, ctypes.byref(_opts()), 0, ctypes.byref(r), None) == 1
    assert "finite" in _lib.last_error()
    # float32 runs in the reference precision only; mixed integrates rk45 only.
    assert L.krr_integrate_batch(0, 1.0, 0.5, y0.ctypes.data, 0, ctypes.byref(_opts(dtype=1)), 1, ctypes.byref(r), None) == 5
    assert L.krr_integrate_batch(0, 1.0, 0.5, y0.ctypes.data, 0, ctypes.byref(_opts(method=1)), 2, ctypes.byref(r), None) == 5


def test_camera_validation_matches_reference() -> None:
    with pytest.raises(ValueError):
        K.Camera(radius=1000.0, inclination_deg=60.0, resolution=3)
    with pytest.raises(ValueError):
        K.Camera(radius=-1.0, inclination_deg=60.0)
    with pytest.raises(ValueError):
        K.Camera(radius=1000.0, inclination_deg=181.0)
    assert K.Camera(radius=1000.0, inclination_deg=0.0).inclination_deg == 1e-3
    d = golden("camera_states")
    for k in range(int(d["n_cameras"])):
        cam = K.Camera(radius=float(d[f"c{k}_camera_radius"]), inclination_deg=float(d[f"c{k}_camera_inclination_deg"]),
                       phi_deg=float(d[f"c{k}_camera_phi_deg"]), fov=float(d[f"c{k}_camera_fov"]),
                       resolution=int(d[f"c{k}_camera_resolution"]))
        a, b = cam.pixel_coordinates()
        assert np.array_equal(a, d[f"c{k}_alpha"]) and np.array_equal(b, d[f"c{k}_beta"])
    # Grid checks happen on the host before any device work.
    L = _lib.lib()
    y = np.empty((4, 8))
    inside = _lib.KrrCamera(radius=1.2, inclination_deg=60.0, phi_deg=0.0, fov=0.5, resolution=2)
    assert L.krr_camera_states(0, 1.0, 0.9, ctypes.byref(inside), None, None, 0, y.ctypes.data) == 1
    wide = _lib.KrrCamera(radius=10.0, inclination_deg=60.0, phi_deg=0.0, fov=20.0, resolution=2)
    assert L.krr_camera_states(0, 1.0, 0.9, ctypes.byref(wide), None, None, 0, y.ctypes.data) == 1


def test_options_validation_mirrors_reference() -> None:
    with pytest.raises(ValueError):
        K.IntegratorOptions(method="euler")
    with pytest.raises(ValueError):
        K.IntegratorOptions(h_max=0.0)
    with pytest.raises(ValueError):
        K.TerminationOptions(horizon_epsilon=-1.0)
    with pytest.raises(ValueError):
        K.EventOptions(r_in=5.0, r_out=1.0)
    with pytest.raises(ValueError):
        K.Spacetime(1.0, 1.0)
    with pytest.raises(ValueError):
        _lib.options_struct(K.IntegratorOptions(method="dop853"), K.TerminationOptions())


def test_backend_unavailable_without_a_device() -> None:
    if _lib.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(K.BackendUnavailable):
        K.CudaBackend()
    with pytest.raises(K.BackendUnavailable):
        K.get_backend("cuda")
    assert K.available_backends()["cuda"] is False
    with pytest.raises(ValueError):
        K.get_backend("opencl")


def test_shadow_npz_round_trip(tmp_path: Path) -> None:
    d = golden("shadow64_a0.9_i60")
    cam = K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64)
    res = K.BatchResult(Y=d["Y"], state=d["state"].astype(np.int64), n_steps=d["n_steps"].astype(np.int64),
                        lam=d["lam"], max_null_error=d["max_null_error"], max_energy_drift=d["max_energy_drift"],
                        max_lz_drift=d["max_lz_drift"], max_carter_drift=d["max_carter_drift"], runtime_s=0.1,
                        n_rejected=d["n_rejected"].astype(np.int64))
    from kerrray_b200.shadow import ShadowImage

    img = ShadowImage.from_result(K.Spacetime(1.0, 0.9), cam, res)
    assert img.count(K.TerminationState.CAPTURED) == 1250 and img.n_failed == 0 and img.n_other == 0
    path = img.save(tmp_path / "s.npz")
    back = K.ShadowImage.load(path)
    assert np.array_equal(back.state, img.state) and np.array_equal(back.result.Y, img.result.Y)
    assert back.camera == cam
    mask = K.shadow_mask_int8(img.state)
    assert mask.dtype == np.int8 and int((mask == 1).sum()) == 1250


def test_batched_trace_writes_the_reference_npz(tmp_path: Path) -> None:
    """Image k of a batched trace (SweepResult rows) as the reference's ShadowImage file."""
    from kerrray_b200.sweep import SweepResult

    d = golden("shadow64_a0.9_i60")
    st = K.Spacetime(1.0, 0.9)
    small = K.ImageSpec(st, K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=2),
                        K.IntegratorOptions(), K.TerminationOptions())
    big = K.ImageSpec(st, K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=64),
                      K.IntegratorOptions(rtol=1e-6, atol=1e-8), K.TerminationOptions())
    def rows(key, dtype=None):
        x = np.asarray(d[key]) if dtype is None else np.asarray(d[key]).astype(dtype)
        return np.concatenate([x[:4], x])
    arrays = {"Y": rows("Y"), "state": rows("state", np.int64), "n_steps": rows("n_steps", np.int64),
              "n_rejected": rows("n_rejected", np.int64), "lam": rows("lam"), "max_null_error": rows("max_null_error"),
              "max_energy_drift": rows("max_energy_drift"), "max_lz_drift": rows("max_lz_drift"),
              "max_carter_drift": rows("max_carter_drift"), "event_Y": None, "event_hit": None}
    sw = SweepResult(specs=[small, big], offsets=np.array([0, 4, 4 + 4096]), arrays=arrays, stats={})
    back = K.ShadowImage.load(sw.shadow_image(1).save(tmp_path / "img1.npz"))
    assert np.array_equal(back.state.ravel(), np.asarray(d["state"]).astype(np.int64))
    assert back.camera == big.camera and back.count(K.TerminationState.CAPTURED) == 1250
    assert sw.shadow_image(0).state.shape == (2, 2)



def test_lensing_workspace_sizes() -> None:
    """The lensing workspace: the minimum holds no stage pool; the staged size adds whole
    chunks (16 steps x 240 B) for the requested steps plus one chunk of rounding per ray."""
    from kerrray_b200 import adjoint as A

    L = A._bind()
    n, cap, k = 1000, 4096, 32
    base = L.krr_lensing_workspace_size(n, cap, k)
    assert base > n * cap * 8 and base % 256 == 0
    assert L.krr_lensing_workspace_size_staged(n, cap, k, 0) == base
    chunk = 16 * 6 * 5 * 8
    for steps in (1, 16, 17, 320_000):
        extra = L.krr_lensing_workspace_size_staged(n, cap, k, steps) - base
        assert extra == (-(-steps // 16) + n) * chunk, steps
    assert L.krr_lensing_workspace_size_staged(n, cap, k, -1) == 0
    assert L.krr_lensing_workspace_size_staged(-1, cap, k, 10) == 0


def test_lensing_trace_order_permutations() -> None:
    """The orders the lensing map can trace its rays in (host logic, no device): by increasing
    impact parameter, by decreasing per-ray cost, or as given; un-permuting restores the rows."""
    torch = pytest.importorskip("torch")
    from kerrray_b200 import adjoint as A

    alpha = torch.tensor([3.0, -0.5, 2.0, 0.0, -4.0], dtype=torch.float64)
    beta = torch.tensor([0.0, 0.5, -2.0, 1.0, 0.0], dtype=torch.float64)
    assert A._trace_order("given", alpha, beta) is None
    imp = A._trace_order("impact", alpha, beta)
    assert imp.tolist() == [1, 3, 2, 0, 4]  # hypot 0.71, 1, 2.83, 3, 4
    cost = torch.tensor([10, 300, 20, 300, 5])
    by_cost = A._trace_order(cost, alpha, beta)
    assert by_cost.tolist() == [1, 3, 2, 0, 4]  # decreasing cost, ties in input order
    rows = torch.arange(5.0) * 10
    traced = rows[by_cost]
    assert torch.equal(A._unpermute(traced, by_cost), rows)
    jac = torch.arange(40.0).reshape(5, 2, 4)
    assert torch.equal(A._unpermute(jac[imp], imp), jac)
    with pytest.raises(ValueError):
        A._trace_order("sideways", alpha, beta)
    with pytest.raises(ValueError):
        A._trace_order(torch.ones(4), alpha, beta)


def test_lensing_entry_points_validate_before_device_work() -> None:
    """krr_lensing_adjoint and krr_lensing_tape_usage reject bad arguments with KRR_ERR_INVALID /
    KRR_ERR_UNSUPPORTED before any device call (the buffer addresses below are never read)."""
    from kerrray_b200 import adjoint as A

    L = A._bind()  # the package's own argument types
    n = 1000
    p = A._params(0.8, 60.0, 1000.0, 1.0, None, None, 32, 4096)
    need = L.krr_lensing_workspace_size(n, 4096, 32)
    fake = [0x10000 * (k + 1) for k in range(6)]  # device addresses of the outputs, never dereferenced

    def call(params, ws, ws_bytes, bufs=fake, a=0x100000, b=0x200000):
        return L.krr_lensing_adjoint(0, ctypes.byref(params), a, b, n, *bufs, ws, ws_bytes, None)

    assert call(p, 0x400000, need - 256) == _lib.KRR_ERR_INVALID        # workspace too small
    assert call(p, 0x400008, need) == _lib.KRR_ERR_INVALID              # not 256-byte aligned
    assert "256-byte aligned" in _lib.lib().krr_last_error().decode()
    assert call(p, 0x400000, need, bufs=[0] + fake[1:]) == _lib.KRR_ERR_INVALID  # a NULL output
    bad = A.KrrLensParams.from_buffer_copy(p)
    bad.checkpoint_every = 0
    assert call(bad, 0x400000, need) == _lib.KRR_ERR_INVALID
    rk4 = A._params(0.8, 60.0, 1000.0, 1.0, K.IntegratorOptions(method="rk4"), None, 32, 4096)
    assert call(rk4, 0x400000, need) == _lib.KRR_ERR_UNSUPPORTED
    import torch

    if not torch.cuda.is_available():  # valid arguments reach the device check and stop there
        assert call(p, 0x400000, need) == _lib.KRR_ERR_NO_DEVICE
    # the usage query: outputs required; no rays, no device work
    out = [ctypes.c_int64() for _ in range(3)]
    assert L.krr_lensing_tape_usage(ctypes.byref(p), n, 0x400000, need, None, None, None, None) == _lib.KRR_ERR_INVALID
    empty = L.krr_lensing_workspace_size_staged(0, 4096, 32, 0)
    assert L.krr_lensing_tape_usage(ctypes.byref(p), 0, 0x400000, empty + 3840 * 5, *[ctypes.byref(o) for o in out],
                                    None) == _lib.KRR_OK
    assert out[0].value == 0 and out[1].value == 0 and out[2].value == 5
