"""The oracle of the per-ray hot path (TEST INFRASTRUCTURE ONLY).

Python side of the CPU restatement in ``krr_oracle.cpp``. Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it,
as the checker; the product (``kerrray_b200``) never does.

* :func:`integrate` restates ``integrate_batch_numba``
  (``src/kerrray/raytracing/backends/numba_backend.py:131-207``): it validates
  ``Y0``, computes the per-ray conservation references with NumPy exactly like
  ``numba_backend.py:174-178`` (``photons/constants.py:65-90, 163-171``) and runs
  the C++ kernel restatement over the rays with OpenMP.
* :func:`initial_states` restates the camera (``raytracing/camera.py:206-381``)
  in NumPy, including the ZAMO tetrad and the cancellation-free ``p_t``
  re-normalisation.
* :func:`count_flops` runs the counting build on a sample of rays and returns
  the operation tallies per phase (initialisation, step attempt, accepted step).

Pinned against the golden fixtures in ``tests/golden`` (made by the reference's
own ``numba`` backend) by ``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

STATE_SIZE = 8
SAFETY, FACTOR_MAX = 0.9, 5.0


class _Params(ctypes.Structure):
    _fields_ = [
        ("mass", ctypes.c_double), ("a", ctypes.c_double),
        ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("step_size", ctypes.c_double),
        ("lambda_max", ctypes.c_double), ("h_min", ctypes.c_double), ("h_max", ctypes.c_double),
        ("max_steps", ctypes.c_int64), ("max_attempts", ctypes.c_int64),
        ("horizon_epsilon", ctypes.c_double), ("escape_radius", ctypes.c_double),
        ("method", ctypes.c_int32), ("dtype", ctypes.c_int32), ("disk", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("r_in", ctypes.c_double), ("r_out", ctypes.c_double),
    ]


_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load (building first if needed) the oracle library."""
    global _LIB
    if _LIB is None:
        from oracle.build import build

        path = build()
        _LIB = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int64)
        _LIB.krr_oracle_integrate.restype = ctypes.c_int
        _LIB.krr_oracle_integrate.argtypes = [ctypes.POINTER(_Params), dp, ctypes.c_int64, dp, dp, dp, dp, dp, dp, dp,
                                              dp, ip, ip, ip, dp, dp, dp, dp, dp, dp,
                                              ctypes.POINTER(ctypes.c_uint8), ctypes.c_int]
        _LIB.krr_oracle_metric_terms.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
        _LIB.krr_oracle_rhs.argtypes = [ctypes.c_double, ctypes.c_double, dp, dp]
        _LIB.krr_oracle_count_flops.restype = ctypes.c_int
        _LIB.krr_oracle_count_flops.argtypes = [ctypes.POINTER(_Params), dp, ctypes.c_int64, dp, dp, dp, dp, dp, dp, dp,
                                                ip, ip, ip, ip]
    return _LIB


def _p(arr: np.ndarray | None, ctype=ctypes.c_double):
    if arr is None:
        return ctypes.cast(None, ctypes.POINTER(ctype))
    return arr.ctypes.data_as(ctypes.POINTER(ctype))


def max_attempts(rtol_unused: float, step_size: float, lambda_max: float, h_min: float, max_steps: int) -> int:
    """``src/kerrray/geodesics/integrators.py:151-162``: the defensive attempt guard."""
    h_max = max(lambda_max, step_size)
    rej = (math.log(h_max / h_min) + max_steps * math.log(FACTOR_MAX)) / math.log(1.0 / SAFETY)
    return max_steps + int(math.ceil(rej)) + 1


@dataclass(frozen=True)
class Options:
    """The fields of ``IntegratorOptions``/``TerminationOptions``/``EventOptions`` the kernel reads."""

    method: str = "rk45"
    rtol: float = 1e-9
    atol: float = 1e-11
    step_size: float = 0.01
    max_steps: int = 100_000
    lambda_max: float = 1.0e4
    h_min: float = 1e-12
    h_max: float | None = None
    dtype: str = "float64"
    horizon_epsilon: float = 1e-6
    escape_radius: float = 1000.0
    disk_plane: bool = False
    r_in: float = 6.0
    r_out: float = 20.0


def _params(mass: float, spin: float, o: Options) -> _Params:
    if o.method not in ("rk45", "rk4"):
        raise ValueError(f"unsupported method {o.method!r}")
    return _Params(
        mass=mass, a=spin * mass, rtol=o.rtol, atol=o.atol, step_size=o.step_size, lambda_max=o.lambda_max,
        h_min=o.h_min, h_max=math.inf if o.h_max is None else o.h_max, max_steps=o.max_steps,
        max_attempts=max_attempts(o.rtol, o.step_size, o.lambda_max, o.h_min, o.max_steps),
        horizon_epsilon=o.horizon_epsilon, escape_radius=o.escape_radius, method=0 if o.method == "rk45" else 1,
        dtype=1 if o.dtype == "float32" else 0, disk=int(o.disk_plane), pad=0, r_in=o.r_in, r_out=o.r_out,
    )


def conservation_refs(mass: float, spin: float, y0: np.ndarray) -> tuple[np.ndarray, ...]:
    """``(e0, lz0, q0, fe, fl, fq, fe2)`` as ``numba_backend.py:174-178`` computes them."""
    a = spin * mass
    e0 = np.ascontiguousarray(-y0[:, 4], dtype=np.float64)
    lz0 = np.ascontiguousarray(y0[:, 7], dtype=np.float64)
    th, p_th, lz, e = y0[:, 2], y0[:, 6], y0[:, 7], -y0[:, 4]
    s2 = np.sin(th) ** 2
    lz2_over_s2 = np.divide(lz * lz, s2, out=np.zeros_like(lz), where=lz != 0)
    q0 = np.ascontiguousarray(p_th * p_th + np.cos(th) ** 2 * (lz2_over_s2 - a**2 * e * e), dtype=np.float64)
    fe = np.abs(e0)
    fe = np.where(fe > 0.0, fe, 1.0)
    fl, fq = fe * mass, fe * fe * mass * mass
    return e0, lz0, q0, np.ascontiguousarray(fe), np.ascontiguousarray(fl), np.ascontiguousarray(fq), np.ascontiguousarray(fe**2)


def integrate(mass: float, spin: float, Y0: np.ndarray, opts: Options, threads: int = 0) -> dict[str, np.ndarray]:
    """Integrate the rays ``Y0`` (N, 8); returns the ``BatchResult`` fields as a dict."""
    y0 = np.array(Y0, dtype=np.float64)
    if y0.ndim != 2 or y0.shape[1] != STATE_SIZE:
        raise ValueError(f"Y0 must have shape (N, {STATE_SIZE}), got {y0.shape}")
    if not np.all(np.isfinite(y0)):
        raise ValueError("Y0 must be finite")
    y0 = np.ascontiguousarray(y0)
    if opts.dtype == "float32":  # numba_backend.py:167: the kernel reads Y0 cast to the working dtype
        y_in = np.ascontiguousarray(y0.astype(np.float32).astype(np.float64))
    else:
        y_in = y0
    n = y0.shape[0]
    refs = conservation_refs(mass, spin, y0)
    out = {
        "Y": np.zeros((n, 8)), "state": np.zeros(n, np.int64), "n_steps": np.zeros(n, np.int64),
        "n_rejected": np.zeros(n, np.int64), "lam": np.zeros(n), "max_null_error": np.zeros(n),
        "max_energy_drift": np.zeros(n), "max_lz_drift": np.zeros(n), "max_carter_drift": np.zeros(n),
    }
    ev_y = np.zeros((n, 8)) if opts.disk_plane else None
    ev_hit = np.zeros(n, np.uint8) if opts.disk_plane else None
    p = _params(mass, spin, opts)
    rc = lib().krr_oracle_integrate(
        ctypes.byref(p), _p(y_in), n, *(_p(r) for r in refs), _p(out["Y"]), _p(out["state"], ctypes.c_int64),
        _p(out["n_steps"], ctypes.c_int64), _p(out["n_rejected"], ctypes.c_int64), _p(out["lam"]),
        _p(out["max_null_error"]), _p(out["max_energy_drift"]), _p(out["max_lz_drift"]), _p(out["max_carter_drift"]),
        _p(ev_y), _p(ev_hit, ctypes.c_uint8), int(threads),
    )
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    if opts.dtype == "float32":
        out["Y"] = out["Y"].astype(np.float32)
    if opts.disk_plane:
        out["event_Y"] = ev_y.astype(np.float32) if opts.dtype == "float32" else ev_y
        out["event_hit"] = ev_hit.astype(bool)
    return out


def metric_terms(mass: float, spin: float, r: float, th: float) -> np.ndarray:
    out = np.zeros(15)
    lib().krr_oracle_metric_terms(mass, spin * mass, r, th, _p(out))
    return out


def rhs(mass: float, spin: float, y: np.ndarray) -> np.ndarray:
    y8 = np.ascontiguousarray(y, dtype=np.float64)
    f = np.zeros(8)
    lib().krr_oracle_rhs(mass, spin * mass, _p(y8), _p(f))
    return f


def count_flops(mass: float, spin: float, Y0: np.ndarray, opts: Options) -> dict[str, object]:
    """Operation tallies of the float64 reference algorithm on the rays ``Y0``.

    Returns ``{"init": {...}, "attempt": {...}, "accept": {...}, "attempts": int,
    "accepted": int, "rays": int}`` where each phase dict holds counts of add, mul,
    div, sqrt, trig and pow operations summed over the rays.
    """
    y0 = np.ascontiguousarray(np.asarray(Y0, dtype=np.float64))
    n = y0.shape[0]
    refs = conservation_refs(mass, spin, y0)
    state = np.zeros(n, np.int64)
    steps = np.zeros(n, np.int64)
    rej = np.zeros(n, np.int64)
    counts = np.zeros(18, np.int64)
    p = _params(mass, spin, Options(**{**opts.__dict__, "dtype": "float64"}))
    rc = lib().krr_oracle_count_flops(ctypes.byref(p), _p(y0), n, *(_p(r) for r in refs),
                                      _p(state, ctypes.c_int64), _p(steps, ctypes.c_int64),
                                      _p(rej, ctypes.c_int64), _p(counts, ctypes.c_int64))
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    names = ("add", "mul", "div", "sqrt", "trig", "pow")
    phases = {ph: dict(zip(names, counts[6 * i: 6 * i + 6].tolist())) for i, ph in enumerate(("init", "attempt", "accept"))}
    return {**phases, "attempts": int(steps.sum() + rej.sum()), "accepted": int(steps.sum()), "rays": n,
            "state": state, "n_steps": steps, "n_rejected": rej}


# ------------------------------------------------------------------------------------------
# Camera (raytracing/camera.py:206-381), NumPy restatement.
# ------------------------------------------------------------------------------------------

def pixel_coordinates(fov: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """``camera.py:206-222``: pixel-centre (alpha, beta), shape (n, n), row 0 on top."""
    centres = fov * (2.0 * np.arange(n, dtype=np.float64) + 1.0 - n) / n
    return np.meshgrid(centres, -centres)


def clamp_inclination(inclination_deg: float) -> float:
    """``camera.py:155-165``: inclination clamped into [1e-3, 180 - 1e-3] degrees."""
    low, high = 1e-3, 180.0 - 1e-3
    return min(max(float(inclination_deg), low), high)


def initial_states(mass: float, spin: float, r_o: float, inclination_deg: float, phi_deg: float,
                   alpha: np.ndarray, beta: np.ndarray) -> np.ndarray:
    """Backward null photon states ``(N, 8)`` at the ZAMO observer for image points (alpha, beta)."""
    a = spin * mass
    m = mass
    th_o = math.radians(clamp_inclination(inclination_deg))
    ph_o = math.radians(phi_deg)
    alpha = np.asarray(alpha, dtype=np.float64).ravel()
    beta = np.asarray(beta, dtype=np.float64).ravel()
    rho2 = (alpha**2 + beta**2) / r_o**2
    r_, th = np.float64(r_o), np.float64(th_o)
    # metric_components (geometry/metric.py:147-163)
    s2 = np.sin(th) ** 2
    sig = r_**2 + a**2 * np.cos(th) ** 2
    dlt = r_**2 - 2.0 * m * r_ + a**2
    g_tt = -(1.0 - 2.0 * m * r_ / sig)
    g_tphi = -2.0 * m * a * r_ * s2 / sig
    g_rr = sig / dlt
    g_thth = sig + 0.0 * dlt
    g_phph = (r_**2 + a**2 + 2.0 * m * a**2 * r_ * s2 / sig) * s2
    # zamo_tetrad (camera.py:225-262)
    omega = -g_tphi / g_phph
    lapse = np.sqrt(-(g_tt - g_tphi**2 / g_phph))
    e = np.zeros((4, 4))
    e[0, 0] = 1.0 / lapse
    e[0, 3] = omega / lapse
    e[1, 1] = 1.0 / np.sqrt(g_rr)
    e[2, 2] = 1.0 / np.sqrt(g_thth)
    e[3, 3] = 1.0 / np.sqrt(g_phph)
    n = alpha.size
    p_local = np.empty((n, 4))
    p_local[:, 0] = 1.0
    p_local[:, 1] = np.sqrt(1.0 - rho2)
    p_local[:, 2] = beta / r_o
    p_local[:, 3] = -alpha / r_o
    p_up = p_local @ e
    g = np.zeros((4, 4))
    g[0, 0], g[0, 3], g[3, 0], g[1, 1], g[2, 2], g[3, 3] = g_tt, g_tphi, g_tphi, g_rr, g_thth, g_phph
    p_dn = -(p_up @ g)
    # inverse_metric_components (metric.py:166-195) and _null_pt (camera.py:265-295)
    big_a = (r_**2 + a**2) ** 2 - a**2 * dlt * s2
    sd = sig * dlt
    gtt = -big_a / sd
    gtphi = -2.0 * m * a * r_ / sd
    grr = dlt / sig
    gthth = 1.0 / sig + 0.0 * dlt
    gphph = (dlt - a**2 * s2) / (sd * s2)
    p_t, p_r, p_th, p_ph = (p_dn[:, k] for k in range(4))
    qa = np.broadcast_to(np.asarray(gtt), p_t.shape)
    qb = 2.0 * gtphi * p_ph
    qc = grr * p_r**2 + gthth * p_th**2 + gphph * p_ph**2
    disc = qb * qb - 4.0 * qa * qc
    q = -0.5 * (qb + np.copysign(np.sqrt(np.maximum(disc, 0.0)), qb))
    root_1 = q / qa
    root_2 = np.divide(qc, q, out=root_1.copy(), where=q != 0.0)
    p_dn[:, 0] = np.where(np.abs(root_1 - p_t) <= np.abs(root_2 - p_t), root_1, root_2)
    y = np.empty((n, 8))
    y[:, 0] = 0.0
    y[:, 1] = r_o
    y[:, 2] = th_o
    y[:, 3] = ph_o
    y[:, 4:8] = p_dn
    return y
