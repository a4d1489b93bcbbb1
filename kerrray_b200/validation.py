"""The exact checks of the hot path, driven through any backend (default: the cuda backend).

KerrRay's own drivers call its NumPy integrator directly; these restate them with a backend
argument:

* :func:`photon_from_constants`, :func:`tangential_photon` -- photon states from
  ``(E, L_z, Q)`` (``src/kerrray/geodesics/initial_conditions.py:83-172``, Carter 1968 potentials);
* :func:`photon_sphere` -- bracketing of the unstable circular photon orbit with tangential
  launches (``src/kerrray/validation/schwarzschild.py:151-200``): captured below, escaped
  above, ``n_probe`` interior probes per iteration;
* :func:`critical_impacts` -- bracketing of the capture threshold in impact parameter for
  inward equatorial rays (``src/kerrray/validation/kerr_bisection.py:96-263``), prograde and
  retrograde searches sharing one batch per iteration;
* :func:`winding_rate_prediction`, :func:`winding_rates` -- the near-critical winding study
  (``scripts/study_winding.py:73-127``): turns of equatorial photons launched at
  ``b = b_c (1 + delta)`` against ``log10(delta)``, compared with the orbit's instability rate
  ``ln(10) / (2 pi gamma_phi)``; all deltas and both directions of one spin in one batch.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from kerrray_b200.types import Spacetime, TerminationState, outer_horizon

__all__ = ["CRITICAL_IMPACT_REFERENCE", "PHOTON_SPHERE_REFERENCE", "WINDING_DELTAS", "WINDING_SPINS", "critical_impacts",
           "equatorial_photon", "photon_from_constants", "photon_sphere", "tangential_photon", "winding_rate_prediction",
           "winding_rates"]

PHOTON_SPHERE_REFERENCE = 3.0                   # r_ph = 3M (a = 0)
CRITICAL_IMPACT_REFERENCE = 3.0 * math.sqrt(3.0)  # b_c = 3 sqrt(3) M (a = 0)
RADICAND_TOLERANCE = 1e-12


def _carter_potentials(st, r, theta, E, Lz, Q):
    a = st.a
    dlt = r * r - 2.0 * st.mass * r + a * a
    term1 = E * (r * r + a * a) - a * Lz
    term2 = dlt * (Q + (Lz - a * E) ** 2)
    c2, s2 = math.cos(theta) ** 2, math.sin(theta) ** 2
    lz_term = 0.0 if Lz == 0.0 else Lz * Lz / s2
    return (term1 * term1 - term2, Q - c2 * (lz_term - a * a * E * E), term1 * term1 + abs(term2),
            abs(Q) + c2 * (lz_term + a * a * E * E), dlt)


def _sqrt_radicand(value: float, scale: float, name: str) -> float:
    if value < -RADICAND_TOLERANCE * max(scale, 1.0):
        raise ValueError(f"{name} = {value!r} < 0: the requested constants of motion are inconsistent here")
    return math.sqrt(max(value, 0.0))


def photon_from_constants(st, r: float, theta: float, E: float, Lz: float, Q: float, *, sign_r: int,
                          sign_theta: int, t: float = 0.0, phi: float = 0.0) -> np.ndarray:
    """State ``[t, r, theta, phi, -E, +-sqrt(R)/Delta, +-sqrt(Theta), L_z]`` of a photon with these constants."""
    if not E > 0.0:
        raise ValueError(f"E must be > 0 for a future-directed photon, got {E!r}")
    if not r > outer_horizon(st):
        raise ValueError(f"r = {r!r} must lie outside the outer horizon r_plus = {outer_horizon(st)!r}")
    if sign_r not in (-1, 1) or sign_theta not in (-1, 1):
        raise ValueError("sign_r and sign_theta must be +1 or -1")
    big_r, big_th, sc_r, sc_th, dlt = _carter_potentials(st, r, theta, E, Lz, Q)
    p_r = sign_r * _sqrt_radicand(big_r, sc_r, "R(r)") / dlt
    p_th = sign_theta * _sqrt_radicand(big_th, sc_th, "Theta(theta)")
    return np.array([t, r, theta, phi, -E, p_r, p_th, Lz], dtype=np.float64)


def _lz_sign(st, prograde: bool) -> float:
    return 1.0 if prograde == (st.a >= 0.0) else -1.0


def equatorial_photon(st, r0: float, b: float, *, inward: bool = True, prograde: bool = True,
                      E: float = 1.0) -> np.ndarray:
    """Equatorial photon at ``r0`` with impact parameter ``b = |L_z| / E``, ``Q = 0``
    (``geodesics/initial_conditions.py:121-141``)."""
    if b < 0.0:
        raise ValueError(f"b must be >= 0, got {b!r}")
    return photon_from_constants(st, r0, 0.5 * math.pi, E, _lz_sign(st, prograde) * b * E, 0.0,
                                 sign_r=-1 if inward else 1, sign_theta=1)


def tangential_photon(st, r0: float, *, prograde: bool = True, E: float = 1.0) -> np.ndarray:
    """Equatorial photon launched tangentially (``p_r = p_theta = 0``) at ``r0``."""
    if not E > 0.0:
        raise ValueError(f"E must be > 0, got {E!r}")
    if not r0 > outer_horizon(st):
        raise ValueError(f"r0 = {r0!r} must lie outside the outer horizon")
    a = st.a
    s = _lz_sign(st, prograde)
    sqrt_delta = math.sqrt(r0 * r0 - 2.0 * st.mass * r0 + a * a)
    denom = a + s * sqrt_delta
    if denom == 0.0:
        raise ValueError("no finite tangential photon: r0 is on the equatorial ergosphere for this direction")
    lz = E * ((r0 * r0 + a * a) + s * a * sqrt_delta) / denom
    return np.array([0.0, r0, 0.5 * math.pi, 0.0, -E, 0.0, 0.0, lz], dtype=np.float64)


def _backend(backend):
    if backend is None:
        from kerrray_b200.backends import CudaBackend

        return CudaBackend(precision="reference")
    return backend


@dataclass
class PhotonSphereResult:
    radius: float
    r_lo: float
    r_hi: float
    width: float
    iterations: int
    n_rays: int
    max_steps: int
    runtime_s: float


def photon_sphere(integ, term, *, r_lo: float, r_hi: float, tol: float, max_iterations: int = 60, n_probe: int = 1,
                  mass: float = 1.0, backend=None) -> PhotonSphereResult:
    """Locate r_ph = 3M by bracketing tangential launches (captured below, escaped above)."""
    if not (0.0 < r_lo < r_hi) or not tol > 0.0 or n_probe < 1 or max_iterations < 1:
        raise ValueError(f"invalid search: r_lo={r_lo}, r_hi={r_hi}, tol={tol}, n_probe={n_probe}")
    st = Spacetime(mass, 0.0)
    engine = _backend(backend)
    t0 = time.perf_counter()
    n_rays = max_steps = iterations = 0

    def classify(radii: np.ndarray) -> np.ndarray:
        nonlocal n_rays, max_steps
        res = engine.integrate_batch(st, np.stack([tangential_photon(st, float(r)) for r in radii]), integ, term)
        n_rays += radii.size
        max_steps = max(max_steps, int(np.max(res.n_steps)))
        ok = (res.state == TerminationState.CAPTURED) | (res.state == TerminationState.ESCAPED)
        if not np.all(ok):
            raise RuntimeError(f"photon sphere: rays ended neither CAPTURED nor ESCAPED: {radii[~ok]}")
        return np.asarray(res.state)

    ends = classify(np.array([r_lo, r_hi]))
    if ends[0] != TerminationState.CAPTURED or ends[1] != TerminationState.ESCAPED:
        raise RuntimeError(f"bracket [{r_lo}, {r_hi}] invalid")
    lo, hi = r_lo, r_hi
    fractions = np.arange(1, n_probe + 1) / (n_probe + 1)
    while hi - lo > tol and iterations < max_iterations:
        radii = lo + (hi - lo) * fractions
        states = classify(radii)
        captured = radii[states == TerminationState.CAPTURED]
        escaped = radii[states == TerminationState.ESCAPED]
        if captured.size and escaped.size and captured.max() > escaped.min():
            raise RuntimeError(f"non-monotone outcome in r0: captured at {captured.max()!r}, escaped at {escaped.min()!r}")
        lo = max(lo, float(captured.max())) if captured.size else lo
        hi = min(hi, float(escaped.min())) if escaped.size else hi
        iterations += 1
    return PhotonSphereResult(0.5 * (lo + hi), lo, hi, hi - lo, iterations, n_rays, max_steps, time.perf_counter() - t0)


@dataclass
class CriticalImpactResult:
    spin: float
    prograde: bool
    b_c: float
    b_lo: float
    b_hi: float
    width: float
    iterations: int
    n_rays: int
    max_steps: int
    runtime_s: float


def critical_impacts(st, integ, term, *, r0: float, b_lo: float, b_hi: float, tol: float, max_iterations: int,
                     n_probe: int = 8, directions: tuple[bool, ...] = (True, False),
                     backend=None) -> tuple[CriticalImpactResult, ...]:
    """Bracket the capture threshold b_c of inward equatorial rays from ``r0`` for each direction."""
    if not (0.0 <= b_lo < b_hi):
        raise ValueError(f"need 0 <= b_lo < b_hi, got {b_lo!r}, {b_hi!r}")
    if not tol > 0.0 or n_probe < 1 or max_iterations < 1:
        raise ValueError("tol, n_probe and max_iterations must be positive")
    engine = _backend(backend)
    t0 = time.perf_counter()
    lo = {p: b_lo for p in directions}
    hi = {p: b_hi for p in directions}
    its = {p: 0 for p in directions}
    n_rays = max_steps = 0

    def probe(bs: np.ndarray, pro: np.ndarray) -> np.ndarray:
        nonlocal n_rays, max_steps
        y0 = np.stack([photon_from_constants(st, r0, 0.5 * math.pi, 1.0, _lz_sign(st, bool(p)) * b, 0.0, sign_r=-1,
                                             sign_theta=1) for b, p in zip(bs, pro)])
        res = engine.integrate_batch(st, y0, integ, term)
        n_rays += bs.size
        max_steps = max(max_steps, int(np.max(res.n_steps)))
        return np.asarray(res.state)

    bs = np.array([b for p in directions for b in (b_lo, b_hi)])
    pro = np.array([p for p in directions for _ in (0, 1)])
    states = probe(bs, pro)
    for k, p in enumerate(directions):
        if states[2 * k] != TerminationState.CAPTURED or states[2 * k + 1] != TerminationState.ESCAPED:
            raise RuntimeError(f"bracket [{b_lo}, {b_hi}] invalid for prograde={p}")
    fractions = np.arange(1, n_probe + 1) / (n_probe + 1)
    while True:
        open_dirs = [p for p in directions if hi[p] - lo[p] > tol and its[p] < max_iterations]
        if not open_dirs:
            break
        bs = np.concatenate([lo[p] + (hi[p] - lo[p]) * fractions for p in open_dirs])
        pro = np.concatenate([np.full(n_probe, p) for p in open_dirs])
        states = probe(bs, pro)
        bad = (states != TerminationState.CAPTURED) & (states != TerminationState.ESCAPED)
        if bad.any():
            raise RuntimeError(f"rays ended neither CAPTURED nor ESCAPED at b = {bs[bad]}")
        for k, p in enumerate(open_dirs):
            sl = slice(k * n_probe, (k + 1) * n_probe)
            cap = bs[sl][states[sl] == TerminationState.CAPTURED]
            esc = bs[sl][states[sl] == TerminationState.ESCAPED]
            if cap.size and esc.size and cap.max() > esc.min():
                raise RuntimeError(f"non-monotone classification in b for prograde={p}")
            if cap.size:
                lo[p] = max(lo[p], float(cap.max()))
            if esc.size:
                hi[p] = min(hi[p], float(esc.min()))
            its[p] += 1
    runtime = time.perf_counter() - t0
    return tuple(CriticalImpactResult(st.spin, p, 0.5 * (lo[p] + hi[p]), lo[p], hi[p], hi[p] - lo[p], its[p], n_rays,
                                      max_steps, runtime) for p in directions)


WINDING_SPINS = (0.0, 0.3, 0.6, 0.9, 0.99)
WINDING_DELTAS = (1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8)


def winding_rate_prediction(spin: float, prograde: bool, mass: float = 1.0) -> float:
    """Turns per decade of ``b / b_c - 1``, ``ln(10) / (2 pi gamma_phi)``, for the circular
    equatorial photon orbit (``study_winding.py:66-83``; Carter 1968, Bardeen, Press & Teukolsky
    1972). With ``E = 1``, ``theta = pi/2`` and signed ``xi = L_z / E`` (positive for prograde at
    ``a >= 0``), ``R(r) = (r^2 + a^2 - a xi)^2 - Delta (xi - a)^2`` and
    ``Phi(r) = (xi - a) + (a / Delta)(r^2 + a^2 - a xi)``; ``gamma_phi = sqrt(R''(r_ph)/2)/|Phi(r_ph)|``.
    ``R''`` is taken in closed form, ``8 r^2 + 4 (r^2 + a^2 - a xi) - 2 (xi - a)^2`` (with
    ``u = r^2 + a^2 - a xi``: ``(u^2)'' = 2 u'^2 + 2 u u''``, ``u' = 2 r``, ``u'' = 2``,
    ``Delta'' = 2``); the study takes it by central differences of ``R``."""
    from kerrray_b200.orbits import critical_impact_parameters, equatorial_photon_orbit_radius

    st = Spacetime(mass, spin)
    a = st.a
    r_ph = equatorial_photon_orbit_radius(st, prograde=prograde)
    b_pro, b_retro = critical_impact_parameters(st)
    xi = b_pro if prograde else -b_retro
    u = r_ph * r_ph + a * a - a * xi
    r2 = 8.0 * r_ph * r_ph + 4.0 * u - 2.0 * (xi - a) ** 2
    delta = r_ph * r_ph - 2.0 * mass * r_ph + a * a
    phi_rate = (xi - a) + a / delta * u
    gamma = math.sqrt(r2 / 2.0) / abs(phi_rate)
    return math.log(10.0) / (2.0 * math.pi * gamma)


@dataclass
class WindingResult:
    spin: float
    prograde: bool
    b_c: float
    turns: np.ndarray          # per delta
    states: np.ndarray         # termination codes per delta
    rate_per_decade: float     # -slope of turns against log10(delta) over the escaped rays
    predicted: float
    relative_difference: float


def winding_rates(spins=WINDING_SPINS, deltas=WINDING_DELTAS, *, rtol: float = 1e-12, r0: float = 50.0,
                  escape_radius: float = 60.0, max_steps: int = 400_000, backend=None) -> list[WindingResult]:
    """Measured against predicted winding rates (``study_winding.py:86-99``, ``:108-114``): the
    nine cases of the study by default (spin 0 has one direction), ``rk45`` at ``rtol`` with
    ``atol = 1e-2 rtol``, launch radius 50 M, escape radius 60 M, horizon margin 1e-6."""
    from kerrray_b200.orbits import critical_impact_parameters
    from kerrray_b200.types import IntegratorOptions, TerminationOptions

    engine = _backend(backend)
    integ = IntegratorOptions(method="rk45", rtol=rtol, atol=rtol * 1e-2, max_steps=max_steps)
    term = TerminationOptions(horizon_epsilon=1e-6, escape_radius=escape_radius)
    deltas = np.asarray(deltas, dtype=np.float64)
    out = []
    for spin in spins:
        st = Spacetime(1.0, spin)
        directions = (True,) if spin == 0.0 else (True, False)
        b_pro, b_retro = critical_impact_parameters(st)
        y0 = np.stack([equatorial_photon(st, r0, (b_pro if p else b_retro) * (1.0 + d), prograde=p)
                       for p in directions for d in deltas])
        res = engine.integrate_batch(st, y0, integ, term)
        turns_all = np.abs(np.asarray(res.Y)[:, 3] - y0[:, 3]) / (2.0 * math.pi)
        for k, p in enumerate(directions):
            sl = slice(k * deltas.size, (k + 1) * deltas.size)
            turns, states = turns_all[sl], np.asarray(res.state)[sl]
            ok = states == TerminationState.ESCAPED
            rate = float("nan")
            if ok.sum() >= 3:
                rate = -float(np.polyfit(np.log10(deltas[ok]), turns[ok], 1)[0])
            pred = winding_rate_prediction(spin, p)
            out.append(WindingResult(spin, p, b_pro if p else b_retro, turns, states, rate, pred, (rate - pred) / pred))
    return out
