"""Analytic Kerr photon orbits and Bardeen's shadow curve (host side, FP64).

Restates ``src/kerrray/photons/orbits.py``: the spherical-photon-orbit constants
(``:spherical_orbit_constants``, Bardeen 1973; Johannsen & Psaltis 2010 eqs. 8-9), the
equatorial photon orbit radii by bracketed root finding of ``r - 3M = -+ 2|a| sqrt(M/r)``
(``:equatorial_photon_orbit_radius``), the critical impact parameters (``:174-185``) and the
shadow curve ``alpha = -xi/sin(i)``, ``beta = +-sqrt(eta + a^2 cos^2 i - xi^2 cot^2 i)`` over
the spherical orbits whose radicand is non-negative, sampled with cosine clustering at the
turning points and ordered by polar angle (``:206-273``). These curves are the reference the
shadow-edge metrics compare against; they are not on the per-ray path.
"""

from __future__ import annotations

import math
from typing import Any

import numpy as np
from scipy.optimize import brentq

__all__ = ["critical_impact_parameters", "equatorial_photon_orbit_radius", "shadow_curve",
           "spherical_orbit_constants", "spherical_orbit_radius_range"]

_ROOT_XTOL = 1e-14
_ROOT_RTOL = 1e-14


def _mass_and_spin(st: Any) -> tuple[float, float]:
    mass, a = float(st.mass), float(st.a)
    if not mass > 0.0:
        raise ValueError(f"mass must be positive, got {mass}")
    if not abs(a) < mass:
        raise ValueError(f"|a| < M required for a black hole, got a={a}, M={mass}")
    return mass, a


def spherical_orbit_constants(st: Any, r):
    """``(xi, eta)`` of the spherical photon orbit at radius ``r`` (``a != 0``)."""
    mass, a = _mass_and_spin(st)
    if a == 0.0:
        raise ValueError("spherical orbit constants are undefined for a = 0 (every orbit sits at r = 3M)")
    r = np.asarray(r, dtype=np.float64)
    r_m3 = r - 3.0 * mass
    xi = -(r * r * r_m3 + a * a * (r + mass)) / (a * (r - mass))
    eta = r**3 * (4.0 * mass * a * a - r * r_m3 * r_m3) / (a * a * (r - mass) ** 2)
    return xi, eta


def equatorial_photon_orbit_radius(st: Any, prograde: bool = True) -> float:
    """Circular equatorial photon orbit radius (prograde: ``a L_z > 0``)."""
    mass, a = _mass_and_spin(st)
    s = 1 if prograde else -1
    abs_a = abs(a)

    def f(r: float) -> float:
        return r - 3.0 * mass + s * 2.0 * abs_a * math.sqrt(mass / r)

    lo, hi = (mass, 3.5 * mass) if prograde else (2.5 * mass, 4.0 * mass)
    return float(brentq(f, lo, hi, xtol=_ROOT_XTOL * mass, rtol=_ROOT_RTOL))


def _equatorial_orbit_xi(mass: float, a: float, r: float, prograde: bool) -> float:
    s = 1 if prograde else -1
    delta = r * r - 2.0 * mass * r + a * a
    spin_sign = -1 if a < 0.0 else 1
    return spin_sign * (abs(a) + s * 2.0 * r * math.sqrt(delta) / (r - mass))


def critical_impact_parameters(st: Any) -> tuple[float, float]:
    """``(b_prograde, b_retrograde) = |L_z| / E`` on the equatorial photon orbits (3 sqrt(3) M at a = 0)."""
    mass, a = _mass_and_spin(st)
    out = []
    for prograde in (True, False):
        r_ph = equatorial_photon_orbit_radius(st, prograde)
        out.append(abs(_equatorial_orbit_xi(mass, a, r_ph, prograde)))
    return out[0], out[1]


def spherical_orbit_radius_range(st: Any) -> tuple[float, float]:
    return equatorial_photon_orbit_radius(st, True), equatorial_photon_orbit_radius(st, False)


def shadow_curve(st: Any, inclination_deg: float, n: int = 720) -> tuple[np.ndarray, np.ndarray]:
    """Bardeen's shadow boundary ``(alpha, beta)`` for an observer at infinity, ``2 (n // 2)`` points."""
    mass, a = _mass_and_spin(st)
    if not 0.0 < inclination_deg < 180.0:
        raise ValueError("inclination_deg must lie strictly between 0 and 180")
    n_points = 2 * (int(n) // 2)
    if n_points < 4:
        raise ValueError("n must be at least 4")
    inc = math.radians(inclination_deg)
    sin_i = math.sin(inc)
    cos_i = 0.0 if inclination_deg == 90.0 else math.cos(inc)
    if a == 0.0:
        b_c = critical_impact_parameters(st)[0]
        angle = np.linspace(-math.pi, math.pi, n_points, endpoint=False)
        return b_c * np.cos(angle), b_c * np.sin(angle)
    cot2 = (cos_i / sin_i) ** 2
    r_lo, r_hi = spherical_orbit_radius_range(st)
    tol = {"xtol": _ROOT_XTOL * mass, "rtol": _ROOT_RTOL}

    def xi_of(r: float) -> float:
        return float(spherical_orbit_constants(st, r)[0])

    def radicand(r: float) -> float:
        xi, eta = spherical_orbit_constants(st, r)
        return float(eta + a * a * cos_i * cos_i - xi * xi * cot2)

    if xi_of(r_lo) * xi_of(r_hi) >= 0.0:
        raise RuntimeError("xi(r) does not change sign on the spherical-orbit range")
    r_0 = brentq(xi_of, r_lo, r_hi, **tol)
    if radicand(r_0) <= 0.0:
        raise RuntimeError("radicand is not positive at the polar orbit")
    r_a = r_lo if radicand(r_lo) >= 0.0 else brentq(radicand, r_lo, r_0, **tol)
    r_b = r_hi if radicand(r_hi) >= 0.0 else brentq(radicand, r_0, r_hi, **tol)
    m = n_points // 2 + 1
    u = np.linspace(0.0, 1.0, m)
    r = r_a + (r_b - r_a) * 0.5 * (1.0 - np.cos(math.pi * u))
    xi, eta = spherical_orbit_constants(st, r)
    rad = eta + a * a * cos_i * cos_i - xi * xi * cot2
    beta_up = np.sqrt(np.clip(rad, 0.0, None))
    beta_up[0] = 0.0   # the turning points are roots of the radicand by construction
    beta_up[-1] = 0.0
    alpha_up = -xi / sin_i
    alpha = np.concatenate([alpha_up, alpha_up[-2:0:-1]])
    beta = np.concatenate([beta_up, -beta_up[-2:0:-1]])
    order = np.argsort(np.arctan2(beta, alpha), kind="stable")
    return alpha[order], beta[order]
