"""Kerr photon orbits and Bardeen's shadow curve on the host (FP64), from the radial potential.

A photon with constants of motion xi = L_z/E and eta = Q/E^2 moves in r under the radial
potential R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2), Delta = r^2 - 2Mr + a^2
(the potential of the device's analytic photon classes). Spherical photon orbits are its
double roots, R = R' = 0, which give (Bardeen 1973)::

    xi(r)  = [M (r^2 - a^2) - r Delta] / [a (r - M)]
    eta(r) = r^3 [4 M Delta - r (r - M)^2] / [a^2 (r - M)^2]

for r between the prograde and the retrograde circular equatorial photon orbits, whose radii
and impact parameters have closed forms (Bardeen, Press & Teukolsky 1972; Chandrasekhar,
*The Mathematical Theory of Black Holes*, section 63), upper sign prograde::

    r_ph = 2M {1 + cos[(2/3) arccos(-+|a|/M)]},   b_c = -+|a| + 6M cos[(1/3) arccos(-+|a|/M)]

An observer at infinity and inclination i sees the photons of the orbit at r at
alpha = -xi / sin i and beta = +-sqrt(Theta(r)), Theta = eta + a^2 cos^2 i - xi^2 cot^2 i.
Bardeen's shadow edge is that closed curve over the interval of r around the polar orbit
(xi = 0) where Theta >= 0; its end points are roots of a degree-6 polynomial (Theta times
a^2 (r - M)^2), found with ``numpy.roots`` and polished by Newton steps.

The curve is convex, so everything here rests on one primitive: the exact distance from an
interior point to the curve along a polar direction (:meth:`BardeenCurve.radii`), found by
bisection on the curve's own parameter -- no sampled polygon is involved. The curve samples
(:func:`shadow_curve`, uniform in polar angle about the origin), its area centroid
(:meth:`BardeenCurve.centroid`, the periodic trapezoid rule on the exact polar radius) and the
edge errors of the shadow metrics all derive from it.

The reference computes the same curve in ``photons/orbits.py:174-273``
(``critical_impact_parameters``, ``shadow_curve``) by sampling it in r, and measures radii on
the sampled polygon (``raytracing/boundary.py:188-218``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

__all__ = ["BardeenCurve", "critical_impact_parameters", "equatorial_photon_orbit_radius", "shadow_curve",
           "spherical_orbit_constants", "spherical_orbit_radius_range"]


def _mass_and_spin(st: Any) -> tuple[float, float]:
    """``(M, a)`` of a spacetime object, checked to describe a black hole (0 <= |a| < M)."""
    mass = float(st.mass)
    a = float(getattr(st, "a", getattr(st, "spin", 0.0)))
    if not (math.isfinite(mass) and mass > 0.0):
        raise ValueError(f"mass must be positive, got {mass}")
    if not abs(a) < mass:
        raise ValueError(f"|a| < M required for a black hole, got a={a}, M={mass}")
    return mass, a


def _equatorial_orbit(mass: float, a: float, prograde: bool) -> tuple[float, float]:
    """(radius, impact parameter |L_z|/E) of the circular equatorial photon orbit, closed form."""
    x = (-1.0 if prograde else 1.0) * abs(a) / mass
    angle = math.acos(x)
    radius = 2.0 * mass * (1.0 + math.cos(2.0 * angle / 3.0))
    impact = x * mass + 6.0 * mass * math.cos(angle / 3.0)
    return radius, impact


def equatorial_photon_orbit_radius(st: Any, prograde: bool = True) -> float:
    """Radius of the circular equatorial photon orbit (prograde: a L_z > 0); 3M at a = 0."""
    mass, a = _mass_and_spin(st)
    return _equatorial_orbit(mass, a, prograde)[0]


def critical_impact_parameters(st: Any) -> tuple[float, float]:
    """``(b_prograde, b_retrograde) = |L_z| / E`` of the equatorial photon orbits (3 sqrt(3) M at a = 0)."""
    mass, a = _mass_and_spin(st)
    return _equatorial_orbit(mass, a, True)[1], _equatorial_orbit(mass, a, False)[1]


def spherical_orbit_radius_range(st: Any) -> tuple[float, float]:
    """Radii of the innermost (prograde) and outermost (retrograde) spherical photon orbits."""
    return equatorial_photon_orbit_radius(st, True), equatorial_photon_orbit_radius(st, False)


def spherical_orbit_constants(st: Any, r):
    """``(xi, eta)`` of the spherical photon orbit at radius ``r`` (``a != 0``)."""
    mass, a = _mass_and_spin(st)
    if a == 0.0:
        raise ValueError("spherical orbit constants are undefined for a = 0 (every orbit sits at r = 3M)")
    return _xi_eta(mass, a, np.asarray(r, dtype=np.float64))


def _xi_eta(mass: float, a: float, r):
    delta = r * r - 2.0 * mass * r + a * a
    rm = r - mass
    xi = (mass * (r * r - a * a) - r * delta) / (a * rm)
    eta = r**3 * (4.0 * mass * delta - r * rm * rm) / (a * a * rm * rm)
    return xi, eta


def _wrap(x):
    """Angle difference mapped into [-pi, pi)."""
    return np.mod(np.asarray(x) + math.pi, 2.0 * math.pi) - math.pi


@dataclass(frozen=True)
class BardeenCurve:
    """Bardeen's shadow edge of ``spacetime`` for a distant observer at ``inclination_deg``.

    The curve is parametrised by ``s`` in [0, 2]: ``s`` in [0, 1] runs along the beta >= 0
    branch from the inner turning orbit r_a to the outer one r_b, ``s`` in [1, 2] back along
    beta <= 0, with r = r_a + (r_b - r_a)(1 - cos(pi s))/2 (smooth at the turning points).
    """

    spacetime: Any
    inclination_deg: float
    _geom: dict = field(init=False, repr=False, compare=False)

    def __post_init__(self) -> None:
        mass, a = _mass_and_spin(self.spacetime)
        incl = float(self.inclination_deg)
        if not 0.0 < incl < 180.0:
            raise ValueError("inclination_deg must lie strictly between 0 and 180")
        g: dict[str, float] = {"mass": mass, "a": a}
        if a == 0.0:
            g["b_c"] = critical_impact_parameters(self.spacetime)[0]
        else:
            inc = math.radians(incl)
            g["sin_i"] = math.sin(inc)
            g["cos_i"] = 0.0 if incl == 90.0 else math.cos(inc)
            g["cot2"] = (g["cos_i"] / g["sin_i"]) ** 2
            g["r_a"], g["r_b"] = self._turning_orbits(mass, a, g["cos_i"], g["cot2"])
        object.__setattr__(self, "_geom", g)

    # -- construction -----------------------------------------------------------------------
    @staticmethod
    def _turning_orbits(mass: float, a: float, cos_i: float, cot2: float) -> tuple[float, float]:
        """The interval [r_a, r_b] around the polar orbit on which Theta(r) >= 0."""
        r_lo = _equatorial_orbit(mass, a, True)[0]
        r_hi = _equatorial_orbit(mass, a, False)[0]
        P = np.polynomial.Polynomial
        r = P([0.0, 1.0])
        delta = r * r - 2.0 * mass * r + a * a
        xi_num = mass * (r * r - a * a) - r * delta          # xi a (r - M)
        theta_poly = r**3 * (4.0 * mass * delta - r * (r - mass) ** 2) \
            + (a * a * cos_i) ** 2 * (r - mass) ** 2 - cot2 * xi_num**2  # Theta a^2 (r - M)^2
        # The polar orbit: xi = 0, a root of the cubic xi_num inside [r_lo, r_hi].
        r0 = [z.real for z in xi_num.roots() if abs(z.imag) < 1e-9 and r_lo <= z.real <= r_hi]
        if len(r0) != 1:
            raise RuntimeError("no unique polar spherical orbit between the equatorial photon orbits")
        r0 = r0[0]
        if theta_poly(r0) <= 0.0:
            raise RuntimeError("Theta is not positive at the polar orbit")
        dpoly = theta_poly.deriv()

        def polish(x: float) -> float:
            for _ in range(4):
                d = dpoly(x)
                if d == 0.0:
                    break
                x -= theta_poly(x) / d
            return x

        roots = sorted(polish(z.real) for z in theta_poly.roots() if abs(z.imag) < 1e-6 * mass)
        below = [x for x in roots if r_lo < x < r0]
        above = [x for x in roots if r0 < x < r_hi]
        r_a = max(below) if below else r_lo
        r_b = min(above) if above else r_hi
        return r_a, r_b

    # -- evaluation -------------------------------------------------------------------------
    def points_at(self, s):
        """``(alpha, beta)`` at curve parameter(s) ``s`` in [0, 2]."""
        g = self._geom
        s = np.asarray(s, dtype=np.float64)
        if g["a"] == 0.0:
            phi = math.pi * (1.0 - s)
            return g["b_c"] * np.cos(phi), g["b_c"] * np.sin(phi)
        u = np.where(s <= 1.0, s, 2.0 - s)
        r = g["r_a"] + (g["r_b"] - g["r_a"]) * 0.5 * (1.0 - np.cos(math.pi * u))
        xi, eta = _xi_eta(g["mass"], g["a"], r)
        theta = eta + (g["a"] * g["cos_i"]) ** 2 - xi * xi * g["cot2"]
        beta = np.sqrt(np.maximum(theta, 0.0))
        beta = np.where((u == 0.0) | (u == 1.0), 0.0, beta)  # the turning points lie on beta = 0
        return -xi / g["sin_i"], np.where(s <= 1.0, beta, -beta)

    def radii(self, centre: tuple[float, float], angles, coarse: int = 2048, iterations: int = 64) -> np.ndarray:
        """Exact distance from ``centre`` (inside the curve) to the curve along each polar angle."""
        g = self._geom
        phi = np.asarray(angles, dtype=np.float64)
        cx, cy = float(centre[0]), float(centre[1])
        if g["a"] == 0.0:  # a circle of radius b_c about the origin
            dx, dy = np.cos(phi), np.sin(phi)
            proj = cx * dx + cy * dy
            disc = proj * proj - (cx * cx + cy * cy - g["b_c"] ** 2)
            if np.any(disc < 0.0) or cx * cx + cy * cy >= g["b_c"] ** 2:
                raise ValueError("the centre lies outside the shadow curve")
            return -proj + np.sqrt(disc)
        s_grid = np.linspace(0.0, 2.0, coarse + 1)
        x, y = self.points_at(s_grid)
        psi = np.unwrap(np.arctan2(y - cy, x - cx))
        turn = psi[-1] - psi[0]
        if abs(abs(turn) - 2.0 * math.pi) > 1e-6:
            raise ValueError("the centre lies outside the shadow curve")
        sign = 1.0 if turn > 0.0 else -1.0
        psi = sign * psi                     # increasing along s
        if np.any(np.diff(psi) <= 0.0):
            raise ValueError("the shadow curve is not star-shaped about the centre")
        target = psi[0] + np.mod(sign * phi - psi[0], 2.0 * math.pi)
        j = np.clip(np.searchsorted(psi, target, side="right") - 1, 0, coarse - 1)
        lo, hi = s_grid[j], s_grid[j + 1]
        base = psi[j]
        for _ in range(iterations):
            mid = 0.5 * (lo + hi)
            mx, my = self.points_at(mid)
            ang = base + _wrap(sign * np.arctan2(my - cy, mx - cx) - base)
            below = ang < target
            lo = np.where(below, mid, lo)
            hi = np.where(below, hi, mid)
        px, py = self.points_at(0.5 * (lo + hi))
        return np.hypot(px - cx, py - cy)

    def centroid(self, n: int = 4096) -> tuple[float, float]:
        """Area centroid of the region inside the curve (periodic trapezoid rule in polar angle
        about the origin, which lies inside every Kerr shadow; spectrally accurate)."""
        phi = 2.0 * math.pi * np.arange(n) / n
        r = self.radii((0.0, 0.0), phi)
        area = 0.5 * np.mean(r * r) * 2.0 * math.pi
        m3 = np.mean(r**3 * np.cos(phi)) * 2.0 * math.pi / 3.0, np.mean(r**3 * np.sin(phi)) * 2.0 * math.pi / 3.0
        return float(m3[0] / area), float(m3[1] / area)

    def sample(self, n: int) -> tuple[np.ndarray, np.ndarray]:
        """``n`` points at polar angles -pi + 2 pi k / n about the origin (ordered by angle)."""
        phi = -math.pi + 2.0 * math.pi * np.arange(n) / n
        r = self.radii((0.0, 0.0), phi)
        return r * np.cos(phi), r * np.sin(phi)


def shadow_curve(st: Any, inclination_deg: float, n: int = 720) -> tuple[np.ndarray, np.ndarray]:
    """Bardeen's shadow edge ``(alpha, beta)`` for an observer at infinity: ``2 (n // 2)`` points
    on the exact curve, uniform in polar angle about the origin and ordered by it."""
    n_points = 2 * (int(n) // 2)
    if n_points < 4:
        raise ValueError("n must be at least 4")
    return BardeenCurve(st, float(inclination_deg)).sample(n_points)
