"""Shadow-edge metrics on the host (FP64): the sub-pixel edge of a captured mask and its radial
distance from Bardeen's curve.

**Edge of a mask.** The captured mask -- 1 on captured pixel centres, 0 on the others and on a
ring of virtual centres one pixel outside the image -- is interpolated bilinearly, and the edge
is the 0.5 level set of the interpolant. Along a straight ray from an interior centre the
interpolant is a quadratic in the ray parameter inside each grid cell. Each polar ray is
therefore cut where it crosses a grid line through pixel centres and, inside each piece, at the
quadratic's extremum; between two consecutive cuts the field is monotone. The edge radius is
the first crossing of 0.5: bracketed by the first cut where the field is below 0.5 and located
by bisection on that piece's quadratic, to rounding error and with no marching step.

**Distance to Bardeen's curve.** :class:`kerrray_b200.orbits.BardeenCurve` gives the exact
distance from a centre to the curve along any direction; a sampled closed curve (any polygon
that is star-shaped about the centre) is handled by locating each direction's edge through the
vertices' unwrapped polar angles.

**Finite observer distance.** A zero-angular-momentum observer at r_o sees image coordinates
smaller than Bardeen's (r_o -> infinity) by sqrt(1 - 2M/r_o) to leading order (exactly at
a = 0); :func:`finite_distance_scale` is the factor that undoes it.

The reference's counterparts are ``raytracing/boundary.py:116-178`` (it marches each ray in
1/8-pixel steps and interpolates linearly between the two samples that bracket 0.5),
``:188-218`` (every ray against every polygon edge), ``:221-229``, ``:247-252`` and
``:255-307``; the tests pin these functions against that module's outputs.
"""

from __future__ import annotations

import math
from typing import Any

import numpy as np

from kerrray_b200.orbits import BardeenCurve, shadow_curve

__all__ = ["analytic_boundary", "boundary_error", "extract_boundary", "extract_boundary_from_mask",
           "finite_distance_scale", "mask_centroid", "mask_edge_error", "polygon_centroid", "polygon_radii"]


def mask_centroid(alpha, beta, captured) -> tuple[float, float]:
    """Mean ``(alpha, beta)`` of the captured pixel centres."""
    keep = np.asarray(captured, dtype=bool)
    if not keep.any():
        raise ValueError("the captured mask is empty: no shadow to extract")
    return (float(np.asarray(alpha, dtype=np.float64)[keep].mean()),
            float(np.asarray(beta, dtype=np.float64)[keep].mean()))


def _pixel_grid(alpha: np.ndarray, beta: np.ndarray) -> tuple[float, float, float]:
    """``(alpha of column 0, beta of row 0, pixel size)`` of a regular camera grid."""
    if alpha.ndim != 2 or alpha.shape != beta.shape or min(alpha.shape) < 2:
        raise ValueError("alpha and beta must be 2-D arrays of the same shape with >= 2 pixels per side")
    step = float(alpha[0, 1] - alpha[0, 0])
    regular = (step > 0.0 and np.allclose(np.diff(alpha, axis=1), step) and np.allclose(np.diff(alpha, axis=0), 0.0)
               and np.allclose(np.diff(beta, axis=0), -step) and np.allclose(np.diff(beta, axis=1), 0.0))
    if not regular:
        raise ValueError("the pixel grid must be regular with alpha increasing rightward and beta downward")
    return float(alpha[0, 0]), float(beta[0, 0]), step


def extract_boundary_from_mask(alpha, beta, captured, *, n_angles: int = 360,
                               centre: tuple[float, float] | None = None) -> tuple[np.ndarray, np.ndarray]:
    """``(angles, radii)``: distance (M) from ``centre`` (default: the captured centroid) to the
    0.5 level set of the mask's bilinear interpolant along ``phi_k = 2 pi k / n_angles``.

    Raises ``ValueError`` when the mask is empty or touches the image border, or when the
    centre lies outside the captured region."""
    a = np.asarray(alpha, dtype=np.float64)
    b = np.asarray(beta, dtype=np.float64)
    mask = np.asarray(captured, dtype=bool)
    if mask.shape != a.shape:
        raise ValueError(f"captured has shape {mask.shape}, expected {a.shape}")
    if n_angles < 1:
        raise ValueError("n_angles must be >= 1")
    border = np.concatenate([mask[0], mask[-1], mask[:, 0], mask[:, -1]])
    if border.any():
        raise ValueError("the captured region touches the image border; widen the field of view")
    a0, b0, step = _pixel_grid(a, b)
    cx, cy = mask_centroid(a, b, mask) if centre is None else (float(centre[0]), float(centre[1]))
    rows, cols = mask.shape
    field = np.zeros((rows + 2, cols + 2))
    field[1:-1, 1:-1] = mask
    # Grid coordinates of the padded field: pixel (i, j) sits at column u = j + 1, row v = i + 1.
    uc, vc = (cx - a0) / step + 1.0, (b0 - cy) / step + 1.0
    angles = 2.0 * math.pi * np.arange(n_angles, dtype=np.float64) / n_angles
    du, dv = np.cos(angles) / step, -np.sin(angles) / step  # per unit length along the ray

    def cell_value(u, v):
        j = np.clip(np.floor(u).astype(np.intp), 0, cols)
        i = np.clip(np.floor(v).astype(np.intp), 0, rows)
        fu, fv = np.clip(u - j, 0.0, 1.0), np.clip(v - i, 0.0, 1.0)
        return ((field[i, j] * (1.0 - fu) + field[i, j + 1] * fu) * (1.0 - fv)
                + (field[i + 1, j] * (1.0 - fu) + field[i + 1, j + 1] * fu) * fv)

    if cell_value(np.array([uc]), np.array([vc]))[0] < 0.5:
        raise ValueError("the centre lies outside the captured region")

    def crossings(c0: float, rate: np.ndarray, upper: int) -> np.ndarray:
        """Ray parameters where the coordinate c0 + rate t meets the integers in (0, upper)."""
        m = np.arange(upper + 1, dtype=np.float64)[None, :]
        first = np.where(rate[:, None] > 0.0, math.floor(c0) + 1.0 + m, math.ceil(c0) - 1.0 - m)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (first - c0) / rate[:, None]
        ok = (rate[:, None] != 0.0) & (first > 0.0) & (first < upper) & (t > 0.0)
        return np.where(ok, t, np.inf)

    def leave(c0: float, rate: np.ndarray, upper: int) -> np.ndarray:
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(rate > 0.0, (upper - c0) / rate, np.where(rate < 0.0, -c0 / rate, np.inf))

    t_exit = np.minimum(leave(uc, du, cols + 1), leave(vc, dv, rows + 1))
    cuts = np.concatenate([np.zeros((n_angles, 1)), crossings(uc, du, cols + 1), crossings(vc, dv, rows + 1),
                           t_exit[:, None]], axis=1)
    cuts = np.sort(np.minimum(cuts, t_exit[:, None]), axis=1)
    t0, t1 = cuts[:, :-1], cuts[:, 1:]
    # The cell of each piece (from its midpoint) and the field along the piece as A + B t + C t^2.
    tm = 0.5 * (t0 + t1)
    j = np.clip(np.floor(uc + du[:, None] * tm).astype(np.intp), 0, cols)
    i = np.clip(np.floor(vc + dv[:, None] * tm).astype(np.intp), 0, rows)
    f00, f01, f10, f11 = field[i, j], field[i, j + 1], field[i + 1, j], field[i + 1, j + 1]
    e1, e2, e3 = f01 - f00, f10 - f00, f11 - f10 - f01 + f00
    pu, pv = uc - j, vc - i
    qu, qv = du[:, None], dv[:, None]
    A = f00 + e1 * pu + e2 * pv + e3 * pu * pv
    B = e1 * qu + e2 * qv + e3 * (pu * qv + pv * qu)
    C = e3 * qu * qv
    with np.errstate(divide="ignore", invalid="ignore"):
        tv = np.where(C > 0.0, -B / (2.0 * C), np.nan)  # a minimum inside the piece splits it
    inner = (tv > t0) & (tv < t1)

    def q(t):
        return A + (B + C * t) * t

    f_vertex = np.where(inner, q(np.where(inner, tv, t0)), np.inf)
    f_end = q(t1)
    live = t1 > t0
    below = live & (np.minimum(f_vertex, f_end) < 0.5)
    k = np.argmax(below, axis=1)
    if not below[np.arange(n_angles), k].all():  # cannot happen: the field is 0 where the ray leaves
        raise ValueError("no 0.5 crossing found along some direction")
    r = np.arange(n_angles)
    Ak, Bk, Ck = A[r, k], B[r, k], C[r, k]
    lo = np.where(inner[r, k] & ~(f_vertex[r, k] < 0.5), tv[r, k], t0[r, k])
    hi = np.where(f_vertex[r, k] < 0.5, tv[r, k], t1[r, k])
    for _ in range(64):
        mid = 0.5 * (lo + hi)
        high = Ak + (Bk + Ck * mid) * mid >= 0.5
        lo = np.where(high, mid, lo)
        hi = np.where(high, hi, mid)
    return angles, 0.5 * (lo + hi)


def extract_boundary(img: Any, n_angles: int = 360, centre: tuple[float, float] | None = None):
    """:func:`extract_boundary_from_mask` of a :class:`~kerrray_b200.shadow.ShadowImage`."""
    return extract_boundary_from_mask(img.alpha, img.beta, img.captured, n_angles=n_angles, centre=centre)


def analytic_boundary(st: Any, inclination_deg: float, n: int = 720) -> tuple[np.ndarray, np.ndarray]:
    """Bardeen's shadow curve sampled at ``2 (n // 2)`` points (:func:`~kerrray_b200.orbits.shadow_curve`)."""
    return shadow_curve(st, inclination_deg, n)


def polygon_radii(alpha, beta, centre: tuple[float, float], angles) -> np.ndarray:
    """Distance from ``centre`` to the closed polygon ``(alpha, beta)`` along each polar angle.

    The polygon must be star-shaped about the centre: its vertices' polar angles, unwrapped
    along the polygon, then turn once monotonically, and each direction's edge is found by a
    binary search on them. Raises ``ValueError`` otherwise."""
    px = np.asarray(alpha, dtype=np.float64).ravel()
    py = np.asarray(beta, dtype=np.float64).ravel()
    if px.size < 3 or px.shape != py.shape:
        raise ValueError("a polygon needs at least three (alpha, beta) points")
    qx = np.append(px, px[0]) - float(centre[0])
    qy = np.append(py, py[0]) - float(centre[1])
    psi = np.unwrap(np.arctan2(qy, qx))
    turn = psi[-1] - psi[0]
    if abs(abs(turn) - 2.0 * math.pi) > 1e-9:
        raise ValueError("the centre lies outside the polygon")
    sign = 1.0 if turn > 0.0 else -1.0
    psi = sign * psi
    if np.any(np.diff(psi) <= 0.0):
        raise ValueError("the polygon is not star-shaped about the centre")
    phi = np.asarray(angles, dtype=np.float64).ravel()
    target = psi[0] + np.mod(sign * phi - psi[0], 2.0 * math.pi)
    k = np.clip(np.searchsorted(psi, target, side="right") - 1, 0, px.size - 1)
    ex, ey = qx[k + 1] - qx[k], qy[k + 1] - qy[k]
    dx, dy = np.cos(phi), np.sin(phi)
    return (qx[k] * ey - qy[k] * ex) / (dx * ey - dy * ex)


def polygon_centroid(x, y) -> tuple[float, float]:
    """Area centroid of the closed polygon ``(x, y)`` (the shoelace sums)."""
    xs = np.asarray(x, dtype=np.float64).ravel()
    ys = np.asarray(y, dtype=np.float64).ravel()
    x1, y1 = np.roll(xs, -1), np.roll(ys, -1)
    w = xs * y1 - x1 * ys  # twice the signed area of each triangle (origin, p_k, p_k+1)
    twice_area = w.sum()
    if twice_area == 0.0:
        raise ValueError("degenerate polygon (zero area)")
    return float(((xs + x1) * w).sum() / (3.0 * twice_area)), float(((ys + y1) * w).sum() / (3.0 * twice_area))


def finite_distance_scale(st: Any, radius: float) -> float:
    """``1 / sqrt(1 - 2M / r_o)``: scales image coordinates seen at ``r_o`` to Bardeen's."""
    mass = float(st.mass)
    if not radius > 2.0 * mass:
        raise ValueError("the observer radius must exceed 2M for the finite-distance factor")
    return 1.0 / math.sqrt(1.0 - 2.0 * mass / float(radius))


def boundary_error(numeric: tuple[Any, Any], analytic: Any, centre: tuple[float, float], *,
                   pixel_size: float | None = None, scale: float = 1.0) -> dict[str, float]:
    """Radial differences ``r_numeric - r_analytic`` of an edge ``(angles, radii)`` about
    ``centre``, after scaling the radii and the centre by ``scale``.

    ``analytic`` is a :class:`~kerrray_b200.orbits.BardeenCurve` (exact radii) or a closed
    ``(alpha, beta)`` polygon. Returns ``max`` (of |d|), ``rms``, ``mean`` and ``mean_abs`` in
    M, both curves' mean radii and ``scale``; with ``pixel_size``, every length also in pixels
    (``*_px``)."""
    phi = np.asarray(numeric[0], dtype=np.float64)
    r_num = np.asarray(numeric[1], dtype=np.float64) * scale
    c = (float(centre[0]) * scale, float(centre[1]) * scale)
    if isinstance(analytic, BardeenCurve):
        r_ana = analytic.radii(c, phi)
    else:
        r_ana = polygon_radii(analytic[0], analytic[1], c, phi)
    diff = r_num - r_ana
    out = {"max": float(np.abs(diff).max()), "rms": float(np.sqrt(np.mean(diff * diff))), "mean": float(diff.mean()),
           "mean_abs": float(np.abs(diff).mean()), "radius_mean_numeric": float(r_num.mean()),
           "radius_mean_analytic": float(r_ana.mean())}
    if pixel_size is not None:
        if not pixel_size > 0.0:
            raise ValueError("pixel_size must be > 0")
        out.update({f"{key}_px": value / pixel_size for key, value in list(out.items())})
    out["scale"] = float(scale)
    return out


def mask_edge_error(st: Any, camera: Any, captured, *, n_angles: int = 360) -> dict[str, float]:
    """Edge of a captured mask traced with ``camera`` against Bardeen's exact curve, about the
    captured centroid, after the finite-distance correction (:func:`boundary_error`, in M and px)."""
    alpha, beta = camera.pixel_coordinates()
    mask = np.asarray(captured, dtype=bool).reshape(alpha.shape)
    c = mask_centroid(alpha, beta, mask)
    edge = extract_boundary_from_mask(alpha, beta, mask, n_angles=n_angles, centre=c)
    return boundary_error(edge, BardeenCurve(st, camera.inclination_deg), c, pixel_size=camera.pixel_size,
                          scale=finite_distance_scale(st, camera.radius))
