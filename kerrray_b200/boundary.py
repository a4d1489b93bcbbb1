"""Shadow-edge metrics on the host: sub-pixel edge of a mask, the analytic Bardeen curve and
the radial differences between them.

Restates ``src/kerrray/raytracing/boundary.py``: the 0.5 level set of the bilinear interpolant
of the captured mask, marched outward along ``n_angles`` polar rays in steps of 1/8 pixel from
the captured centroid (``:116-170``); exact ray-segment intersection with a closed polygon
(``:188-218``); the shoelace centroid (``:221-229``); the finite-distance factor
``1/sqrt(1 - 2M/r_o)`` (``:247-252``); and the error summary (``:255-307``, ``:310-338``).
"""

from __future__ import annotations

import math
from typing import Any

import numpy as np

from kerrray_b200.orbits import shadow_curve

__all__ = ["STEP_FRACTION", "analytic_boundary", "boundary_error", "curve_summary", "extract_boundary",
           "extract_boundary_from_mask", "finite_distance_scale", "mask_centroid", "polygon_centroid",
           "polygon_radii", "summarise_shadow"]

STEP_FRACTION = 0.125
EDGE_TOLERANCE = 1e-9


def mask_centroid(alpha, beta, captured) -> tuple[float, float]:
    mask = np.asarray(captured, dtype=bool)
    if not np.any(mask):
        raise ValueError("the captured mask is empty: no shadow to extract")
    a, b = np.asarray(alpha, dtype=np.float64), np.asarray(beta, dtype=np.float64)
    return float(a[mask].mean()), float(b[mask].mean())


def _grid_geometry(alpha: np.ndarray, beta: np.ndarray) -> tuple[float, float, float]:
    if alpha.ndim != 2 or alpha.shape != beta.shape or min(alpha.shape) < 2:
        raise ValueError("alpha and beta must be 2-D arrays of the same shape with >= 2 pixels per side")
    d = float(alpha[0, 1] - alpha[0, 0])
    if not d > 0.0:
        raise ValueError("alpha must increase along the columns")
    if not np.allclose(np.diff(alpha, axis=1), d) or not np.allclose(np.diff(beta, axis=0), -d):
        raise ValueError("the pixel grid must be regular with alpha increasing rightward and beta downward")
    return float(alpha[0, 0]), float(beta[0, 0]), d


def _bilinear(field: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    n_rows, n_cols = field.shape
    padded = np.pad(field, 1)
    up, vp = u + 1.0, v + 1.0
    inside = (up >= 0.0) & (up <= n_cols) & (vp >= 0.0) & (vp <= n_rows)
    j0 = np.clip(np.floor(up).astype(np.intp), 0, n_cols)
    i0 = np.clip(np.floor(vp).astype(np.intp), 0, n_rows)
    fu = np.clip(up - j0, 0.0, 1.0)
    fv = np.clip(vp - i0, 0.0, 1.0)
    j1 = np.minimum(j0 + 1, n_cols + 1)
    i1 = np.minimum(i0 + 1, n_rows + 1)
    value = (padded[i0, j0] * (1.0 - fu) * (1.0 - fv) + padded[i0, j1] * fu * (1.0 - fv)
             + padded[i1, j0] * (1.0 - fu) * fv + padded[i1, j1] * fu * fv)
    return np.where(inside, value, 0.0)


def extract_boundary_from_mask(alpha, beta, captured, *, n_angles: int = 360,
                               centre: tuple[float, float] | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Sub-pixel edge radii ``r(phi_k)``, ``phi_k = 2 pi k / n_angles``, about ``centre``."""
    a = np.asarray(alpha, dtype=np.float64)
    b = np.asarray(beta, dtype=np.float64)
    mask = np.asarray(captured, dtype=bool)
    if mask.shape != a.shape:
        raise ValueError(f"captured has shape {mask.shape}, expected {a.shape}")
    if n_angles < 1:
        raise ValueError("n_angles must be >= 1")
    if mask[0, :].any() or mask[-1, :].any() or mask[:, 0].any() or mask[:, -1].any():
        raise ValueError("the captured region touches the image border; increase the field of view")
    a0, b0, d = _grid_geometry(a, b)
    ca, cb = mask_centroid(a, b, mask) if centre is None else (float(centre[0]), float(centre[1]))
    field = mask.astype(np.float64)
    angles = 2.0 * np.pi * np.arange(n_angles, dtype=np.float64) / n_angles
    ds = STEP_FRACTION * d
    reach = math.hypot(a[0, -1] - a[0, 0], b[0, 0] - b[-1, 0]) + 2.0 * d
    s = ds * np.arange(int(math.ceil(reach / ds)) + 1, dtype=np.float64)
    x = ca + np.cos(angles)[:, None] * s[None, :]
    y = cb + np.sin(angles)[:, None] * s[None, :]
    f = _bilinear(field, (x - a0) / d, (b0 - y) / d)
    if np.any(f[:, 0] < 0.5):
        raise ValueError("the centre lies outside the captured region")
    below = f < 0.5
    k = np.argmax(below, axis=1)
    rows = np.arange(n_angles)
    f_in, f_out = f[rows, k - 1], f[rows, k]
    radii = s[k - 1] + ds * (f_in - 0.5) / (f_in - f_out)
    return angles, radii


def extract_boundary(img, n_angles: int = 360, centre: tuple[float, float] | None = None):
    return extract_boundary_from_mask(img.alpha, img.beta, img.captured, n_angles=n_angles, centre=centre)


def analytic_boundary(st, inclination_deg: float, n: int = 720) -> tuple[np.ndarray, np.ndarray]:
    return shadow_curve(st, inclination_deg, n)


def polygon_radii(alpha, beta, centre: tuple[float, float], angles) -> np.ndarray:
    """Distance from ``centre`` to the closed polygon along each angle (smallest ``t > 0``)."""
    px = np.asarray(alpha, dtype=np.float64).ravel()
    py = np.asarray(beta, dtype=np.float64).ravel()
    if px.size < 3 or px.shape != py.shape:
        raise ValueError("a polygon needs at least three (alpha, beta) points")
    phi = np.asarray(angles, dtype=np.float64).ravel()
    ca, cb = float(centre[0]), float(centre[1])
    qx, qy = px - ca, py - cb
    ex, ey = np.roll(qx, -1) - qx, np.roll(qy, -1) - qy
    dx, dy = np.cos(phi)[:, None], np.sin(phi)[:, None]
    det = dx * (-ey[None, :]) - dy * (-ex[None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (qx[None, :] * (-ey[None, :]) - qy[None, :] * (-ex[None, :])) / det
        s = (dx * qy[None, :] - dy * qx[None, :]) / det
    valid = np.isfinite(t) & (t > 0.0) & (s >= -EDGE_TOLERANCE) & (s <= 1.0 + EDGE_TOLERANCE)
    radii = np.where(valid, t, np.inf).min(axis=1)
    if not np.all(np.isfinite(radii)):
        raise ValueError("a polar ray from the centre does not intersect the analytic curve")
    return radii


def polygon_centroid(x, y) -> tuple[float, float]:
    xs, ys = np.asarray(x, dtype=np.float64).ravel(), np.asarray(y, dtype=np.float64).ravel()
    xn, yn = np.roll(xs, -1), np.roll(ys, -1)
    cross = xs * yn - xn * ys
    area = 0.5 * cross.sum()
    if area == 0.0:
        raise ValueError("degenerate polygon (zero area)")
    return float(((xs + xn) * cross).sum() / (6.0 * area)), float(((ys + yn) * cross).sum() / (6.0 * area))


def curve_summary(angles, radii, centre: tuple[float, float]) -> dict[str, float]:
    phi, r = np.asarray(angles, dtype=np.float64), np.asarray(radii, dtype=np.float64)
    cx, cy = polygon_centroid(centre[0] + r * np.cos(phi), centre[1] + r * np.sin(phi))
    return {"radius_mean": float(r.mean()), "radius_min": float(r.min()), "radius_max": float(r.max()),
            "asymmetry": float(r.max() - r.min()), "centroid_alpha": cx, "centroid_beta": cy,
            "centroid_displacement": math.hypot(cx, cy)}


def finite_distance_scale(st, radius: float) -> float:
    """``1 / sqrt(1 - 2M / r_o)``: ZAMO pixel coordinates at ``r_o`` -> Bardeen's (leading order)."""
    if not radius > 2.0 * st.mass:
        raise ValueError("the observer radius must exceed 2M for the finite-distance factor")
    return 1.0 / math.sqrt(1.0 - 2.0 * st.mass / radius)


def boundary_error(numeric, analytic, centre, *, pixel_size: float | None = None, scale: float = 1.0) -> dict[str, float]:
    """max / rms / mean of ``r_numeric * scale - r_analytic`` (M, and px with ``pixel_size``)."""
    angles = np.asarray(numeric[0], dtype=np.float64)
    r_num = np.asarray(numeric[1], dtype=np.float64) * scale
    c = (float(centre[0]) * scale, float(centre[1]) * scale)
    r_ana = polygon_radii(analytic[0], analytic[1], c, angles)
    diff = r_num - r_ana
    out: dict[str, float] = {"max": float(np.max(np.abs(diff))), "rms": float(np.sqrt(np.mean(diff**2))),
                             "mean": float(np.mean(diff)), "mean_abs": float(np.mean(np.abs(diff))),
                             "scale": float(scale)}
    for prefix, radii in (("numeric_", r_num), ("analytic_", r_ana)):
        out.update({prefix + key: value for key, value in curve_summary(angles, radii, c).items()})
    ax, ay = polygon_centroid(analytic[0], analytic[1])
    out["analytic_centroid_alpha"], out["analytic_centroid_beta"] = ax, ay
    out["analytic_centroid_displacement"] = math.hypot(ax, ay)
    out["centroid_shift_alpha"] = out["numeric_centroid_alpha"] - ax
    out["centroid_shift_beta"] = out["numeric_centroid_beta"] - ay
    out["centroid_shift_norm"] = math.hypot(out["centroid_shift_alpha"], out["centroid_shift_beta"])
    if pixel_size is not None:
        if not pixel_size > 0.0:
            raise ValueError("pixel_size must be > 0")
        for key in [k for k in out if k != "scale" and not k.endswith("_px")]:
            out[key + "_px"] = out[key] / pixel_size
    return out


def summarise_shadow(img, *, n_angles: int = 360, n_analytic: int = 720,
                     centre: tuple[float, float] | None = None) -> dict[str, Any]:
    """Edge, analytic curve and both raw and finite-distance-corrected errors of a ShadowImage."""
    angles, radii = extract_boundary(img, n_angles=n_angles, centre=centre)
    c = mask_centroid(img.alpha, img.beta, img.captured) if centre is None else centre
    curve = analytic_boundary(img.spacetime, img.camera.inclination_deg, n_analytic)
    factor = finite_distance_scale(img.spacetime, img.camera.radius)
    return {"centre": (float(c[0]), float(c[1])), "angles": angles, "radii": radii, "analytic": curve,
            "finite_distance_scale": factor,
            "error": boundary_error((angles, radii), curve, c, pixel_size=img.pixel_size),
            "error_corrected": boundary_error((angles, radii), curve, c, pixel_size=img.pixel_size, scale=factor)}
