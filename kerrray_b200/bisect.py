"""Shadow-edge bisection on the device.

Restates ``bisect_edge`` of ``scripts/study_edge_bisection.py:53-68`` (with its ``PointCamera``,
``:39-50``): along each polar direction about an image-plane centre the image radius is halved
between a captured and an escaped photon; the integrator uses ``rtol``, ``atol = 1e-2 rtol``,
``max_steps = 2e6``, ``lambda_max = 4 r_o`` and terminates at ``r_o`` with a 1e-6 horizon
margin. Here every direction of every case is one work item of a single persistent launch
(``krr_bisect_edges``): a lane runs all the halvings of its item in registers.

:func:`edge_study` builds the reference's study set-up for one case -- the Bardeen curve's
centroid scaled by the finite-distance factor as centre, a bracket around the curve's radius
-- and :func:`edge_error` reports the edge error against the curve. Both use the exact curve
(:class:`~kerrray_b200.orbits.BardeenCurve`); the reference samples it at 40,000 points, whose
polygon lies inside the curve by up to ~1.5e-8 M.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any, Sequence

import numpy as np

from kerrray_b200 import _lib
from kerrray_b200.boundary import finite_distance_scale
from kerrray_b200.orbits import BardeenCurve
from kerrray_b200.types import IntegratorOptions, TerminationOptions

__all__ = ["EdgeCase", "bisect_edge", "bisect_edges", "edge_options", "edge_study", "item_cost"]


def edge_options(rtol: float, r_o: float) -> tuple[IntegratorOptions, TerminationOptions]:
    """The integrator and termination options of the edge study (study_edge_bisection.py:54-55)."""
    integ = IntegratorOptions(method="rk45", rtol=rtol, atol=rtol * 1e-2, max_steps=2_000_000, lambda_max=4.0 * r_o)
    return integ, TerminationOptions(horizon_epsilon=1e-6, escape_radius=r_o)


@dataclass
class EdgeCase:
    """One bisection case: spacetime, observer, tolerance, centre, directions and brackets."""

    spacetime: Any
    inclination_deg: float
    r_o: float
    rtol: float
    centre: tuple[float, float]
    angles: np.ndarray
    r_lo: np.ndarray
    r_hi: np.ndarray

    def struct(self) -> _lib.KrrEdgeCase:
        integ, term = edge_options(self.rtol, self.r_o)
        return _lib.KrrEdgeCase(mass=float(self.spacetime.mass), spin=float(self.spacetime.spin), radius=float(self.r_o),
                                inclination_deg=float(self.inclination_deg), phi_deg=0.0,
                                options=_lib.options_struct(integ, term), centre_alpha=float(self.centre[0]),
                                centre_beta=float(self.centre[1]))


def item_cost(case: EdgeCase) -> float:
    """Predicted cost of one of the case's directions relative to others: rtol^(-1/5), the
    controller's step count scaling (the same model shards the items over ranks)."""
    return float(case.rtol) ** -0.2


def bisect_edges(cases: Sequence[EdgeCase], iterations: int, *, precision: str = "reference",
                 device: int = 0, item_failures: bool = False,
                 order: str = "cost") -> tuple[list[tuple[np.ndarray, np.ndarray, object]], dict]:
    """Run every case's bisection in one launch; per case ``(r_mid, width, failures)`` and the stats.

    ``failures`` counts the photons of the case that ended neither ESCAPED nor CAPTURED (the
    reference's lost photons); with ``item_failures`` it is that count per direction (an array).
    ``order="cost"`` hands the launch's work queue the cases' directions most expensive first
    (``item_cost``), so that the cheap ones make the tail; ``"given"`` keeps the order of
    ``cases``. Each direction's result does not depend on the order.
    """
    cases = list(cases)
    if order not in ("cost", "given"):
        raise ValueError(f"order must be 'cost' or 'given', got {order!r}")
    arr = (_lib.KrrEdgeCase * len(cases))(*[c.struct() for c in cases])
    sizes = [np.asarray(c.angles).size for c in cases]
    seq = list(range(len(cases)))
    if order == "cost":
        seq.sort(key=lambda k: -item_cost(cases[k]))  # stable: equal costs keep their order
    start_of = {}
    pos = 0
    for k in seq:
        start_of[k] = pos
        pos += sizes[k]
    item_case = np.concatenate([np.full(sizes[k], k, dtype=np.int32) for k in seq])
    angles = np.concatenate([np.asarray(cases[k].angles, dtype=np.float64).ravel() for k in seq])
    cos_phi, sin_phi = np.ascontiguousarray(np.cos(angles)), np.ascontiguousarray(np.sin(angles))
    lo = np.ascontiguousarray(np.concatenate([np.broadcast_to(np.asarray(cases[k].r_lo, np.float64), (sizes[k],))
                                              for k in seq]))
    hi = np.ascontiguousarray(np.concatenate([np.broadcast_to(np.asarray(cases[k].r_hi, np.float64), (sizes[k],))
                                              for k in seq]))
    fails = np.zeros(lo.size, dtype=np.int64)
    stats = _lib.KrrStats()
    if precision not in _lib.PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_lib.PRECISIONS)}, got {precision!r}")
    rc = _lib.lib().krr_bisect_edges(device, arr, len(cases), item_case.ctypes.data, cos_phi.ctypes.data,
                                     sin_phi.ctypes.data, lo.ctypes.data, hi.ctypes.data, fails.ctypes.data, lo.size,
                                     int(iterations), _lib.PRECISIONS[precision], ctypes.byref(stats))
    _lib.check(rc)
    out = []
    for k, n in enumerate(sizes):
        sl = slice(start_of[k], start_of[k] + n)
        out.append((0.5 * (lo[sl] + hi[sl]), hi[sl] - lo[sl], fails[sl].copy() if item_failures else int(fails[sl].sum())))
    return out, stats.as_dict()


def bisect_edge(st, incl, r_o, rtol, centre, angles, r_lo, r_hi, iterations, *, precision: str = "reference",
                device: int = 0) -> tuple[np.ndarray, np.ndarray, int]:
    """``(r_mid, width, failures)`` for one case; the arguments of study_edge_bisection.bisect_edge."""
    case = EdgeCase(st, float(incl), float(r_o), float(rtol), (float(centre[0]), float(centre[1])),
                    np.asarray(angles, dtype=np.float64), np.asarray(r_lo, dtype=np.float64),
                    np.asarray(r_hi, dtype=np.float64))
    (res,), _ = bisect_edges([case], iterations, precision=precision, device=device)
    return res


def edge_study(st, incl: float, r_o: float, rtol: float, angles, *, bracket: tuple[float, float] | None = None,
               rel_bracket: float = 0.02) -> EdgeCase:
    """The study's case: centre = Bardeen centroid / k; bracket ``(1 -+ rel_bracket) r_Bardeen / k``,
    or the absolute image radii ``bracket`` about that centre."""
    k = finite_distance_scale(st, r_o)
    curve = BardeenCurve(st, float(incl))
    c_ana = curve.centroid()
    angles = np.asarray(angles, dtype=np.float64)
    if bracket is None:
        r_img = curve.radii(c_ana, angles) / k
        lo, hi = (1.0 - rel_bracket) * r_img, (1.0 + rel_bracket) * r_img
    else:
        lo, hi = np.full(angles.size, float(bracket[0])), np.full(angles.size, float(bracket[1]))
    return EdgeCase(st, incl, r_o, rtol, (c_ana[0] / k, c_ana[1] / k), angles, lo, hi)


def edge_error(case: EdgeCase, r_mid: np.ndarray, keep: np.ndarray | None = None) -> dict[str, float]:
    """Edge error against Bardeen's exact curve after the finite-distance correction (M), over the
    directions selected by ``keep`` (a boolean mask; all by default)."""
    k = finite_distance_scale(case.spacetime, case.r_o)
    r_ana = BardeenCurve(case.spacetime, case.inclination_deg).radii((case.centre[0] * k, case.centre[1] * k),
                                                                     case.angles)
    err = r_mid * k - r_ana
    if keep is not None:
        err = err[np.asarray(keep, dtype=bool)]
    return {"rms_M": float(np.sqrt(np.mean(err**2))), "max_M": float(np.max(np.abs(err))), "mean_M": float(np.mean(err))}
