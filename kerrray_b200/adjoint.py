"""Differentiable lensing map on the GPU.

For an observer (spin a*, inclination i, radius r_o) the lensing map sends an image-plane point
(alpha, beta) to the terminal celestial direction (theta_e, phi_e) of its backward photon: theta
and phi on the termination surface (the escape radius), located from the last accepted state by
one step along the flow. :func:`lensing_map` evaluates it with its Jacobian
d(theta_e, phi_e)/d(alpha, beta, a*, i) by the hand-written adjoint of the discretised
Dormand-Prince 5(4) map (``krr_lensing_adjoint``: accepted step sizes recorded, controller held
fixed, checkpoints every K steps, recomputation in the reverse sweep, event-time correction at
the surface). :class:`LensingFunction` exposes it to ``torch.autograd``; :func:`magnification`
is the inverse determinant of the (alpha, beta) block; :func:`fit_spin_inclination` is a
Gauss-Newton fit of (a*, i) to a target map.

Inclination derivatives are per degree in the Python API (the C ABI returns per radian).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any

import numpy as np

from kerrray_b200 import _lib
from kerrray_b200.types import IntegratorOptions, TerminationOptions

__all__ = ["LensingFunction", "LensingResult", "fit_spin_inclination", "lensing_map", "magnification"]

DEG = math.pi / 180.0


class KrrLensParams(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("spin", ctypes.c_double), ("radius", ctypes.c_double),
                ("inclination_deg", ctypes.c_double), ("phi_deg", ctypes.c_double), ("options", _lib.KrrOptions),
                ("checkpoint_every", ctypes.c_int32), ("tape_capacity", ctypes.c_int32)]


def _bind():
    L = _lib.lib()
    if not getattr(L, "_krr_lens_bound", False):
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
        L.krr_lensing_workspace_size.restype = ctypes.c_size_t
        L.krr_lensing_workspace_size.argtypes = [i64, i32, i32]
        L.krr_lensing_adjoint.restype = ctypes.c_int
        L.krr_lensing_adjoint.argtypes = [ctypes.c_int, ctypes.POINTER(KrrLensParams), vp, vp, i64, vp, vp, vp, vp, vp,
                                          vp, vp, ctypes.c_size_t, vp]
        L.krr_lensing_replay.restype = ctypes.c_int
        L.krr_lensing_replay.argtypes = [ctypes.c_int, ctypes.POINTER(KrrLensParams), vp, vp, i64, vp, vp, vp, vp, vp,
                                         vp, ctypes.c_size_t, vp]
        L._krr_lens_bound = True
    return L


@dataclass
class LensingResult:
    theta: Any        # (n,) terminal theta on the escape surface
    phi: Any          # (n,)
    jac: Any          # (n, 2, 4): d(theta, phi)/d(alpha, beta, spin, inclination [deg])
    state: Any        # (n,) termination codes
    n_steps: Any      # (n,) accepted steps (the recorded sequence)
    status: Any       # (n,) 0 ok, 1 tape full, 2 neither escaped nor captured
    workspace: Any    # the tape (kept for replay)
    params: KrrLensParams


def _params(spin, inclination_deg, r_o, mass, integ, term, checkpoint_every, tape_capacity) -> KrrLensParams:
    integ = integ or IntegratorOptions(method="rk45", rtol=1e-10, atol=1e-12)
    term = term or TerminationOptions(escape_radius=r_o)
    return KrrLensParams(mass=float(mass), spin=float(spin), radius=float(r_o), inclination_deg=float(inclination_deg),
                         phi_deg=0.0, options=_lib.options_struct(integ, term), checkpoint_every=int(checkpoint_every),
                         tape_capacity=int(tape_capacity))


def lensing_map(alpha, beta, spin: float, inclination_deg: float, *, r_o: float = 1000.0, mass: float = 1.0,
                integ=None, term=None, checkpoint_every: int = 32, tape_capacity: int = 8192,
                device: int = 0) -> LensingResult:
    """Map and Jacobian for image points ``alpha``, ``beta`` (torch float64 tensors on the device)."""
    import torch

    L = _bind()
    dev = torch.device("cuda", device)
    a = alpha.to(dev, torch.float64).contiguous()
    b = beta.to(dev, torch.float64).contiguous()
    n = a.numel()
    p = _params(spin, inclination_deg, r_o, mass, integ, term, checkpoint_every, tape_capacity)
    ws_bytes = int(L.krr_lensing_workspace_size(n, p.tape_capacity, p.checkpoint_every))
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=dev)
    theta = torch.empty(n, dtype=torch.float64, device=dev)
    phi = torch.empty_like(theta)
    jac = torch.empty((n, 2, 4), dtype=torch.float64, device=dev)
    state = torch.empty(n, dtype=torch.int64, device=dev)
    steps = torch.empty(n, dtype=torch.int64, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(L.krr_lensing_adjoint(device, ctypes.byref(p), a.data_ptr(), b.data_ptr(), n, theta.data_ptr(),
                                     phi.data_ptr(), jac.data_ptr(), state.data_ptr(), steps.data_ptr(),
                                     status.data_ptr(), ws.data_ptr(), ws.numel(), stream))
    jac[:, :, 3] *= DEG  # per degree of inclination
    return LensingResult(theta, phi, jac, state, steps, status, ws, p)


def replay(res: LensingResult, alpha, beta, spin: float, inclination_deg: float, device: int = 0):
    """The map with ``res``'s recorded step sequence at other inputs (the map the adjoint differentiates)."""
    import torch

    L = _bind()
    p = KrrLensParams.from_buffer_copy(res.params)
    p.spin = float(spin)
    p.inclination_deg = float(inclination_deg)
    dev = res.theta.device
    a = alpha.to(dev, torch.float64).contiguous()
    b = beta.to(dev, torch.float64).contiguous()
    n = a.numel()
    theta = torch.empty(n, dtype=torch.float64, device=dev)
    phi = torch.empty_like(theta)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(L.krr_lensing_replay(device, ctypes.byref(p), a.data_ptr(), b.data_ptr(), n, res.state.data_ptr(),
                                    res.n_steps.data_ptr(), theta.data_ptr(), phi.data_ptr(), status.data_ptr(),
                                    res.workspace.data_ptr(), res.workspace.numel(), stream))
    return theta, phi


def magnification(jac) -> Any:
    """|det d(theta, phi)/d(alpha, beta)|^-1 per ray (the lensing map's area distortion)."""
    det = jac[:, 0, 0] * jac[:, 1, 1] - jac[:, 0, 1] * jac[:, 1, 0]
    return 1.0 / det.abs()


class LensingFunction:
    """``torch.autograd.Function`` of the lensing map: ``apply(alpha, beta, spin, inclination_deg)``
    -> ``(theta, phi)`` with gradients to all four inputs (spin and inclination are 0-d tensors)."""

    _fn = None

    @classmethod
    def apply(cls, alpha, beta, spin, inclination_deg, **kw):
        if cls._fn is None:
            import torch

            class _F(torch.autograd.Function):
                @staticmethod
                def forward(ctx, a, b, s, i):
                    res = lensing_map(a.detach(), b.detach(), float(s), float(i), **ctx_kw)
                    ctx.save_for_backward(res.jac)
                    return res.theta, res.phi

                @staticmethod
                def backward(ctx, g_theta, g_phi):
                    (jac,) = ctx.saved_tensors
                    g = g_theta[:, None] * jac[:, 0, :] + g_phi[:, None] * jac[:, 1, :]
                    return g[:, 0], g[:, 1], g[:, 2].sum().reshape(()), g[:, 3].sum().reshape(())

            cls._fn = _F
        global ctx_kw
        ctx_kw = kw
        return cls._fn.apply(alpha, beta, spin, inclination_deg)


ctx_kw: dict = {}


def fit_spin_inclination(alpha, beta, target_theta, target_phi, *, p0=(0.5, 50.0), iterations: int = 20,
                         r_o: float = 1000.0, integ=None, device: int = 0, tol: float = 0.0) -> dict:
    """Gauss-Newton fit of (a*, i) minimising |map(a*, i) - target|^2 over the rays that escape."""
    import torch

    p = np.array(p0, dtype=np.float64)
    history = []
    for it in range(iterations):
        res = lensing_map(alpha, beta, p[0], p[1], r_o=r_o, integ=integ, device=device)
        ok = (res.status == 0) & (res.state == 1) & torch.isfinite(target_theta) & torch.isfinite(target_phi)
        r = torch.cat([(res.theta - target_theta)[ok], (res.phi - target_phi)[ok]])
        J = torch.cat([res.jac[ok][:, 0, 2:], res.jac[ok][:, 1, 2:]])  # d/d(spin, incl_deg)
        step = torch.linalg.lstsq(J, -r[:, None]).solution[:, 0].cpu().numpy()
        cost = float((r * r).sum().item())
        history.append({"iteration": it, "spin": float(p[0]), "inclination_deg": float(p[1]), "cost": cost,
                        "rays": int(ok.sum().item())})
        p = p + step
        p[0] = float(np.clip(p[0], -0.999, 0.999))
        if tol and np.all(np.abs(step) < tol):
            break
    return {"spin": float(p[0]), "inclination_deg": float(p[1]), "history": history}
