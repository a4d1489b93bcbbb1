"""Differentiable lensing map on the GPU.

For an observer (spin a*, inclination i, radius r_o) the lensing map sends an image-plane point
(alpha, beta) to the terminal celestial direction (theta_e, phi_e) of its backward photon: theta
and phi on the termination surface (the escape radius), located from the last accepted state by
one step along the flow. :func:`lensing_map` evaluates it with its Jacobian
d(theta_e, phi_e)/d(alpha, beta, a*, i) by the hand-written adjoint of the discretised
Dormand-Prince 5(4) map (``krr_lensing_adjoint``: accepted step sizes recorded, controller held
fixed, the stage inputs of every step kept in a device pool and swept back from there --
checkpoints every K steps with recomputation for the rays the pool cannot hold -- and the
event-time correction at the surface). :class:`LensingFunction` exposes it to ``torch.autograd``; :func:`magnification`
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

__all__ = ["DEFAULT_STAGE_STEPS_PER_RAY", "LensingFunction", "LensingResult", "edge_distant_rays",
           "fit_spin_inclination", "lensing_map", "magnification", "tape_usage", "workspace_bytes"]

DEG = math.pi / 180.0
# Accepted steps per ray the default stage pool is sized for (240 B each); the pool is shared,
# so it is the total that counts.  Escaping rays at rtol 1e-10 from r_o = 1000 M take about 320.
DEFAULT_STAGE_STEPS_PER_RAY = 512


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
        L.krr_lensing_workspace_size_staged.restype = ctypes.c_size_t
        L.krr_lensing_workspace_size_staged.argtypes = [i64, i32, i32, i64]
        L.krr_lensing_tape_usage.restype = ctypes.c_int
        L.krr_lensing_tape_usage.argtypes = [ctypes.POINTER(KrrLensParams), i64, vp, ctypes.c_size_t,
                                             ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64), vp]
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
    perm: Any = None  # the order the rays were traced in (input indices), None: the input order


def _params(spin, inclination_deg, r_o, mass, integ, term, checkpoint_every, tape_capacity) -> KrrLensParams:
    integ = integ or IntegratorOptions(method="rk45", rtol=1e-10, atol=1e-12)
    term = term or TerminationOptions(escape_radius=r_o)
    return KrrLensParams(mass=float(mass), spin=float(spin), radius=float(r_o), inclination_deg=float(inclination_deg),
                         phi_deg=0.0, options=_lib.options_struct(integ, term), checkpoint_every=int(checkpoint_every),
                         tape_capacity=int(tape_capacity))


def lensing_map(alpha, beta, spin: float, inclination_deg: float, *, r_o: float = 1000.0, mass: float = 1.0,
                integ=None, term=None, checkpoint_every: int = 32, tape_capacity: int = 8192,
                stage_steps: int | None = None, workspace=None, order: Any = "impact",
                device: int = 0) -> LensingResult:
    """Map and Jacobian for image points ``alpha``, ``beta`` (torch float64 tensors on the device).

    ``stage_steps`` sizes the stage pool in accepted steps over all rays (default
    ``DEFAULT_STAGE_STEPS_PER_RAY`` per ray; 0: no pool, every ray's sweep recomputes from
    checkpoints).  Rays beyond the pool fall back to recomputation: same derivative to rounding.
    ``workspace``: a uint8 tensor on the device to hold the tape instead of a fresh allocation
    (any size from ``workspace_bytes(...)`` up: bytes beyond the minimum become stage pool); the
    result keeps it for ``replay`` until the next call given the same tensor.

    ``order``: the order the rays are traced in, one ray per thread. A warp lasts as long as its
    longest ray, so rays of like length belong together, the longest first. ``"impact"`` (the
    default) traces them by increasing impact parameter hypot(alpha, beta): an escaping ray's
    step count falls as it passes farther from the hole. A tensor of per-ray costs -- the step
    counts of an earlier map of the same rays, as a fit has them -- traces them by decreasing
    cost; ``"given"`` keeps the input order. The results come back in the input order, and are
    the same bit for bit in every order."""
    import torch

    L = _bind()
    dev = torch.device("cuda", device)
    a = alpha.to(dev, torch.float64).contiguous()
    b = beta.to(dev, torch.float64).contiguous()
    n = a.numel()
    perm = _trace_order(order, a, b)
    if perm is not None:
        a, b = a[perm].contiguous(), b[perm].contiguous()
    p = _params(spin, inclination_deg, r_o, mass, integ, term, checkpoint_every, tape_capacity)
    if workspace is not None:
        need = int(L.krr_lensing_workspace_size(n, p.tape_capacity, p.checkpoint_every))
        if workspace.dtype != torch.uint8 or workspace.device != dev or workspace.numel() < need:
            raise ValueError(f"workspace must be a uint8 tensor on {dev} of at least {need} bytes")
        ws = workspace
    else:
        ws = torch.empty(max(workspace_bytes(n, checkpoint_every=checkpoint_every, tape_capacity=tape_capacity,
                                             stage_steps=stage_steps), 8), dtype=torch.uint8, device=dev)
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
    if perm is not None:
        theta, phi, jac, state, steps, status = (_unpermute(x, perm) for x in (theta, phi, jac, state, steps, status))
    return LensingResult(theta, phi, jac, state, steps, status, ws, p, perm)


def _trace_order(order, alpha, beta):
    """The permutation (input indices in trace order) that ``order`` asks for, or None."""
    import torch

    if isinstance(order, str):
        if order == "given":
            return None
        if order == "impact":
            return torch.argsort(torch.hypot(alpha, beta), stable=True)
        raise ValueError(f"order must be 'impact', 'given' or a tensor of per-ray costs, got {order!r}")
    cost = torch.as_tensor(order, device=alpha.device)
    if cost.shape != alpha.shape:
        raise ValueError(f"order: one cost per ray expected, shape {tuple(alpha.shape)}, got {tuple(cost.shape)}")
    return torch.argsort(cost.to(torch.float64), descending=True, stable=True)


def _unpermute(x, perm):
    """Rows of ``x`` (in trace order) back in input order."""
    import torch

    out = torch.empty_like(x)
    out[perm] = x
    return out


def workspace_bytes(n: int, *, checkpoint_every: int = 32, tape_capacity: int = 8192,
                    stage_steps: int | None = None) -> int:
    """Bytes of the tape for ``n`` rays with a stage pool of ``stage_steps`` accepted steps in all
    (default ``DEFAULT_STAGE_STEPS_PER_RAY`` per ray; 0: the minimum, no pool)."""
    if stage_steps is None:
        stage_steps = n * DEFAULT_STAGE_STEPS_PER_RAY
    if stage_steps < 0:
        raise ValueError(f"stage_steps must be >= 0, got {stage_steps}")
    size = int(_bind().krr_lensing_workspace_size_staged(int(n), int(tape_capacity), int(checkpoint_every),
                                                         int(stage_steps)))
    if size == 0 and n > 0:
        raise ValueError("invalid tape_capacity or checkpoint_every")
    return size


def tape_usage(res: LensingResult, device: int = 0) -> dict[str, int]:
    """Of ``res``'s rays: how many were swept from the stage pool, and the pool's chunks used/held."""
    import torch

    L = _bind()
    staged, used, total = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(L.krr_lensing_tape_usage(ctypes.byref(res.params), res.theta.numel(), res.workspace.data_ptr(),
                                        res.workspace.numel(), ctypes.byref(staged), ctypes.byref(used),
                                        ctypes.byref(total), stream))
    return {"staged_rays": staged.value, "chunks_used": used.value, "chunks_total": total.value}


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
    state, steps = res.state, res.n_steps
    if res.perm is not None:  # the tape holds the rays in their trace order
        a, b = a[res.perm].contiguous(), b[res.perm].contiguous()
        state, steps = state[res.perm].contiguous(), steps[res.perm].contiguous()
    theta = torch.empty(n, dtype=torch.float64, device=dev)
    phi = torch.empty_like(theta)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(L.krr_lensing_replay(device, ctypes.byref(p), a.data_ptr(), b.data_ptr(), n, state.data_ptr(),
                                    steps.data_ptr(), theta.data_ptr(), phi.data_ptr(), status.data_ptr(),
                                    res.workspace.data_ptr(), res.workspace.numel(), stream))
    if res.perm is not None:
        theta, phi = _unpermute(theta, res.perm), _unpermute(phi, res.perm)
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
                def forward(ctx, a, b, s, i, options):
                    res = lensing_map(a.detach(), b.detach(), float(s), float(i), **options)
                    ctx.save_for_backward(res.jac)
                    return res.theta, res.phi

                @staticmethod
                def backward(ctx, g_theta, g_phi):
                    (jac,) = ctx.saved_tensors
                    g = g_theta[:, None] * jac[:, 0, :] + g_phi[:, None] * jac[:, 1, :]
                    return g[:, 0], g[:, 1], g[:, 2].sum().reshape(()), g[:, 3].sum().reshape(()), None

            cls._fn = _F
        # lensing_map's keyword options go in as a plain (non-tensor) argument of this call
        return cls._fn.apply(alpha, beta, spin, inclination_deg, dict(kw))


def fit_spin_inclination(alpha, beta, target_theta, target_phi, *, p0=(0.5, 50.0), iterations: int = 20,
                         r_o: float = 1000.0, integ=None, device: int = 0, tol: float = 0.0,
                         robust: bool = True, leverage: float | None = 3.0) -> dict:
    """Fit (a*, i) so that the lensing map matches ``(target_theta, target_phi)``.

    Damped Gauss-Newton (Levenberg-Marquardt): the normal equations of the (a*, i) columns of the
    adjoint Jacobian, ``(J^T W J + lambda diag(J^T W J)) d = -J^T W r``, a trial step accepted when
    the cost falls (lambda / 3) and retried with lambda x 4 otherwise. Residuals are theta and phi
    differences with phi wrapped to (-pi, pi]; a ray that does not escape at the evaluated
    parameters (or whose target is not finite) gets the residual pi. With ``robust`` the weights
    W are Cauchy's, ``1 / (1 + (r / s)^2)`` with ``s`` = 1.4826 x the median absolute residual at
    the current point. With ``leverage`` the weights are further multiplied by
    ``1 / (1 + (l / leverage)^2)``, ``l`` the norm of the row's (a*, i) derivatives in units of
    their median over the rays: strongly lensed rays near the shadow edge (|d phi / d a*| up to
    ~1e2 against ~4e-2 for the rest) otherwise dominate the normal equations although their
    linearisation fails a few tenths away in spin. Positive weights leave the minimiser of a
    target the map itself produced (zero residual) unchanged.
    """
    import torch

    targets_ok = torch.isfinite(target_theta) & torch.isfinite(target_phi)
    evaluations = 0
    # One tape for every evaluation: the fit reads each result's map and Jacobian, never its tape.
    ws = torch.empty(workspace_bytes(alpha.numel()), dtype=torch.uint8, device=torch.device("cuda", device))

    hint = "impact"  # then each evaluation's step counts order the next one's rays

    def evaluate(q):
        nonlocal evaluations, hint
        evaluations += 1
        res = lensing_map(alpha, beta, float(q[0]), float(q[1]), r_o=r_o, integ=integ, workspace=ws, order=hint,
                          device=device)
        hint = res.n_steps
        ok = (res.status == 0) & (res.state == 1) & targets_ok
        d_th = res.theta - target_theta
        d_ph = torch.remainder(res.phi - target_phi + math.pi, 2.0 * math.pi) - math.pi
        r = torch.stack([d_th, d_ph], dim=1)
        r = torch.where(ok[:, None], r, torch.full_like(r, math.pi))
        return res, r, ok

    def cost(r, scale, lev_w):
        rho = 0.5 * r * r if scale is None else 0.5 * scale * scale * torch.log1p((r / scale) ** 2)
        return float((lev_w * rho).sum().item())

    def clip(q):
        return np.array([float(np.clip(q[0], -0.999, 0.999)), float(np.clip(q[1], 1e-3, 180.0 - 1e-3))])

    p = clip(np.array(p0, dtype=np.float64))
    res, r, ok = evaluate(p)
    lam = 1e-3
    history = []
    for it in range(iterations):
        scale = None
        w = ok.to(torch.float64)[:, None].expand(-1, 2)
        lev_w = torch.ones_like(r)
        if robust:
            med = float(r[ok].abs().median().item()) if bool(ok.any()) else 0.0
            scale = max(1.4826 * med, 1e-15)
            w = w / (1.0 + (r / scale) ** 2)
        J = res.jac[:, :, 2:]  # d(theta, phi)/d(spin, inclination [deg]); zero rows where not ok
        J = torch.where(ok[:, None, None], J, torch.zeros_like(J))
        if leverage and bool(ok.any()):
            med = J[ok].abs().reshape(-1, 2).median(dim=0).values.clamp_min(1e-300)
            lev = torch.linalg.vector_norm(J / med, dim=2) / math.sqrt(2.0)
            lev_w = 1.0 / (1.0 + (lev / leverage) ** 2)
            w = w * lev_w
        A = torch.einsum("nc,nci,ncj->ij", w, J, J)
        g = torch.einsum("nc,nci,nc->i", w, J, r)
        c0 = cost(r, scale, lev_w)
        history.append({"iteration": it, "spin": float(p[0]), "inclination_deg": float(p[1]),
                        "cost": float(0.5 * (r[ok] ** 2).sum().item()), "rays": int(ok.sum().item()),
                        "damping": lam})
        step = np.zeros(2)
        accepted = False
        for _ in range(12):
            M = A + lam * torch.diag(torch.diagonal(A))
            step = torch.linalg.solve(M, -g).cpu().numpy()
            q = clip(p + step)
            res_q, r_q, ok_q = evaluate(q)
            if cost(r_q, scale, lev_w) < c0:
                p, res, r, ok = q, res_q, r_q, ok_q
                lam = max(lam / 3.0, 1e-12)
                accepted = True
                break
            lam *= 4.0
        if not accepted or (tol and np.all(np.abs(step) < tol)):
            break
    history.append({"iteration": len(history), "spin": float(p[0]), "inclination_deg": float(p[1]),
                    "cost": float(0.5 * (r[ok] ** 2).sum().item()), "rays": int(ok.sum().item()), "damping": lam})
    return {"spin": float(p[0]), "inclination_deg": float(p[1]), "history": history, "evaluations": evaluations}


def edge_distant_rays(spin: float, inclination_deg: float, *, r_o: float = 1000.0, fov: float = 12.0,
                      resolution: int = 256, margin_px: float = 3.0, rtol: float = 1e-10, precision: str = "fast64",
                      device: int = 0):
    """Image points ``(alpha, beta)`` (torch float64 on the device) of the escaped pixels of a
    ``resolution``^2 image over +-``fov`` M that lie more than ``margin_px`` pixels from every
    pixel that did not escape: the rays on which the lensing map is smooth. The image is traced
    on the device (rk45 at ``rtol``, ``atol = 1e-2 rtol``, escape at ``r_o``)."""
    import torch
    from scipy.ndimage import distance_transform_edt

    from kerrray_b200.camera import Camera
    from kerrray_b200.sweep import ImageSpec, trace_images
    from kerrray_b200.types import Spacetime, TerminationState

    cam = Camera(radius=r_o, inclination_deg=inclination_deg, fov=fov, resolution=resolution)
    spec = ImageSpec(Spacetime(1.0, spin), cam, IntegratorOptions(method="rk45", rtol=rtol, atol=1e-2 * rtol),
                     TerminationOptions(escape_radius=r_o))
    res = trace_images([spec], precision=precision, device=device)
    escaped = (res.arrays["state"] == TerminationState.ESCAPED).reshape(cam.shape)
    keep = escaped & (distance_transform_edt(escaped) > margin_px)
    alpha, beta = cam.pixel_coordinates()
    dev = torch.device("cuda", device)
    return (torch.tensor(np.asarray(alpha)[keep], dtype=torch.float64, device=dev),
            torch.tensor(np.asarray(beta)[keep], dtype=torch.float64, device=dev))
