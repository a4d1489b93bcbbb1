"""Chunked tracing over any backend (``src/kerrray/raytracing/rays.py:31-117``).

The ``cuda`` backend holds a whole image in device memory, so its default chunk is the whole
batch; ``chunk_size`` keeps the reference's meaning (and its progress callback) for callers
that want it.
"""

from __future__ import annotations

import time
from typing import Any, Callable

import numpy as np
from numpy.typing import ArrayLike, NDArray

from kerrray_b200.backends import get_backend
from kerrray_b200.types import STATE_SIZE, BatchResult

__all__ = ["DEFAULT_CHUNK_SIZE", "ProgressCallback", "concatenate_results", "trace_rays"]

DEFAULT_CHUNK_SIZE = 1 << 24
ProgressCallback = Callable[[float], None]


def _optional_concat(parts: list[NDArray | None]) -> NDArray | None:
    if any(part is None for part in parts):
        return None
    return np.concatenate([part for part in parts if part is not None], axis=0)


def concatenate_results(parts: list[Any], runtime_s: float | None = None) -> BatchResult:
    """Join the per-ray fields of ``parts`` in order into one ``BatchResult``."""
    if not parts:
        raise ValueError("concatenate_results needs at least one BatchResult")
    if len(parts) == 1 and runtime_s is None:
        return parts[0]
    cls = type(parts[0])
    return cls(
        Y=np.concatenate([p.Y for p in parts], axis=0),
        state=np.concatenate([p.state for p in parts]),
        n_steps=np.concatenate([p.n_steps for p in parts]),
        lam=np.concatenate([p.lam for p in parts]),
        max_null_error=np.concatenate([p.max_null_error for p in parts]),
        max_energy_drift=np.concatenate([p.max_energy_drift for p in parts]),
        max_lz_drift=np.concatenate([p.max_lz_drift for p in parts]),
        max_carter_drift=np.concatenate([p.max_carter_drift for p in parts]),
        runtime_s=float(sum(p.runtime_s for p in parts)) if runtime_s is None else float(runtime_s),
        event_Y=_optional_concat([p.event_Y for p in parts]),
        event_hit=_optional_concat([p.event_hit for p in parts]),
        n_rejected=_optional_concat([p.n_rejected for p in parts]),
    )


def trace_rays(st: Any, Y0: ArrayLike, integ: Any, term: Any, *, backend: Any = "cuda", events: Any = None,
               progress: ProgressCallback | None = None, chunk_size: int = DEFAULT_CHUNK_SIZE) -> BatchResult:
    """Integrate the states ``Y0`` (N, 8), ``N >= 1``, in chunks on ``backend``."""
    y0 = np.asarray(Y0)
    if y0.ndim != 2 or y0.shape[1] != STATE_SIZE:
        raise ValueError(f"Y0 must have shape (N, {STATE_SIZE}), got {y0.shape}")
    n_rays = y0.shape[0]
    if n_rays < 1:
        raise ValueError("Y0 must contain at least one ray")
    if chunk_size < 1:
        raise ValueError(f"chunk_size must be >= 1, got {chunk_size!r}")
    engine = get_backend(backend) if isinstance(backend, str) else backend
    t0 = time.perf_counter()
    parts = []
    for start in range(0, n_rays, chunk_size):
        stop = min(start + chunk_size, n_rays)
        parts.append(engine.integrate_batch(st, y0[start:stop], integ, term, events=events))
        if progress is not None:
            progress(stop / n_rays)
    return concatenate_results(parts, runtime_s=time.perf_counter() - t0)
