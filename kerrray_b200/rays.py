"""Tracing a batch of initial states on any backend, range by range.

The ``cuda`` backend takes the whole batch in one call: the device holds it, and its host-buffer
path already overlaps the copies of consecutive photon ranges with the trace. Other backends
(KerrRay's ``numpy`` and ``numba`` objects) are called on consecutive ranges of ``chunk_size``
rows, and ``progress`` is told the fraction done after each. Every range's per-ray fields are
written into one result allocated after the first range returns (each array field at the
batch's length, with that range's dtype), so no list of partial results is kept and joined.

The reference's counterpart is ``raytracing/rays.py:72-117`` (``trace_rays``: 16,384-row
chunks joined with ``np.concatenate``); the argument meanings and the ``ValueError`` cases are
the same.
"""

from __future__ import annotations

import dataclasses
import time
from typing import Any, Callable

import numpy as np
from numpy.typing import ArrayLike

from kerrray_b200.backends import CudaBackend, get_backend
from kerrray_b200.types import STATE_SIZE, BatchResult

__all__ = ["DEFAULT_CHUNK_SIZE", "HOST_CHUNK_SIZE", "ProgressCallback", "trace_rays"]

ProgressCallback = Callable[[float], None]
DEFAULT_CHUNK_SIZE: int | None = None  # the whole batch on the cuda backend, HOST_CHUNK_SIZE elsewhere
HOST_CHUNK_SIZE = 1 << 14


def _per_ray_fields(part: Any, rows: int) -> list[str]:
    """Names of the array fields of a result that hold one entry per ray."""
    names = [f.name for f in dataclasses.fields(part)] if dataclasses.is_dataclass(part) else list(vars(part))
    return [n for n in names if isinstance(getattr(part, n), np.ndarray) and getattr(part, n).shape[:1] == (rows,)]


def trace_rays(st: Any, Y0: ArrayLike, integ: Any, term: Any, *, backend: Any = "cuda", events: Any = None,
               progress: ProgressCallback | None = None, chunk_size: int | None = DEFAULT_CHUNK_SIZE) -> BatchResult:
    """Integrate the states ``Y0`` (N x 8, N >= 1) on ``backend`` (a name or a backend object)
    and return one result over all rows, ``runtime_s`` the wall time of the whole call."""
    y0 = np.asarray(Y0)
    if y0.ndim != 2 or y0.shape[1] != STATE_SIZE:
        raise ValueError(f"Y0 must have shape (N, {STATE_SIZE}), got {y0.shape}")
    n = int(y0.shape[0])
    if n < 1:
        raise ValueError("Y0 must contain at least one ray")
    if chunk_size is not None and chunk_size < 1:
        raise ValueError(f"chunk_size must be >= 1, got {chunk_size!r}")
    engine = get_backend(backend) if isinstance(backend, str) else backend
    span = chunk_size or (n if isinstance(engine, CudaBackend) else HOST_CHUNK_SIZE)
    started = time.perf_counter()
    merged: dict[str, np.ndarray | None] = {}
    first = None
    for lo in range(0, n, span):
        hi = min(lo + span, n)
        part = engine.integrate_batch(st, y0[lo:hi], integ, term, events=events)
        if first is None:
            first = part
            if hi == n:  # a single range: its result is the batch's
                break
            merged = {name: np.empty((n,) + getattr(part, name).shape[1:], getattr(part, name).dtype)
                      for name in _per_ray_fields(part, hi - lo)}
        for name, out in merged.items():
            value = getattr(part, name, None)
            if out is not None and value is not None:
                out[lo:hi] = value
            else:
                merged[name] = None  # a field that some range does not report is not reported
        if progress is not None:
            progress(hi / n)
    assert first is not None
    elapsed = time.perf_counter() - started
    if not merged:
        if progress is not None:
            progress(1.0)
        return dataclasses.replace(first, runtime_s=elapsed)
    return dataclasses.replace(first, runtime_s=elapsed, **merged)
