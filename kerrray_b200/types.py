"""Value types of the hot path, with the reference's fields, defaults and validation.

* :class:`Spacetime` -- ``src/kerrray/geometry/metric.py:66-98``
* :func:`outer_horizon` -- ``src/kerrray/geometry/horizons.py:33-42``
* :class:`IntegratorOptions`, :class:`TerminationOptions`, :class:`EventOptions`,
  :func:`max_attempts` -- ``src/kerrray/geodesics/integrators.py:71-162``
* :class:`TerminationState` -- ``src/kerrray/photons/classification.py:60-69``
* :class:`BatchResult` -- ``src/kerrray/photons/trajectories.py:99-137``

Every backend entry point of this package also accepts the reference's own objects (it reads
the same attribute names), so a KerrRay caller passes its ``Spacetime`` and option objects
unchanged.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from enum import IntEnum

import numpy as np
from numpy.typing import NDArray

SAFETY = 0.9
FACTOR_MAX = 5.0
STATE_SIZE = 8
IDX_T, IDX_R, IDX_TH, IDX_PH, IDX_PT, IDX_PR, IDX_PTH, IDX_PPH = range(8)
SUPPORTED_METHODS = frozenset({"rk4", "rk45", "dop853"})


@dataclass(frozen=True)
class Spacetime:
    """A Kerr (or Schwarzschild) black hole in geometric units: ``mass > 0``, ``|spin| < 1``."""

    mass: float = 1.0
    spin: float = 0.0

    def __post_init__(self) -> None:
        mass, spin = float(self.mass), float(self.spin)
        if not (math.isfinite(mass) and mass > 0.0):
            raise ValueError(f"mass must be a finite number > 0, got {self.mass!r}")
        if not (math.isfinite(spin) and abs(spin) < 1.0):
            raise ValueError(f"spin must satisfy abs(spin) < 1, got {self.spin!r}")
        object.__setattr__(self, "mass", mass)
        object.__setattr__(self, "spin", spin)

    @property
    def a(self) -> float:
        """Kerr parameter ``a = spin * mass``."""
        return self.spin * self.mass

    @property
    def is_schwarzschild(self) -> bool:
        return self.spin == 0.0


def outer_horizon(st) -> float:
    """``r_plus = M + sqrt(M^2 - a^2)``."""
    m = st.mass
    return m + math.sqrt(m * m - st.a * st.a)


@dataclass(frozen=True)
class IntegratorOptions:
    """Integration scheme, tolerances and budgets (defaults as the reference)."""

    method: str = "rk45"
    rtol: float = 1e-9
    atol: float = 1e-11
    step_size: float = 0.01
    max_steps: int = 100_000
    lambda_max: float = 1.0e4
    h_min: float = 1e-12
    dtype: str = "float64"
    h_max: float | None = None

    def __post_init__(self) -> None:
        if self.method not in SUPPORTED_METHODS:
            raise ValueError(f"method must be one of {sorted(SUPPORTED_METHODS)}, got {self.method!r}")
        for name in ("rtol", "atol", "step_size", "lambda_max", "h_min"):
            value = getattr(self, name)
            if not (math.isfinite(value) and value > 0.0):
                raise ValueError(f"{name} must be a finite number > 0, got {value!r}")
        if self.h_max is not None and not (math.isfinite(self.h_max) and self.h_max > 0.0):
            raise ValueError(f"h_max must be None or a finite number > 0, got {self.h_max!r}")
        if self.max_steps < 1:
            raise ValueError(f"max_steps must be >= 1, got {self.max_steps!r}")
        if self.dtype not in ("float32", "float64"):
            raise ValueError(f"dtype must be 'float32' or 'float64', got {self.dtype!r}")

    @property
    def np_dtype(self) -> np.dtype:
        return np.dtype(self.dtype)


@dataclass(frozen=True)
class TerminationOptions:
    """Capture margin and escape radius."""

    horizon_epsilon: float = 1e-6
    escape_radius: float = 1000.0

    def __post_init__(self) -> None:
        if not (math.isfinite(self.horizon_epsilon) and self.horizon_epsilon >= 0.0):
            raise ValueError(f"horizon_epsilon must be >= 0, got {self.horizon_epsilon!r}")
        if not (math.isfinite(self.escape_radius) and self.escape_radius > 0.0):
            raise ValueError(f"escape_radius must be > 0, got {self.escape_radius!r}")


@dataclass(frozen=True)
class EventOptions:
    """Optional equatorial disk-plane event (stop as DISK_HIT when theta crosses pi/2 in [r_in, r_out])."""

    disk_plane: bool = False
    r_in: float = 6.0
    r_out: float = 20.0

    def __post_init__(self) -> None:
        if not (0.0 < self.r_in <= self.r_out):
            raise ValueError(f"need 0 < r_in <= r_out, got r_in={self.r_in!r}, r_out={self.r_out!r}")


def max_attempts(integ) -> int:
    """Upper bound on step attempts before ``h < h_min`` (the defensive loop guard)."""
    h_max = max(integ.lambda_max, integ.step_size)
    rej = (math.log(h_max / integ.h_min) + integ.max_steps * math.log(FACTOR_MAX)) / math.log(1.0 / SAFETY)
    return integ.max_steps + int(math.ceil(rej)) + 1


class TerminationState(IntEnum):
    """Why a ray stopped (``RUNNING`` is the internal 'not yet' value)."""

    RUNNING = 0
    ESCAPED = 1
    CAPTURED = 2
    MAX_AFFINE_PARAMETER = 3
    NUMERICAL_FAILURE = 4
    OUT_OF_DOMAIN = 5
    DISK_HIT = 6


@dataclass
class BatchResult:
    """Final states and per-ray summaries of a batch (fields and dtypes as the reference).

    ``max_null_error``, ``max_energy_drift``, ``max_lz_drift`` and ``max_carter_drift`` are the
    running maxima over accepted steps. From the ``cuda`` backend in its ``"mixed"`` precision
    they are evaluated in FP32 from the FP32 copy of each accepted state, so they measure that
    copy's round-off (about 1e-7 relative) rather than the FP64 integration's drift."""

    Y: NDArray
    state: NDArray[np.int64]
    n_steps: NDArray[np.int64]
    lam: NDArray[np.float64]
    max_null_error: NDArray[np.float64]
    max_energy_drift: NDArray[np.float64]
    max_lz_drift: NDArray[np.float64]
    max_carter_drift: NDArray[np.float64]
    runtime_s: float
    event_Y: NDArray | None = None
    event_hit: NDArray[np.bool_] | None = None
    n_rejected: NDArray[np.int64] | None = None

    @property
    def n_rays(self) -> int:
        return int(self.Y.shape[0])

    def count(self, state: TerminationState) -> int:
        return int(np.count_nonzero(self.state == int(state)))
