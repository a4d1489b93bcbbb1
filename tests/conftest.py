"""Shared pytest set-up: the ``gpu`` marker, the repo on ``sys.path`` and golden-fixture loaders."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name: str) -> dict:
    """Load ``tests/golden/<name>.npz`` into a plain dict."""
    with np.load(GOLDEN / f"{name}.npz") as d:
        return {k: d[k] for k in d.files}


def golden_options(d: dict):
    """The oracle's ``Options`` for a fixture written by ``make_golden._run``."""
    from oracle.oracle import Options

    return Options(
        method=str(d["integ_method"]), rtol=float(d["integ_rtol"]), atol=float(d["integ_atol"]),
        step_size=float(d["integ_step_size"]), max_steps=int(d["integ_max_steps"]),
        lambda_max=float(d["integ_lambda_max"]), h_min=float(d["integ_h_min"]),
        h_max=None if np.isinf(d["integ_h_max"]) else float(d["integ_h_max"]), dtype=str(d["integ_dtype"]),
        horizon_epsilon=float(d["term_horizon_epsilon"]), escape_radius=float(d["term_escape_radius"]),
        disk_plane=bool(d.get("event_disk_plane", False)), r_in=float(d.get("event_r_in", 6.0)),
        r_out=float(d.get("event_r_out", 20.0)),
    )


TRACE_FIXTURES = (
    "shadow64_a0.9_i60", "camera24_rtol1e-8", "budget_max_steps30", "budget_lambda500", "hmax_none", "hmax_20",
    "hmax_3", "schwarzschild_6x6_rtol1e-9", "failures_512_rtol1e-4", "hmin_failure", "axis_lz0", "float32_6x6",
    "rk4_budget", "disk_float64", "disk_float32", "tangential_photons_a0",
)
