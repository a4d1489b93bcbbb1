"""Accuracy of the step kernels' own sine and cosine forms (``krr_trig_eval``) against FP64
``numpy.sin``/``numpy.cos`` (correctly rounded to well below an FP32 unit):

- the FP32 sine/cosine of an FP64 angle (Cody-Waite reduction by pi/2, Taylor series on packed
  pairs) used for the mixed mode's accepted states: within 2 FP32 units of the value, including
  next to the axis, where the value is small and an FP32 argument would lose it;
- the FP32 small-angle shift used by the mixed stages, over the range where the kernel uses it
  (|sin theta0| >= 1/50, |delta| <= 1/4): within 4 FP32 units of 1 (absolute);
- the FP64 shift used by the fast64 stages (|delta| <= 1/10): within 4 FP64 units of 1.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

K = pytest.importorskip("kerrray_b200")
torch = pytest.importorskip("torch")


def _on_device(x: np.ndarray):
    return torch.tensor(x, dtype=torch.float64, device="cuda")


def test_reduced_sincos_within_two_fp32_units() -> None:
    rng = np.random.default_rng(11)
    th = np.concatenate([
        rng.uniform(-20.0, 20.0, 1_000_000),                         # several turns
        np.pi + rng.uniform(-1e-3, 1e-3, 100_000),                   # next to theta = pi
        rng.uniform(-1e-3, 1e-3, 100_000),                           # next to theta = 0
        np.pi * rng.integers(-6, 7, 100_000) + rng.uniform(-1e-9, 1e-9, 100_000),
        0.5 * np.pi + rng.uniform(-1e-4, 1e-4, 100_000),             # quadrant boundaries
        0.25 * np.pi * rng.integers(-12, 13, 100_000) + rng.uniform(-1e-7, 1e-7, 100_000),
    ])
    s, c = K.trig_eval(0, _on_device(th))
    s, c = s.cpu().numpy(), c.cpu().numpy()
    for got, true in ((s, np.sin(th)), (c, np.cos(th))):
        unit = np.spacing(np.abs(true).astype(np.float32)).astype(np.float64)
        err = np.abs(got - true) / unit
        print("reduced sincos: max error", err.max(), "FP32 units")
        assert err.max() <= 2.0
        # the values are FP32 numbers
        assert np.array_equal(got, got.astype(np.float32).astype(np.float64))


def test_fp32_shift_within_range() -> None:
    rng = np.random.default_rng(12)
    th0 = rng.uniform(0.0, np.pi, 1_000_000)
    th0 = th0[np.abs(np.sin(th0)) >= 0.02]
    d = rng.uniform(-0.25, 0.25, th0.size)
    s, c = K.trig_eval(1, _on_device(th0), _on_device(d))
    s, c = s.cpu().numpy(), c.cpu().numpy()
    arg = th0 + d.astype(np.float32).astype(np.float64)
    err = max(np.abs(s - np.sin(arg)).max(), np.abs(c - np.cos(arg)).max())
    print("FP32 shift: max absolute error", err)
    assert err <= 4 * 2.0 ** -24
    # outside the series' range the shift declines (the kernel then evaluates the angle itself)
    s_out, _ = K.trig_eval(1, _on_device(np.array([1.0, 1.0])), _on_device(np.array([0.3, -0.26])))
    assert np.all(np.isnan(s_out.cpu().numpy()))


def test_fp64_shift_within_range() -> None:
    rng = np.random.default_rng(13)
    th0 = rng.uniform(-4.0, 4.0, 1_000_000)
    d = rng.uniform(-0.1, 0.1, th0.size)
    s, c = K.trig_eval(2, _on_device(th0), _on_device(d))
    s, c = s.cpu().numpy(), c.cpu().numpy()
    # true values of sin/cos(th0 + d) without rounding th0 + d: angle addition in FP64 around
    # numpy's correctly rounded sin/cos of th0 and of d (error ~1e-16 absolute)
    ts = np.sin(th0) * np.cos(d) + np.cos(th0) * np.sin(d)
    tc = np.cos(th0) * np.cos(d) - np.sin(th0) * np.sin(d)
    err = max(np.abs(s - ts).max(), np.abs(c - tc).max())
    print("FP64 shift: max absolute error", err)
    assert err <= 4 * 2.0 ** -52
    s_out, _ = K.trig_eval(2, _on_device(np.array([1.0])), _on_device(np.array([0.11])))
    assert np.isnan(s_out.cpu().numpy()[0])


def test_trig_eval_validates() -> None:
    with pytest.raises(ValueError):
        K.trig_eval(0, torch.zeros(4, dtype=torch.float32, device="cuda"))
    with pytest.raises(Exception):
        K.trig_eval(3, _on_device(np.zeros(4)))
    with pytest.raises(Exception):
        K.trig_eval(1, _on_device(np.zeros(4)))  # the shifts need delta
