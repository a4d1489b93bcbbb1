"""The allocation-free entry point ``krr_trace_images_noalloc``.

It serves callers that cannot allocate device memory on the trace path (an application with a
fixed device-memory budget that forbids allocations after start-up, a plug-in whose host owns
all device memory): the launch scratch lives in a static array in the library's device image.
The results must equal those of ``krr_trace_images_device`` (the entry point with
caller-provided workspace) on the same inputs, on two calls in a row (the shared array keeps
the previous call's counters, which each call clears), with and without the disk-plane event
(whose outputs the kernel writes only on a hit, so each call clears them). This file is
collected last so that a run stopping at the first failure has run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("Y", "state", "n_steps", "n_rejected", "lam", "max_null_error", "max_energy_drift", "max_lz_drift",
          "max_carter_drift")


def _specs(K, disk: bool = False):
    cams = [(0.9, 60.0, 64, 1e-6), (0.5, 17.0, 48, 1e-8), (0.99, 85.0, 32, 1e-6)]
    events = K.EventOptions(disk_plane=True, r_in=6.0, r_out=20.0) if disk else None
    return [K.ImageSpec(K.Spacetime(1.0, a), K.Camera(radius=1000.0, inclination_deg=i, fov=8.0 if not disk else 24.0,
                                                      resolution=n),
                        K.IntegratorOptions(rtol=rt, atol=1e-2 * rt), K.TerminationOptions(), events)
            for a, i, n, rt in cams]


def _outputs(torch, total: int, disk: bool = False, fill: int = -7):
    out = {"Y": torch.full((total, 8), np.nan, dtype=torch.float64, device="cuda")}
    for name in ("state", "n_steps", "n_rejected"):
        out[name] = torch.full((total,), fill, dtype=torch.int64, device="cuda")
    for name in ("lam", "max_null_error", "max_energy_drift", "max_lz_drift", "max_carter_drift"):
        out[name] = torch.full((total,), np.nan, dtype=torch.float64, device="cuda")
    if disk:
        # Garbage in the event outputs: the entry points must clear what a miss leaves unwritten.
        out["event_Y"] = torch.full((total, 8), 3.25, dtype=torch.float64, device="cuda")
        out["event_hit"] = torch.full((total,), 0xA5, dtype=torch.uint8, device="cuda")
    return out


@pytest.mark.parametrize("disk", [False, True], ids=["shadow", "disk_plane"])
def test_noalloc_entry_point_matches_the_workspace_entry_point_twice(disk: bool) -> None:
    torch = pytest.importorskip("torch")
    from kerrray_b200.build import build

    build()
    import kerrray_b200 as K
    from kerrray_b200 import _lib

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device")
    specs = _specs(K, disk)
    images = (_lib.KrrImage * len(specs))(*[s.as_struct() for s in specs])
    total = sum(s.n_rays for s in specs)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for precision in ("fast64", "mixed"):
        launch = _lib.KrrLaunch(precision=_lib.PRECISIONS[precision], block=0, blocks_per_sm=0, refill_threshold=0,
                                plain=0, variant=0, retrace=0, critical_sms=0)
        ref = _outputs(torch, total, disk)
        ws = torch.zeros(int(L.krr_workspace_size(len(specs), 0)), dtype=torch.uint8, device="cuda")
        st = _lib.KrrStats()
        _lib.check(L.krr_trace_images_device(0, images, len(specs), None, ctypes.byref(launch),
                                             ctypes.byref(_lib.result_struct(ref, device=True)), ws.data_ptr(),
                                             ws.numel(), stream, ctypes.byref(st)))
        assert st.retired == total
        for call in range(2):
            got = _outputs(torch, total, disk, fill=-9 - call)
            st2 = _lib.KrrStats(critical=77, rechecked=77, speculative=77, discarded_attempts=77, kernel_ms=5.0)
            _lib.check(L.krr_trace_images_noalloc(0, images, len(specs), None, ctypes.byref(launch),
                                                  ctypes.byref(_lib.result_struct(got, device=True)), stream,
                                                  ctypes.byref(st2)))
            assert st2.retired == total and st2.attempts == st.attempts and st2.accepted == st.accepted, call
            # Every counter the call does not report is written as zero, not left as the caller's.
            assert (st2.critical, st2.rechecked, st2.speculative, st2.discarded_attempts, st2.kernel_ms) == (0, 0, 0, 0, 0.0)
            for name in FIELDS + (("event_Y", "event_hit") if disk else ()):
                assert torch.equal(got[name], ref[name]), (precision, call, name)
        if disk:
            hits = int(ref["event_hit"].sum())
            assert 0 < hits < total and set(ref["event_hit"].unique().tolist()) == {0, 1}


def test_noalloc_entry_point_rejects_batches_beyond_its_scratch() -> None:
    from kerrray_b200.build import build

    build()
    import kerrray_b200 as K
    from kerrray_b200 import _lib

    spec = _specs(K)[2]
    n = 129  # KRR_NOALLOC_MAX_IMAGES + 1
    images = (_lib.KrrImage * n)(*[spec.as_struct()] * n)
    launch = _lib.KrrLaunch(precision=1)
    res = _lib.KrrResult()  # the size check comes before any output is looked at
    rc = _lib.lib().krr_trace_images_noalloc(0, images, n, None, ctypes.byref(launch), ctypes.byref(res), None, None)
    assert rc == _lib.KRR_ERR_INVALID and "at most 128 images" in _lib.last_error()
