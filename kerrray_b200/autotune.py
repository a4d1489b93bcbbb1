"""Autotuner of the persistent kernel's launch shape.

Chooses, for a list of images and a precision, the compiled launch variant (threads per block
and register cap, i.e. how many warps stay resident per SM) and the refill threshold (how many
lanes of a warp may sit idle before the warp pulls new photons from the queue) by timing
each candidate on a reduced copy of the workload: the same images at a half or a quarter of the
resolution per side (same field of view, so the same mix of escaping, captured and
near-critical photons), reduced only while at least half a million photons remain -- fewer
leave the launch's tail in charge and favour other shapes than the full workload would. The
reduced copy ranks the candidates; the fastest few are then timed again on the workload itself
(candidates within a percent or two at a quarter of the resolution need not keep their order
at full size: a refill threshold of 8 won the reduced sweep once and ran 2 % slower than 4 on the
full one). Each
warp handles 32 photons at a time, one per lane; the refill claims as many queue entries as
the warp has idle lanes.

Results are cached per device, precision and workload signature in memory and, when
``KRR_AUTOTUNE_CACHE`` names a file, in that JSON file.
"""

from __future__ import annotations

import ctypes
import json
import os
from dataclasses import replace
from pathlib import Path
from typing import Sequence

from kerrray_b200 import _lib
from kerrray_b200.camera import Camera
from kerrray_b200.sweep import DeviceSweep, ImageSpec, LaunchConfig

__all__ = ["autotune", "list_variants"]

_CACHE: dict[str, dict] = {}


def list_variants(precision: str, integ, term, device: int = 0) -> list[dict]:
    """The compiled launch shapes for this precision and scheme, with registers and occupancy."""
    opts = _lib.options_struct(integ, term)
    count = ctypes.c_int32(0)
    _lib.check(_lib.lib().krr_list_variants(device, _lib.PRECISIONS[precision], ctypes.byref(opts), None, 0,
                                            ctypes.byref(count)))
    arr = (_lib.KrrVariantInfo * max(count.value, 1))()
    _lib.check(_lib.lib().krr_list_variants(device, _lib.PRECISIONS[precision], ctypes.byref(opts), arr, count.value,
                                            ctypes.byref(count)))
    return [{"variant": k, "block": v.block, "min_blocks": v.min_blocks, "registers": v.registers,
             "blocks_per_sm": v.blocks_per_sm} for k, v in enumerate(arr[: count.value])]


def _signature(specs: Sequence[ImageSpec], precision: str, device: int) -> str:
    import torch

    name = torch.cuda.get_device_name(device)
    rows = sorted({(round(float(s.spacetime.spin), 6), round(float(s.camera.inclination_deg), 4),
                    int(s.camera.resolution), float(s.integ.rtol), str(s.integ.method),
                    tuple(s.pixels) if s.pixels is not None else None) for s in specs})
    return json.dumps([name, precision, len(specs), rows])


def _reduced(specs: Sequence[ImageSpec], scale: int) -> list[ImageSpec]:
    """The images at 1/scale of their resolution per side; a pixel range keeps its share of the
    image (the same fraction of rows at the same place)."""
    out = []
    for s in specs:
        res = max(2, (s.camera.resolution // scale) // 2 * 2)
        cam = Camera(radius=s.camera.radius, inclination_deg=s.camera.inclination_deg, phi_deg=s.camera.phi_deg,
                     fov=s.camera.fov, resolution=res)
        pixels = None
        if s.pixels is not None:
            n, m = s.camera.n_rays, res * res
            first = s.pixels[0] * m // n
            pixels = (min(first, m - 1), max(1, min(s.pixels[1] * m // n, m - min(first, m - 1))))
        out.append(replace(s, camera=cam, pixels=pixels))
    return out


def _load_file() -> dict:
    path = os.environ.get("KRR_AUTOTUNE_CACHE")
    if not path or not Path(path).exists():
        return {}
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def _save_file(table: dict) -> None:
    path = os.environ.get("KRR_AUTOTUNE_CACHE")
    if path:
        Path(path).write_text(json.dumps(table, indent=1))


MIN_TUNING_PHOTONS = 500_000


def tuning_scale(specs: Sequence[ImageSpec]) -> int:
    """Largest reduction per side in (4, 2, 1) that keeps MIN_TUNING_PHOTONS photons."""
    total = sum(s.n_rays for s in specs)
    for scale in (4, 2):
        if total // (scale * scale) >= MIN_TUNING_PHOTONS:
            return scale
    return 1


def autotune(specs: Sequence[ImageSpec], *, precision: str = "fast64", device: int = 0, scale: int | None = None,
             thresholds: Sequence[int] = (1, 4, 8, 16), repeats: int = 2, finalists: int = 3,
             use_cache: bool = True) -> tuple[LaunchConfig, dict]:
    """Return the fastest ``LaunchConfig`` for ``specs`` and a report of every candidate's time
    (``scale``: reduction per side of the tuning workload; None chooses ``tuning_scale``;
    ``finalists``: how many of the fastest on the reduced workload are timed on ``specs``
    itself to decide)."""
    specs = list(specs)
    if scale is None:
        scale = tuning_scale(specs)
    key = _signature(specs, precision, device)
    if use_cache:
        if key in _CACHE:
            hit = _CACHE[key]
            return LaunchConfig(**hit["config"]), hit
        table = _load_file()
        if key in table:
            _CACHE[key] = table[key]
            return LaunchConfig(**table[key]["config"]), table[key]
    small = _reduced(specs, scale) if scale > 1 else specs
    variants = list_variants(precision, specs[0].integ, specs[0].term, device)
    def timed(images, cfg) -> float:
        sweep = DeviceSweep(images, precision=precision, launch=cfg, device=device, minimal=True, graph=False)
        sweep.run()
        ms = min(sweep.run()["kernel_ms"] for _ in range(repeats))
        sweep.close()
        return ms

    trials = []
    for v in variants:
        if v["blocks_per_sm"] < 1:
            continue
        for t in thresholds:
            ms = timed(small, LaunchConfig(variant=v["variant"], refill_threshold=t))
            trials.append({**v, "refill_threshold": t, "ms": ms})
    ranked = sorted(trials, key=lambda tr: tr["ms"])
    final = []
    if scale > 1 and finalists > 1:
        for tr in ranked[:finalists]:
            ms = timed(specs, LaunchConfig(variant=tr["variant"], refill_threshold=tr["refill_threshold"]))
            final.append({"variant": tr["variant"], "refill_threshold": tr["refill_threshold"], "ms": ms})
        win = min(final, key=lambda tr: tr["ms"])
    else:
        win = ranked[0]
    best = (LaunchConfig(variant=win["variant"], refill_threshold=win["refill_threshold"]), win["ms"])
    report = {"config": {"variant": best[0].variant, "refill_threshold": best[0].refill_threshold},
              "ms": best[1], "photons": sum(s.n_rays for s in small), "scale": scale, "trials": trials,
              "final": final, "final_photons": sum(s.n_rays for s in specs) if final else None}
    _CACHE[key] = report
    if use_cache and os.environ.get("KRR_AUTOTUNE_CACHE"):
        table = _load_file()
        table[key] = report
        _save_file(table)
    return best[0], report
