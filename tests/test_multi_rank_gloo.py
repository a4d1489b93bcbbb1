"""The multi-GPU path's host logic on two CPU ranks (gloo): each rank takes its share of the
images (kerrray_b200.shard), traces it -- here with the oracle, the CPU restatement of the
reference's kernel, as the GPU kernel is not available on CPU ranks -- and the results gathered
to every rank equal a single-process trace of all images; the maximum over ranks of a timing
is every rank's maximum."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from kerrray_b200 import shard  # noqa: E402

WORLD = 2


def _specs():
    import kerrray_b200 as K

    out = []
    for spin, incl, rtol in ((0.0, 60.0, 1e-6), (0.9, 17.0, 1e-6), (0.99, 85.0, 1e-8), (0.5, 60.0, 1e-6),
                             (0.9, 60.0, 1e-8)):
        out.append(K.ImageSpec(K.Spacetime(1.0, spin), K.Camera(radius=1000.0, inclination_deg=incl, fov=8.0,
                                                                   resolution=8),
                               K.IntegratorOptions(rtol=rtol, atol=1e-2 * rtol), K.TerminationOptions()))
    return out


def _trace_with_oracle(spec):
    from oracle import oracle as O

    cam = spec.camera
    alpha, beta = O.pixel_coordinates(cam.fov, cam.resolution)
    y0 = O.initial_states(spec.spacetime.mass, spec.spacetime.spin, cam.radius, cam.inclination_deg, cam.phi_deg,
                          alpha.ravel(), beta.ravel())
    opts = O.Options(rtol=spec.integ.rtol, atol=spec.integ.atol)
    res = O.integrate(spec.spacetime.mass, spec.spacetime.spin, y0, opts, threads=1)
    return np.asarray(res["state"]), np.asarray(res["Y"])


def _rank_main(rank: int, port: int, out_dir: str) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        specs = shard.replicate_specs(_specs(), WORLD)
        mine = shard.shard_specs(specs, rank, WORLD)
        results = [_trace_with_oracle(specs[k]) for k in mine]
        gathered = shard.gather_results(mine, results, len(specs))
        t_max = shard.max_over_ranks(float(rank + 1))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), mine=np.array(mine), t_max=t_max,
                 **{f"state{k}": g[0] for k, g in enumerate(gathered)}, **{f"Y{k}": g[1] for k, g in enumerate(gathered)})
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_shard_trace_and_gather(tmp_path) -> None:
    mp.start_processes(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=WORLD, start_method="spawn")
    specs = shard.replicate_specs(_specs(), WORLD)
    ref = [_trace_with_oracle(s) for s in specs]
    owned = []
    for rank in range(WORLD):
        d = np.load(tmp_path / f"rank{rank}.npz")
        assert float(d["t_max"]) == WORLD
        owned += list(d["mine"])
        for k, (st, y) in enumerate(ref):
            assert np.array_equal(d[f"state{k}"], st) and np.array_equal(d[f"Y{k}"], y)
    assert sorted(owned) == list(range(len(specs)))


def test_shards_are_disjoint_and_balanced() -> None:
    specs = shard.replicate_specs(_specs(), 4)
    cost = np.array([shard.image_cost(s) for s in specs])
    parts = [shard.shard_specs(specs, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == list(range(len(specs)))
    loads = [cost[p].sum() for p in parts]
    # four copies of each image: each rank takes one copy of every image, equal loads
    assert max(loads) - min(loads) <= 1e-9 * max(loads)
    # the copies are distinct images of the same cost: the observer turned in azimuth
    assert {s.camera.phi_deg for s in specs} == {0.0, 90.0, 180.0, 270.0}
    assert shard.shard_specs(specs[:1], 0, 2) == [0] and shard.shard_specs(specs[:1], 1, 2) == []
    with pytest.raises(ValueError):
        shard.shard_specs(specs, 2, 2)


def test_single_process_gather_and_reduce() -> None:
    """Without a process group the helpers are the identity; a missing image is an error."""
    assert shard.max_over_ranks(3.5) == 3.5
    assert shard.gather_results([1, 0], ["b", "a"], 2) == ["a", "b"]
    with pytest.raises(RuntimeError):
        shard.gather_results([0], ["a"], 2)
    with pytest.raises(ValueError):
        shard.gather_results([0, 1], ["a"], 2)
    with pytest.raises(ValueError):
        shard.replicate_specs(_specs(), 0)

