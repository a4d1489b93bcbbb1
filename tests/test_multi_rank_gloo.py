"""The multi-GPU path's host logic on two CPU ranks (gloo): each rank takes its share of the
work (kerrray_b200.shard) -- whole images, pixel ranges of one image, or the directions of an
edge study -- traces it -- here with the oracle, the CPU restatement of the reference's
kernel, as the GPU kernel is not available on CPU ranks -- and the results gathered to every
rank equal a single-process run of the whole job; the maximum over ranks of a timing is every
rank's maximum."""
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



def _oracle_pixels(spec, first: int, count: int):
    """The oracle's trace of pixels first .. first + count - 1 of an image (row-major)."""
    from oracle import oracle as O

    cam = spec.camera
    alpha, beta = O.pixel_coordinates(cam.fov, cam.resolution)
    sl = slice(first, first + count)
    y0 = O.initial_states(spec.spacetime.mass, spec.spacetime.spin, cam.radius, cam.inclination_deg, cam.phi_deg,
                          alpha.ravel()[sl], beta.ravel()[sl])
    res = O.integrate(spec.spacetime.mass, spec.spacetime.spin, y0,
                      O.Options(rtol=spec.integ.rtol, atol=spec.integ.atol), threads=1)
    return {"state": np.asarray(res["state"]), "Y": np.asarray(res["Y"]), "n_steps": np.asarray(res["n_steps"])}


def _one_image():
    import kerrray_b200 as K

    return [K.ImageSpec(K.Spacetime(1.0, 0.9), K.Camera(radius=1000.0, inclination_deg=60.0, fov=8.0, resolution=12),
                        K.IntegratorOptions(rtol=1e-6, atol=1e-8), K.TerminationOptions())]


def _edge_cases():
    import kerrray_b200 as K

    angles = 2.0 * np.pi * np.arange(5) / 5 + 0.1
    return [K.edge_study(K.Spacetime(1.0, 0.9), 60.0, 1.0e5, 1e-6, angles),
            K.edge_study(K.Spacetime(1.0, 0.5), 17.0, 1.0e5, 1e-8, angles[:3])]


def _oracle_bisect(case, first: int, count: int, iterations: int = 6) -> np.ndarray:
    """The reference's bisection loop (study_edge_bisection.py:53-68) on directions
    first .. first + count - 1 of a case, with the oracle as the integrator."""
    from oracle import oracle as O

    sl = slice(first, first + count)
    ang, lo, hi = case.angles[sl], case.r_lo[sl].copy(), case.r_hi[sl].copy()
    spin, r_o = case.spacetime.spin, case.r_o
    opts = O.Options(rtol=case.rtol, atol=1e-2 * case.rtol, max_steps=2_000_000, lambda_max=4.0 * r_o,
                     horizon_epsilon=1e-6, escape_radius=r_o)
    for _ in range(iterations):
        mid = 0.5 * (lo + hi)
        y0 = O.initial_states(1.0, spin, r_o, case.inclination_deg, 0.0, case.centre[0] + mid * np.cos(ang),
                              case.centre[1] + mid * np.sin(ang))
        escaped = O.integrate(1.0, spin, y0, opts, threads=1)["state"] == 1
        hi = np.where(escaped, mid, hi)
        lo = np.where(escaped, lo, mid)
    return 0.5 * (lo + hi)


def _split_main(rank: int, port: int, out_dir: str) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        # one image over both ranks, by pixel ranges
        specs = _one_image()
        mine = shard.shard_pieces(specs, rank, WORLD)
        entries = shard.piece_specs(specs, mine)
        assert all(e.n_rays == p.count for e, p in zip(entries, mine))
        image = shard.gather_pieces(mine, [_oracle_pixels(specs[p.image], p.first, p.count) for p in mine], specs)[0]
        # the directions of an edge study over both ranks
        cases = _edge_cases()
        runs = shard.shard_items([c.rtol ** -0.2 for c in cases], [c.angles.size for c in cases], rank, WORLD)
        parts = [None] * WORLD
        dist.all_gather_object(parts, [(k, f, n, _oracle_bisect(cases[k], f, n)) for k, f, n in runs])
        edges = [np.full(c.angles.size, np.nan) for c in cases]
        for part in parts:
            for k, f, n, r in part:
                assert np.all(np.isnan(edges[k][f:f + n]))
                edges[k][f:f + n] = r
        np.savez(os.path.join(out_dir, f"split{rank}.npz"), pixels=sum(p.count for p in mine), runs=len(runs),
                 **{f"img_{k}": v for k, v in image.items()}, **{f"edge{k}": e for k, e in enumerate(edges)})
    finally:
        dist.destroy_process_group()


def test_one_image_and_an_edge_study_split_over_two_ranks(tmp_path) -> None:
    mp.start_processes(_split_main, args=(_free_port(), str(tmp_path)), nprocs=WORLD, start_method="spawn")
    spec = _one_image()[0]
    whole = _oracle_pixels(spec, 0, spec.camera.n_rays)
    cases = _edge_cases()
    edges = [_oracle_bisect(c, 0, c.angles.size) for c in cases]
    shares = []
    for rank in range(WORLD):
        d = np.load(tmp_path / f"split{rank}.npz")
        shares.append(int(d["pixels"]))
        assert int(d["runs"]) >= 1  # every rank bisects some directions
        for name, v in whole.items():
            assert np.array_equal(d[f"img_{name}"], v), name
        for k, e in enumerate(edges):
            assert np.array_equal(d[f"edge{k}"], e)
    assert sum(shares) == spec.camera.n_rays and min(shares) > 0  # both ranks trace part of the image


def test_pixel_pieces_cover_every_pixel_once_and_balance() -> None:
    import kerrray_b200 as K

    specs = shard.replicate_specs(_specs(), 1) + [
        K.ImageSpec(K.Spacetime(1.0, 0.99), K.Camera(radius=1000.0, inclination_deg=85.0, fov=8.0, resolution=64),
                    K.IntegratorOptions(rtol=1e-10, atol=1e-12), K.TerminationOptions())]
    for world in (1, 2, 3, 8):
        pieces = [shard.shard_pieces(specs, r, world) for r in range(world)]
        count = [np.zeros(s.camera.n_rays, int) for s in specs]
        for rank_pieces in pieces:
            for p in rank_pieces:
                count[p.image][p.first:p.first + p.count] += 1
        assert all(np.all(c == 1) for c in count)
        density = [shard.image_cost(s) / s.camera.n_rays for s in specs]
        loads = [sum(p.count * density[p.image] for p in rp) for rp in pieces]
        assert max(loads) <= 1.3 * sum(loads) / world, (world, loads)
    # one image alone still spreads over every rank
    one = specs[-1:]
    assert all(shard.shard_pieces(one, r, 4) for r in range(4))
    entry = shard.piece_specs(one, shard.shard_pieces(one, 1, 4))[0]
    assert entry.pixels is not None and entry.n_rays == entry.pixels[1] and not entry.whole
    with pytest.raises(ValueError):
        K.ImageSpec(one[0].spacetime, one[0].camera, one[0].integ, one[0].term, pixels=(4090, 10))


def test_items_split_in_equal_cost_runs() -> None:
    costs, counts = [1.0, 2.0, 1.0], [30, 20, 40]
    for world in (1, 2, 3, 5):
        runs = [shard.shard_items(costs, counts, r, world) for r in range(world)]
        seen = [np.zeros(n, int) for n in counts]
        loads = []
        for rr in runs:
            loads.append(sum(costs[k] * n for k, _, n in rr))
            for k, f, n in rr:
                seen[k][f:f + n] += 1
        assert all(np.all(x == 1) for x in seen)
        assert max(loads) - min(loads) <= 2 * max(costs)
    assert shard.split_range(10, 0, 3) == slice(0, 3) and shard.split_range(10, 2, 3) == slice(6, 10)
