"""Work split over several GPUs: one process per GPU, no collective on the data path.

Photons never interact, and a bisection direction depends only on its own history, so every
workload here splits into independent units:

* images, or ranges of an image's pixels (:func:`split_pixels`, :func:`shard_pieces`): each
  image is cut into contiguous pixel ranges of at most ``1 / (world * pieces_per_rank)`` of the
  job's predicted cost (whole images when they fit), and the pieces are dealt to ranks
  longest-first to the least-loaded rank. A single image (a 2048^2 shadow, the lensing map)
  therefore spreads over every rank, and a many-image sweep splits its large images only;
* whole images (:func:`shard_specs`);
* bisection items, the (case, direction) pairs of an edge study (:func:`shard_items`):
  contiguous runs of the item list with equal predicted cost per rank;
* plain index ranges (:func:`split_range`), for rays of equal expected cost.

Each rank traces its share with its own persistent work queue. The only collectives are
outside the traced region: the maximum over ranks of a timing, and an optional gather of the
results to every rank (``torch.distributed`` over NCCL on GPUs, gloo on CPUs). Every partition
is a pure function of the job, so every rank computes the same one without communicating.
"""
from __future__ import annotations

import dataclasses
from typing import Any, Sequence

import numpy as np

__all__ = ["Piece", "image_cost", "shard_specs", "split_pixels", "shard_pieces", "piece_specs", "gather_pieces",
           "shard_items", "split_range", "replicate_specs", "max_over_ranks", "gather_results"]


def image_cost(spec) -> float:
    """Predicted cost of an image: its photons times rtol^(-1/5) (a DP5 step count's growth)."""
    return float(spec.n_rays) * (1.0 / float(spec.integ.rtol)) ** 0.2


def shard_specs(specs: Sequence[Any], rank: int, world: int) -> list[int]:
    """Indices (ascending) of the images rank ``rank`` of ``world`` traces.

    Longest-processing-time assignment: images in decreasing predicted cost, each to the rank
    with the least load so far (the lowest rank on ties). Every image goes to exactly one rank.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"need 0 <= rank < world, got rank {rank} of {world}")
    cost = [image_cost(s) for s in specs]
    load = [0.0] * world
    owner = [0] * len(specs)
    for k in sorted(range(len(specs)), key=lambda i: (-cost[i], i)):
        r = min(range(world), key=lambda j: (load[j], j))
        owner[k] = r
        load[r] += cost[k]
    return [k for k in range(len(specs)) if owner[k] == rank]


def replicate_specs(specs: Sequence[Any], copies: int) -> list[Any]:
    """``copies`` copies of ``specs`` with the observer turned in azimuth by 360/copies degrees
    per copy: distinct images of the same cost (the spacetime is axisymmetric), for a workload
    that grows with the number of GPUs (weak scaling). One copy returns the images unchanged."""
    if copies < 1:
        raise ValueError(f"copies must be >= 1, got {copies}")
    out = []
    for c in range(copies):
        for s in specs:
            if c == 0:
                out.append(s)
            else:
                cam = dataclasses.replace(s.camera, phi_deg=float(s.camera.phi_deg) + 360.0 * c / copies)
                out.append(dataclasses.replace(s, camera=cam))
    return out


def max_over_ranks(value: float, group=None) -> float:
    """The maximum of ``value`` over the ranks of ``group`` (``value`` itself without a group)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(indices: Sequence[int], results: Sequence[Any], n_images: int, group=None) -> list[Any]:
    """Every rank's ``results`` (one per image of ``indices``), gathered to every rank and
    returned in image order: a list of ``n_images`` entries."""
    import torch.distributed as dist

    if len(indices) != len(results):
        raise ValueError("one result per image index")
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        parts = [(list(indices), list(results))]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, (list(indices), list(results)), group=group)
    out: list[Any] = [None] * n_images
    seen = 0
    for idx, res in parts:
        for k, r in zip(idx, res):
            if out[k] is not None:
                raise RuntimeError(f"image {k} traced by two ranks")
            out[k] = r
            seen += 1
    if seen != n_images:
        raise RuntimeError(f"{n_images - seen} images traced by no rank")
    return out


@dataclasses.dataclass(frozen=True)
class Piece:
    """Pixels ``first .. first + count - 1`` (row-major) of image ``image`` of a job."""

    image: int
    first: int
    count: int


def split_pixels(specs: Sequence[Any], world: int, pieces_per_rank: int = 4) -> list[Piece]:
    """Every image of ``specs`` cut into contiguous pixel ranges of at most
    ``total cost / (world * pieces_per_rank)`` predicted cost each (equal sizes within an image;
    an image that fits stays whole). Pieces in image order, each image's in pixel order."""
    if world < 1 or pieces_per_rank < 1:
        raise ValueError(f"need world >= 1 and pieces_per_rank >= 1, got {world}, {pieces_per_rank}")
    cost = [image_cost(s) for s in specs]
    quantum = sum(cost) / (world * pieces_per_rank)
    out = []
    for k, s in enumerate(specs):
        n = int(s.camera.n_rays)
        cuts = max(1, min(n, int(np.ceil(cost[k] / quantum - 1e-9)))) if world > 1 else 1
        bounds = [n * j // cuts for j in range(cuts + 1)]
        out += [Piece(k, bounds[j], bounds[j + 1] - bounds[j]) for j in range(cuts)]
    return out


def shard_pieces(specs: Sequence[Any], rank: int, world: int, pieces_per_rank: int = 4) -> list[Piece]:
    """The pieces (:func:`split_pixels`) that rank ``rank`` of ``world`` traces, in job order.

    Longest-processing-time assignment: pieces in decreasing predicted cost, each to the rank
    with the least load so far (the lowest rank on ties). Every pixel goes to exactly one rank.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"need 0 <= rank < world, got rank {rank} of {world}")
    pieces = split_pixels(specs, world, pieces_per_rank)
    density = [image_cost(s) / s.camera.n_rays for s in specs]
    cost = [p.count * density[p.image] for p in pieces]
    load = [0.0] * world
    owner = [0] * len(pieces)
    for j in sorted(range(len(pieces)), key=lambda i: (-cost[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[j] = r
        load[r] += cost[j]
    return [p for p, o in zip(pieces, owner) if o == rank]


def piece_specs(specs: Sequence[Any], pieces: Sequence[Piece]) -> list[Any]:
    """The batched-launch entries of ``pieces``: each image's spec with its pixel range."""
    out = []
    for p in pieces:
        s = specs[p.image]
        whole = p.first == 0 and p.count == s.camera.n_rays
        out.append(s if whole else dataclasses.replace(s, pixels=(p.first, p.count)))
    return out


def gather_pieces(pieces: Sequence[Piece], arrays: Sequence[dict], specs: Sequence[Any], group=None) -> list[dict]:
    """Every rank's per-piece result arrays (dicts of equal keys, ``count`` rows each), gathered
    to every rank and assembled per image: a list with one dict of full-image arrays per spec."""
    import torch.distributed as dist

    if len(pieces) != len(arrays):
        raise ValueError("one array dict per piece")
    mine = [(dataclasses.astuple(p), a) for p, a in zip(pieces, arrays)]
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        parts = [mine]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, mine, group=group)
    out: list[dict] = [{} for _ in specs]
    covered = [np.zeros(int(s.camera.n_rays), dtype=np.int32) for s in specs]
    for part in parts:
        for (k, first, count), a in part:
            for name, value in a.items():
                if name not in out[k]:
                    value = np.asarray(value)
                    out[k][name] = np.zeros((int(specs[k].camera.n_rays),) + value.shape[1:], value.dtype)
                out[k][name][first:first + count] = value
            covered[k][first:first + count] += 1
    for k, c in enumerate(covered):
        if np.any(c != 1):
            raise RuntimeError(f"image {k}: {int((c == 0).sum())} pixels traced by no rank, "
                               f"{int((c > 1).sum())} by more than one")
    return out


def shard_items(costs: Sequence[float], counts: Sequence[int], rank: int, world: int) -> list[tuple[int, int, int]]:
    """Rank ``rank``'s share of a list of work items grouped in cases: case ``k`` holds
    ``counts[k]`` items of predicted cost ``costs[k]`` each (an edge study: one item per
    direction). The items, in case order, are cut into ``world`` contiguous runs of equal
    cumulative cost; returns this rank's ``(case, first item, item count)`` runs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"need 0 <= rank < world, got rank {rank} of {world}")
    per_item = np.repeat(np.asarray(costs, dtype=np.float64), np.asarray(counts, dtype=np.int64))
    edges = np.concatenate([[0.0], np.cumsum(per_item)])
    total = edges[-1]
    # item i goes to the rank whose cost interval holds the item's cost midpoint
    owner = np.minimum((0.5 * (edges[:-1] + edges[1:]) / total * world).astype(np.int64), world - 1)
    case_of = np.repeat(np.arange(len(counts)), np.asarray(counts, dtype=np.int64))
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    runs = []
    for k in range(len(counts)):
        sel = np.flatnonzero((case_of == k) & (owner == rank))
        if sel.size:
            runs.append((k, int(sel[0] - start[k]), int(sel.size)))
    return runs


def split_range(n: int, rank: int, world: int) -> slice:
    """Rank ``rank``'s contiguous share of ``n`` equal-cost units."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"need 0 <= rank < world, got rank {rank} of {world}")
    return slice(n * rank // world, n * (rank + 1) // world)
