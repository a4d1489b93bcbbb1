"""Batched image traces over several GPUs: one process per GPU, no collective on the data path.

Photons never interact, so a sweep's images are split across ranks, balanced by their
predicted cost, and each rank traces its share with its own persistent work queue. The only
collectives are outside the traced region: the maximum over ranks of a timing, and an optional
gather of the results to every rank (``torch.distributed`` over NCCL on GPUs, gloo on CPUs).

The partition is a pure function of the image list, so every rank computes the same one
without communicating.
"""
from __future__ import annotations

import dataclasses
from typing import Any, Sequence

__all__ = ["image_cost", "shard_specs", "replicate_specs", "max_over_ranks", "gather_results"]


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
