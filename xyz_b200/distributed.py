"""Sample-parallel rendering over several GPUs (one process per GPU).

Pixel samples are independent, so N ranks render disjoint sample ranges of
the same image with the scene replicated on each GPU, and the films are
summed once at the end with one reduce (NCCL over NVLink on GPUs).  There is
no other exchange: the reference has no distributed code, and its integrator
only adds samples into one film (xyz/integrator/integrator.cpp:119-128).

Batches of scenes are split by job instead (assign_by_cost: each rank renders
whole jobs, no collective), and a learned guide is trained on one rank and its
weights broadcast to the others (broadcast_guide: one broadcast of the
parameter vector after a training pass).
"""

from __future__ import annotations

import math
from typing import Callable, List, Sequence, Tuple


def sample_range(spp_total: int, rank: int, world: int) -> Tuple[int, int]:
    """(first sample, count) of `rank` when `spp_total` samples per pixel are
    split into contiguous blocks over `world` ranks (strong scaling)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(spp_total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def weak_range(spp_per_rank: int, rank: int) -> Tuple[int, int]:
    """(first sample, count) when every rank renders its own `spp_per_rank`
    samples per pixel (weak scaling, as the benchmark runs)."""
    return rank * spp_per_rank, spp_per_rank


def render_and_reduce(render: Callable[[int, int], "object"], first: int, count: int,
                      dst: int = 0, group=None):
    """Renders samples [first, first + count) with render(first, count) -> film
    (a torch tensor of per-pixel sums) and sums the films of all ranks into
    rank `dst` with one reduce.  Returns the film (complete on `dst`)."""
    import torch.distributed as dist
    film = render(first, count)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return film


def job_cost(n_tris: int, width: int, height: int, spp: int) -> float:
    """Estimated cost of rendering one job: its paths times the depth of a
    kd-tree over its triangles (traversal work per ray grows with log n)."""
    return float(width) * height * spp * math.log2(2.0 + max(0, n_tris))


def assign_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
    """Jobs to ranks by estimated cost: longest job first onto the least
    loaded rank (ties to the lower rank), so every rank computes the same
    assignment without an exchange.  Returns each rank's job indices in
    ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for j in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += float(costs[j])
        out[r].append(j)
    return [sorted(x) for x in out]


def broadcast_guide(guide, src: int = 0, group=None) -> None:
    """Copies rank `src`'s guide parameters (Guide.params, xyzgpu_guide_get_params) to the
    guides of all ranks with one broadcast: the guide is trained on one GPU and
    every rank renders with the same network.  On NCCL the vector travels as a
    CUDA tensor, on gloo as a CPU tensor."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return
    p = torch.from_numpy(guide.params().astype("float32", copy=True))
    if dist.get_backend(group) == "nccl":
        p = p.cuda()
    dist.broadcast(p, src=src, group=group)
    if dist.get_rank(group) != src:
        guide.set_params(p.cpu().numpy())
