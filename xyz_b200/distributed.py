"""Sample-parallel rendering over several GPUs (one process per GPU).

Pixel samples are independent, so N ranks render disjoint sample ranges of
the same image with the scene replicated on each GPU, and the films are
summed once at the end with one reduce (NCCL over NVLink on GPUs).  There is
no other exchange: the reference has no distributed code, and its integrator
only adds samples into one film (xyz/integrator/integrator.cpp:119-128).
"""

from __future__ import annotations

from typing import Callable, Tuple


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
