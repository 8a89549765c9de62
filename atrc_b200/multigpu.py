"""Sample-split rendering over several GPUs (one process per GPU).

The `pt` path has no cross-pixel dependency (perpixel_renderer.cpp:21-53) and
pt_cuda seeds every sample's random stream from (pixel, sample index) alone, so
a frame's samples shard exactly: rank r of world w renders the sample indices
`first_spp(step, r, w, spp)` .. + spp of every pixel, and summing the FP64
films gives the same film as rendering all indices on one GPU (up to the order
of floating-point additions).  The only exchange is one reduce of the film.
"""
from __future__ import annotations

FILM_FIELDS = ("value", "weight", "value_sq", "albedo", "normal", "denoise")


def first_spp(step: int, rank: int, world: int, spp_per_rank: int) -> int:
    """First sample index rendered by `rank` in `step` (disjoint over ranks and steps)."""
    if not (0 <= rank < world) or spp_per_rank <= 0 or step < 0:
        raise ValueError("invalid sample-range request")
    return (step * world + rank) * spp_per_rank


def reduce_film(film, dist, dst: int = 0) -> None:
    """Sum every accumulator of `film` (torch tensors) onto rank `dst`.

    The other ranks' accumulators restart from zero afterwards (a reduce
    leaves a non-root buffer unspecified), so a reduce after every step adds
    each rank's new samples to `dst` once: `dst` then holds every sample
    rendered so far and the others only what they rendered since."""
    rank = dist.get_rank()
    on_device = False
    for name in FILM_FIELDS:
        t = getattr(film, name, None)
        if t is not None:
            dist.reduce(t, dst)
            if rank != dst:
                t.zero_()
            on_device = on_device or t.is_cuda
    if on_device:
        # the library renders on its own stream, which does not wait for
        # torch's: the reduce and the zero fill end before the next render
        import torch
        torch.cuda.current_stream().synchronize()
