"""Pixel slabs across processes: one process per GPU, replicas of the inversion.

Pixels are independent, so a cube shards into contiguous slabs with no exchange
on the data path -- the partition of pmilos' MPI driver (pmilos.c:1181-1205:
npix // world pixels per rank, the first npix % world ranks one more) -- and the
only collective is the results-only gather of models, chi^2 and iterations
(pmilos.c's Gatherv of the same planes).  ``torch.distributed`` carries the
gather (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def slab(npix: int, rank: int, world: int) -> tuple[int, int]:
    """(first pixel, pixel count) of ``rank``'s slab."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, rest = divmod(int(npix), int(world))
    count = base + (1 if rank < rest else 0)
    start = rank * base + min(rank, rest)
    return start, count


def invert_slab(inv, cube: np.ndarray, guess, rank: int, world: int, **kw) -> dict:
    """Invert this rank's slab of a host cube [npix][4][nl] with an Inverter."""
    s, n = slab(cube.shape[0], rank, world)
    return inv.invert(cube[s:s + n], guess, **kw)


def gather(local: dict, npix: int, group=None, dst: int = 0) -> dict | None:
    """Gather every rank's slab results into full-cube arrays on ``dst``
    (None elsewhere).  Every rank calls it, in the same order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = [slab(npix, r, world)[1] for r in range(world)]
    width = max(counts)
    out = {} if rank == dst else None
    for key, cols, dtype in (("models", 11, torch.float64), ("chisq", 1, torch.float32), ("iters", 1, torch.int32)):
        mine = torch.zeros((width, cols), dtype=dtype)
        mine[: counts[rank]] = torch.as_tensor(np.asarray(local[key]).reshape(counts[rank], cols))
        bufs = [torch.zeros_like(mine) for _ in range(world)] if rank == dst else None
        dist.gather(mine, bufs, dst=dst, group=group)
        if rank == dst:
            full = torch.cat([b[:c] for b, c in zip(bufs, counts)]).numpy()
            out[key] = full if cols > 1 else full.reshape(-1)
    return out
