"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host
side only.  Pixels, samples and frames are independent (the RNG depends on
pixel, sample and seed alone), so work shards without any data-path
collective:

  * weak scaling -- each rank renders its own frame (seed = rank);
  * strong scaling -- ranks render disjoint row bands of one frame and the
    bands are gathered to rank 0 afterwards (host memory, outside the timed
    region).

Timing is the maximum over ranks of each rank's device time."""

from __future__ import annotations

import os


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def frame_seed(rank: int) -> int:
    """Seed of the frame a rank renders under weak scaling."""
    return rank


def row_band(rank: int, world: int, height: int) -> tuple[int, int]:
    """(first row, row count) of a rank's band of a `height`-row frame:
    contiguous, disjoint, covering every row, sizes differing by at most one."""
    base, extra = divmod(height, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device: str | None = None) -> float:
    """Maximum of `value` over the process group (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_bands(band, height: int, device: str | None = None):
    """Rank 0 receives the full frame assembled from every rank's row band
    (a float32 array of shape [rows, width, channels]); other ranks get None."""
    import numpy as np
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return band
    world = dist.get_world_size()
    rank = dist.get_rank()
    width, channels = band.shape[1], band.shape[2]
    rows = [row_band(r, world, height)[1] for r in range(world)]
    t = torch.from_numpy(np.ascontiguousarray(band, np.float32)).to(device or "cpu")
    # equal-size buffers for all_gather: pad every band to the largest
    pad = max(rows)
    buf = torch.zeros((pad, width, channels), dtype=torch.float32, device=t.device)
    buf[: t.shape[0]] = t
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf)
    if rank != 0:
        return None
    return np.concatenate([o[: rows[r]].cpu().numpy() for r, o in enumerate(out)], axis=0)
