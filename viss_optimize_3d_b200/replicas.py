"""Observation days over several GPUs: independent replicas, one summed image.

The reference spreads its 450 days over the GPUs round-robin, one OpenMP
thread per device, with no communication (vissgen3d_blockage.cu:271-279), and
its notebooks then add the 450 per-day images on the host, replacing NaN by 0
(healpix3d_blockage.ipynb:103-116).  Here each rank of a torch.distributed
process group (one process per GPU, NCCL; or gloo on CPU) takes the same
round-robin days, accumulates its images on its own device, and one
all-reduce (SUM) produces the summed image on every rank -- the only
collective on this path, one npix-sized vector per run.  Timing helpers take
the max over ranks.
"""
from __future__ import annotations

from typing import Callable, Iterable

import torch
import torch.distributed as dist


def days_for_rank(n_days: int, rank: int, world: int, first_day: int = 1) -> list[int]:
    """Days (1-based) handled by `rank`: first_day + rank, + world, ...
    (vissgen3d_blockage.cu:279: p = tid; p < days; p += nDevices)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return [first_day + p for p in range(rank, n_days, world)]


def _group_ready() -> bool:
    return dist.is_available() and dist.is_initialized()


def max_over_ranks(values: Iterable[float], device=None) -> list[float]:
    """Element-wise max of per-rank values (device-timed seconds and the like)."""
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if _group_ready() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def sum_images(image: torch.Tensor) -> torch.Tensor:
    """In-place SUM of a per-rank image over the process group."""
    if _group_ready() and dist.get_world_size() > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM)
    return image


def add_day_image(total: torch.Tensor, img: torch.Tensor) -> torch.Tensor:
    """total += img (FP64), non-finite pixels counted as 0.  On a CUDA device
    this is one viss_accumulate_image launch; CPU tensors (the gloo tests'
    stand-ins for a rank's images) take the same arithmetic in torch."""
    if total.is_cuda:
        from . import api
        return api.accumulate_image(total, img)
    img = torch.nan_to_num(img.to(torch.float64), nan=0.0, posinf=0.0, neginf=0.0)
    total += img
    return total


def accumulate_days(n_days: int, npix: int, image_of_day: Callable[[int], torch.Tensor],
                    device=None, first_day: int = 1, nan_to_zero: bool = True) -> torch.Tensor:
    """Sum of image_of_day(d) over all days d, each rank computing its own
    round-robin share; NaN entries count as 0 as in the notebooks."""
    rank = dist.get_rank() if _group_ready() else 0
    world = dist.get_world_size() if _group_ready() else 1
    total = torch.zeros(npix, dtype=torch.float64, device=device)
    for d in days_for_rank(n_days, rank, world, first_day):
        img = image_of_day(d).to(device=total.device)
        if nan_to_zero:
            add_day_image(total, img)
        else:
            total += img.to(torch.float64)
    return sum_images(total)
