"""Data-parallel plumbing of the chain: one process per GPU, frames sharded.

Frames are independent through the whole chain (forward and adjoints), so a
rank renders its own frames with all their views; per-frame parameters (node
rotations / translations, joint angles) get their full gradient locally.  The
parameters shared by all frames (vertex colours, texture, SH) are the only
exchange: one all-reduce (sum) per step, the data-parallel SUM of the
reference's MirroredStrategy (Projects/HoloportedCharacters/HPCMeshDL.py:85,
485-492).  Works with the NCCL backend on GPUs and gloo on CPU.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank() -> tuple[int, int, int]:
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0, device: torch.device | None = None) -> tuple[int, int, int]:
    """Join the process group when WORLD_SIZE > 1; returns (world, rank, local_rank)."""
    world, rank, local = env_rank()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None and backend == "nccl":
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return world, rank, local


def shard_frames(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous block of frames of `rank`: (first, count); the first
    total % world ranks get one extra frame."""
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def allreduce_shared(tensors, world: int) -> None:
    """Sum the shared-parameter gradients over the ranks, in place."""
    if world > 1:
        for t in tensors:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)


def shared_gradient(per_frame: torch.Tensor, out: torch.Tensor, world: int) -> torch.Tensor:
    """Gradient of a parameter that every frame shares (the vertex colours
    [N,3] of the character): the chain writes one gradient per frame slot
    [B,...]; the parameter's gradient is their sum over this rank's frames,
    then over the ranks (one all-reduce).  ``out`` [...] receives it."""
    torch.sum(per_frame, dim=0, out=out)
    allreduce_shared([out], world)
    return out


def rank_frames(total_per_rank: int, world: int, rank: int) -> tuple[int, int]:
    """Weak scaling: the job has ``total_per_rank * world`` frames, rank r
    renders the contiguous block ``shard_frames`` gives it."""
    return shard_frames(total_per_rank * world, world, rank)


def max_over_ranks(x: float, world: int, device: torch.device | str = "cpu") -> float:
    """The largest value of x over the ranks (step times are reported this way)."""
    if world == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        dist.barrier()


def finalize(world: int) -> None:
    if world > 1 and dist.is_initialized():
        dist.destroy_process_group()
