"""Fly sharding across GPUs: one process per GPU, flies split into contiguous shards.

Flies are independent, so stepping needs no exchange: each rank owns flies
[fly0, fly0 + count) of the job, holds a read-only replica of the graph, and keys its Poisson
streams by the global fly index (flyb_lif_args.fly0), which makes an N-rank run draw exactly what
one rank running every fly would. The only collectives are the ones a caller asks for:
`allreduce_gradients` sums adjoint gradients over ranks (NCCL over NVLink on GPUs, gloo on CPU),
and `gather_rows` collects per-fly readouts on every rank.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first global fly, fly count) of `rank`: contiguous, sizes differing by at most one."""
    if total < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("need total >= 0, world >= 1 and 0 <= rank < world")
    base, extra = divmod(total, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def allreduce_gradients(tensors, group=None) -> None:
    """Sum each tensor over ranks in place (no-op without an initialised process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def gather_rows(local: torch.Tensor, total: int, group=None) -> torch.Tensor:
    """Concatenate per-rank (count, ...) blocks in rank order into (total, ...) on every rank."""
    if not (dist.is_available() and dist.is_initialized()):
        return local
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    counts = [shard(total, world, r)[1] for r in range(world)]
    width = max(counts)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], 0)
