"""Query sharding over several GPUs, one process per GPU.

The search shards by queries: every rank holds the whole base, matches a
contiguous slice of the queries with the single-GPU path (no collective inside
the search) and, when the caller wants every rank to see every result, one
all-gather assembles them. Ranks and the process group come from
``torch.distributed`` (NCCL for GPUs; the gathering helper also runs on CPU
tensors with gloo).
"""
from __future__ import annotations


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [start, end) slice of n rows for `rank` of `world`; sizes
    differ by at most one and the slices cover [0, n) in rank order."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} world={world} rank={rank}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_rows(local, n_total: int, group=None):
    """All ranks' row blocks (rank order, each from shard_range) concatenated
    into one [n_total, ...] tensor on every rank; one all_gather of blocks
    padded to the largest shard."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    start, end = shard_range(n_total, world, rank)
    if local.shape[0] != end - start:
        raise ValueError(f"rank {rank}: {local.shape[0]} rows, its shard has {end - start}")
    width = -(-n_total // world) if n_total else 0
    padded = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    out = [parts[r][: shard_range(n_total, world, r)[1] - shard_range(n_total, world, r)[0]] for r in range(world)]
    return torch.cat(out, 0) if out else padded[:0]


def match_sharded(q, r, threshold: float = 0.8, group=None, gather: bool = True):
    """Exact 2-NN of all queries q against the base r (both on this rank's
    GPU), each rank searching its shard_range of the queries.

    Returns {"matches", "nn_idx", "nn_dist"} for this rank's shard, or for all
    queries when `gather` (one all-gather per output).
    """
    import torch.distributed as dist

    from . import match

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    start, end = shard_range(q.shape[0], world, rank)
    out = match(q[start:end], r, threshold=threshold, outputs=("matches", "nn_idx", "nn_dist"))
    if gather:
        import torch

        gathered = {}
        for k, v in out.items():
            u32 = hasattr(torch, "uint32") and v.dtype == torch.uint32
            g = gather_rows(v.view(torch.int32) if u32 else v, q.shape[0], group)
            gathered[k] = g.view(torch.uint32) if u32 else g
        out = gathered
    return out
