"""Multi-GPU search, one process per GPU.

Two ways to split the work, both over ``torch.distributed`` (NCCL for GPUs;
the gathering helpers also run on CPU tensors with gloo):

* query sharding (``match_sharded``): every rank holds the whole base and
  searches a contiguous slice of the queries with the single-GPU path, no
  collective inside the search; one all-gather assembles the results when
  every rank wants all of them.
* base sharding (``match_base_sharded``): every rank holds a slice of the
  base (a base too large for one GPU, or many GPUs on one query set) and
  searches all queries against it; one all-gather of the per-query top-2
  lists (16 bytes per query per rank) and a merge kernel give every rank the
  result of one search over the whole base.
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


def gather_parts(nn_idx, nn_dist, base_offset: int, group=None):
    """All ranks' per-query top-2 lists ([q, 2] int32 indices local to the
    rank's base slice, [q, 2] float32 distances) and slice offsets, stacked in
    rank order: ([world, q, 2], [world, q, 2], list of world offsets)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    idx_parts = [torch.empty_like(nn_idx) for _ in range(world)]
    dist_parts = [torch.empty_like(nn_dist) for _ in range(world)]
    dist.all_gather(idx_parts, nn_idx.contiguous(), group=group)
    dist.all_gather(dist_parts, nn_dist.contiguous(), group=group)
    off = torch.tensor([int(base_offset)], dtype=torch.int64, device=nn_idx.device)
    offs = [torch.empty_like(off) for _ in range(world)]
    dist.all_gather(offs, off, group=group)
    return torch.stack(idx_parts), torch.stack(dist_parts), [int(o.item()) for o in offs]


def match_base_sharded(q, r_local, base_offset: int, threshold: float = 0.8, group=None):
    """Exact 2-NN of the queries q (the same on every rank) against a base
    split over the ranks: this rank holds rows [base_offset, base_offset +
    r_local.shape[0]) of it (disjoint slices, e.g. from shard_range).

    Returns {"matches", "nn_idx", "nn_dist"} with global base indices, equal on
    every rank and equal to one search over the whole base.
    """
    from . import match

    local = match(q, r_local, threshold=threshold, outputs=("nn_idx", "nn_dist"))
    idx_parts, dist_parts, offsets = gather_parts(local["nn_idx"], local["nn_dist"], base_offset, group)
    return merge_parts(idx_parts, dist_parts, offsets, threshold)


def merge_parts(idx_parts, dist_parts, offsets, threshold: float = 0.8):
    """The merge of match_base_sharded on stacked [parts, q, 2] CUDA tensors
    (already gathered, or searched one after another on one GPU)."""
    import ctypes

    import numpy as np
    import torch

    from . import check, lib

    parts, n = idx_parts.shape[0], idx_parts.shape[1]
    out = {"matches": torch.empty(n, dtype=torch.int32, device=idx_parts.device),
           "nn_idx": torch.empty((n, 2), dtype=torch.int32, device=idx_parts.device),
           "nn_dist": torch.empty((n, 2), dtype=torch.float32, device=idx_parts.device)}
    offs = np.asarray(offsets, dtype=np.int32)
    s = torch.cuda.current_stream(idx_parts.device)
    check(lib().sift_merge_top2(dist_parts.contiguous().data_ptr(), idx_parts.contiguous().data_ptr(),
                                offs.ctypes.data_as(ctypes.c_void_p), parts, n, threshold,
                                out["matches"].data_ptr(), out["nn_idx"].data_ptr(), out["nn_dist"].data_ptr(),
                                s.cuda_stream), "sift_merge_top2")
    if hasattr(torch, "uint32"):
        out["matches"] = out["matches"].view(torch.uint32)  # as match() returns them
    return out
