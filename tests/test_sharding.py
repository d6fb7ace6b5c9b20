"""Query sharding across ranks: the split on its own, the all-gather with two
gloo ranks on CPU (world size 2), and the sharded GPU match with one rank."""
import os
import socket

import numpy as np
import pytest

from matching_sift_b200.sharding import gather_rows, shard_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("n", [0, 1, 7, 10, 10000, 10001])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_range_covers_in_order(n, world):
    spans = [shard_range(n, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_shard_range_rejects_bad_requests():
    with pytest.raises(ValueError):
        shard_range(10, 0, 0)
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _gather_worker(rank, world, port, n, q):
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        a, b = shard_range(n, world, rank)
        rows = torch.arange(a, b, dtype=torch.int64)
        local = torch.stack([rows * 10, rows * 10 + 1], 1).to(torch.int32)  # [shard, 2] like nn_idx
        full = gather_rows(local, n)
        want = torch.stack([torch.arange(n) * 10, torch.arange(n) * 10 + 1], 1).to(torch.int32)
        q.put((rank, bool(torch.equal(full, want))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1, 9, 1000])
def test_gather_rows_two_gloo_ranks(n):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    results = sorted(q.get(timeout=10) for _ in procs)
    assert [p.exitcode for p in procs] == [0, 0]
    assert results == [(0, True), (1, True)]


@pytest.mark.gpu
def test_match_sharded_single_rank_gpu(cuda_device):
    """One NCCL rank: the sharded call equals the direct call."""
    import torch
    import torch.distributed as dist

    import matching_sift_b200 as ms
    from matching_sift_b200 import datagen
    from matching_sift_b200.sharding import match_sharded

    q, r = datagen.make_workload(1000, 20000, seed=3)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            device_id=cuda_device)
    try:
        got = match_sharded(qd, rd)
        want = ms.match(qd, rd, outputs=("matches", "nn_idx", "nn_dist"))
        for k in want:
            assert torch.equal(got[k], want[k]), k
    finally:
        dist.destroy_process_group()


def _parts_worker(rank, world, port, n, q):
    import torch
    import torch.distributed as dist

    from matching_sift_b200.sharding import gather_parts

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        idx = torch.arange(2 * n, dtype=torch.int32).reshape(n, 2) + 1000 * rank
        dst = idx.to(torch.float32) * 0.5
        ip, dp, offs = gather_parts(idx, dst, base_offset=rank * 777)
        ok = (tuple(ip.shape) == (world, n, 2) and offs == [r * 777 for r in range(world)]
              and all(torch.equal(ip[r], torch.arange(2 * n, dtype=torch.int32).reshape(n, 2) + 1000 * r)
                      for r in range(world))
              and torch.equal(dp, ip.to(torch.float32) * 0.5))
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_gather_parts_two_gloo_ranks():
    """Base sharding: every rank receives all ranks' top-2 lists and slice offsets in rank order."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_parts_worker, args=(r, 2, port, 13, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    results = sorted(q.get(timeout=10) for _ in procs)
    assert [p.exitcode for p in procs] == [0, 0]
    assert results == [(0, True), (1, True)]


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 3, 8])
def test_base_shards_merge_to_the_whole_search(cuda_device, parts):
    """The base split into `parts` slices searched one after another on one GPU
    and merged by the kernel of match_base_sharded equals one search over the
    whole base (indices, distances, ratio-test matches), bit for bit."""
    import torch

    import matching_sift_b200 as ms
    from matching_sift_b200 import datagen
    from matching_sift_b200.sharding import merge_parts

    q, r = datagen.make_workload(3000, 50000, seed=8)
    # duplicate base rows across slice boundaries: ties must resolve to the lower global index
    r[shard_range(50000, parts, 1)[0]] = r[0]
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    want = ms.match(qd, rd, outputs=("matches", "nn_idx", "nn_dist"))
    idx_parts, dist_parts, offs = [], [], []
    for p in range(parts):
        a, b = shard_range(r.shape[0], parts, p)
        o = ms.match(qd, rd[a:b], outputs=("nn_idx", "nn_dist"))
        idx_parts.append(o["nn_idx"])
        dist_parts.append(o["nn_dist"])
        offs.append(a)
    got = merge_parts(torch.stack(idx_parts), torch.stack(dist_parts), offs)
    for k in want:
        assert torch.equal(got[k], want[k]), k


@pytest.mark.gpu
def test_match_base_sharded_single_rank_gpu(cuda_device):
    """One NCCL rank holding the whole base: the base-sharded call equals the direct call."""
    import torch
    import torch.distributed as dist

    import matching_sift_b200 as ms
    from matching_sift_b200 import datagen
    from matching_sift_b200.sharding import match_base_sharded

    q, r = datagen.make_workload(800, 30000, seed=4)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            device_id=cuda_device)
    try:
        got = match_base_sharded(qd, rd, 0)
        want = ms.match(qd, rd, outputs=("matches", "nn_idx", "nn_dist"))
        for k in want:
            assert torch.equal(got[k], want[k]), k
    finally:
        dist.destroy_process_group()
