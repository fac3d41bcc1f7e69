"""Frame sharding across ranks (CPU, gloo, world size 2): every output frame is
owned by exactly one rank, every rank has the halo it needs, and timings
reduce to the slowest rank."""
import os

import pytest
import torch.multiprocessing as mp

from dfttest2_b200.shard import frame_shard


def test_frame_shard_covers_clip():
    for total in (1, 7, 64, 129):
        for world in (1, 2, 3, 8):
            if world > total:
                continue
            owned = []
            for rank in range(world):
                lo, hi, in_lo, in_hi = frame_shard(total, rank, world, 1)
                owned += range(lo, hi)
                assert in_lo == max(lo - 1, 0) and in_hi == min(hi + 1, total)
            assert owned == list(range(total))
    with pytest.raises(ValueError):
        frame_shard(10, 2, 2, 1)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from dfttest2_b200.shard import frame_shard, max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lo, hi, in_lo, in_hi = frame_shard(64 * world, rank, world, 1)
    t = torch.tensor([lo, hi], dtype=torch.int64)
    gathered = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(gathered, t)
    slowest = max_over_ranks(1.0 + rank, True)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [tuple(g.tolist()) for g in gathered], slowest))


def test_two_rank_gloo_sharding():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ranges, slowest in results:
        assert ranges == [(0, 64), (64, 128)]
        assert slowest == 2.0
