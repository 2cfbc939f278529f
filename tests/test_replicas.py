"""Multi-process (world_size 2, gloo, CPU) checks of the replica bookkeeping
that bench.py and multi-GPU simulations use: frame sharding, max-over-ranks
timing and the sum of Monte-Carlo counters."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fast_ldpc_decoder_for_gpu_fixed_b200 import replicas


def test_shard_partitions_frames():
    for total in (4, 64, 65536, 65540, 1000):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(total, r, world) for r in range(world)]
            assert sum(c for _, c in parts) == total // 4 * 4
            starts = [s for s, _ in parts]
            assert starts == sorted(starts)
            for (s0, c0), (s1, _) in zip(parts, parts[1:]):
                assert s0 + c0 == s1
            assert all(s % 4 == 0 and c % 4 == 0 for s, c in parts)


def test_channel_offsets_disjoint():
    offs = {replicas.channel_offset(r, b) for r in range(8) for b in range(100)}
    assert len(offs) == 800


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = replicas.max_over_ranks(10.0 + rank)
        counts = torch.tensor([100 * (rank + 1), 7 * rank, rank], dtype=torch.int64)
        replicas.sum_counters(counts)
        q.put((rank, t, counts.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, counts in res:
        assert t == 11.0
        assert counts == [300, 7, 1]
