"""Rank sharding of independent domains, on CPU ranks over gloo (the host
logic the multi-GPU benchmark runs under torchrun with NCCL)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, q):
    import torch.distributed as dist

    from qesb import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.rank_share(n, world, rank)
        slowest = shard.max_over_ranks(10.0 + rank)
        everything = shard.gather_lists([(i, rank) for i in mine])
        q.put((rank, mine, slowest, everything))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [7, 64])
def test_two_ranks_split_units_without_overlap(n):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(n))
    assert not set(shares[0]) & set(shares[1])
    assert abs(len(shares[0]) - len(shares[1])) <= 1
    assert all(r[2] == 11.0 for r in res)
    for r in res:
        assert sorted(i for i, _ in r[3]) == list(range(n))


def test_rank_share_rejects_bad_rank():
    from qesb import shard

    with pytest.raises(ValueError):
        shard.rank_share(4, 2, 2)
