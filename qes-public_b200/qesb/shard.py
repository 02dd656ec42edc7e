"""Independent domains across ranks (one process per GPU).

A lambda solve does not shard: one domain lives on one GPU. What shards are
independent domains (a batch of cities, an ensemble's cities): each rank takes
its own share, no data crosses ranks during the solves, and only scalars and
per-solve statistics are combined at the end (torch.distributed, NCCL on GPUs,
gloo on CPU).
"""
from __future__ import annotations


def rank_share(n: int, world: int, rank: int) -> list[int]:
    """Indices of the n units that rank `rank` of `world` takes (round robin,
    so uneven units spread evenly)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return list(range(rank, n, world))


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank float over all ranks (the slowest rank's time)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_lists(values: list, device=None) -> list:
    """Concatenation over ranks of each rank's list (rank order)."""
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(values))
    return [v for part in out for v in part]


def rank_seeds(seed0: int, batch: int, rank: int) -> list[int]:
    """Seeds of the cities rank `rank` solves when every rank takes its own
    batch of `batch` cities (weak scaling): seed0 + rank*batch + i."""
    if batch < 1 or rank < 0:
        raise ValueError(f"batch {batch}, rank {rank}")
    return [seed0 + rank * batch + i for i in range(batch)]


def launch_command(python: str, script: str, nproc: int, port: int, argv: list[str]) -> list[str]:
    """The torch.distributed.run command line that runs `script` as `nproc`
    ranks on one node, rendezvous on 127.0.0.1:port."""
    if nproc < 1:
        raise ValueError(f"nproc {nproc}")
    return [python, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), script, *argv]
