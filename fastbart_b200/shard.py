"""Multi-GPU plumbing for independent chains: one process per GPU, no exchange on the data path.

Chains share nothing while they sample, so a set of chains is partitioned across ranks and each rank runs its part
as one batch on its own GPU (src/bart_kernel.cpp:304-580 is per chain; gpu/bart_gpu.cu:326-404 batches independent
fits the same way on one GPU).  The only collective is the timing reduction (max over ranks) and, when wanted, the
gather of per-chain outputs to one rank.
"""
from __future__ import annotations

from typing import Sequence


def chain_cost(ch: dict) -> int:
    """Work of one chain: rows x (trees + 1) x sweeps (one fused pass per tree plus the end-of-sweep refresh)."""
    n = int(ch["q"].shape[1]) if hasattr(ch["q"], "shape") else len(ch["y"])
    return n * (int(ch["ntree"]) + 1) * (int(ch["nskip"]) + int(ch["ndpost"]))


def shard_chains(chains: Sequence[dict], rank: int, world: int) -> list[int]:
    """Indices of the chains rank `rank` of `world` runs: longest-processing-time assignment (largest cost first,
    each to the least-loaded rank, ties to the lower rank), deterministic, so every rank computes the same partition
    without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    order = sorted(range(len(chains)), key=lambda i: (-chain_cost(chains[i]), i))
    load = [0] * world
    owner = [0] * len(chains)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += chain_cost(chains[i])
    return [i for i in range(len(chains)) if owner[i] == rank]


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank number (e.g. device-timed milliseconds) over the default process group; x itself when
    no group is initialised.  `device` is the tensor device the backend needs (a CUDA device for NCCL)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
