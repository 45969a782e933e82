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


def _default_runner(nskip: int, ndpost: int, kw: dict):
    def run(sub: list, device: int) -> list:
        from .api import fit_batch
        return fit_batch(sub, nskip, ndpost, device=device, **kw)
    return run


def fit_sharded(chains: Sequence[dict], nskip: int, ndpost: int, devices: Sequence[int], runner=None,
                **kw) -> list:
    """Runs a set of independent chains on several GPUs of this process: the longest-processing-time partition of
    shard_chains gives each device its share, one host thread per device runs that share as one batch (the library's
    calls release the interpreter and are thread-safe across batches), and the outputs come back in the order of
    `chains`.  runner(sub_chains, device) -> outputs replaces the batch call (tests use a fake one)."""
    import threading
    devices = list(devices)
    if not devices:
        raise ValueError("devices is empty")
    run = runner or _default_runner(nskip, ndpost, kw)
    parts = [shard_chains(chains, r, len(devices)) for r in range(len(devices))]
    results: list = [None] * len(chains)
    errors: list = []

    def work(r: int):
        try:
            idx = parts[r]
            if idx:
                outs = run([chains[i] for i in idx], devices[r])
                for i, o in zip(idx, outs):
                    results[i] = o
        except BaseException as e:   # re-raised in the caller's thread
            errors.append((r, e))

    threads = [threading.Thread(target=work, args=(r,)) for r in range(len(devices))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        r, e = min(errors, key=lambda x: x[0])
        raise RuntimeError(f"device {devices[r]}: {e}") from e
    return results


def fit_distributed(chains: Sequence[dict], nskip: int, ndpost: int, device: int, runner=None, dst: int = 0,
                    **kw):
    """One process per GPU (torch.distributed initialised, e.g. under torchrun): every rank runs its shard_chains share
    of `chains` on `device`, and the per-chain outputs are gathered to rank `dst` in the order of `chains`.  Returns the
    full list on rank dst and None elsewhere.  The only collective is that gather, after sampling."""
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    run = runner or _default_runner(nskip, ndpost, kw)
    idx = shard_chains(chains, rank, world)
    outs = run([chains[i] for i in idx], device) if idx else []
    mine = list(zip(idx, outs))
    got = [None] * world if rank == dst else None
    dist.gather_object(mine, got, dst=dst)
    if rank != dst:
        return None
    results: list = [None] * len(chains)
    for part in got:
        for i, o in part:
            results[i] = o
    return results


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
