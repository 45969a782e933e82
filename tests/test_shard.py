"""Multi-rank plumbing of independent chains on CPU: gloo, world size 2 (the N > 1 path of bench.py)."""
import os
import socket

import numpy as np
import torch.multiprocessing as tmp

from fastbart_b200 import shard


def _chains():
    rng = np.random.default_rng(0)
    out = []
    for k in range(13):
        n = int(rng.integers(100, 5000))
        out.append(dict(q=np.zeros((3, n), np.uint8), y=np.zeros(n), ntree=int(rng.integers(20, 201)),
                        nskip=100, ndpost=10))
    return out


def test_shard_partition_is_a_balanced_cover():
    ch = _chains()
    for world in (1, 2, 3, 8):
        parts = [shard.shard_chains(ch, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(ch)))
        loads = [sum(shard.chain_cost(ch[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(shard.chain_cost(c) for c in ch)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _tagged(n=13):
    ch = _chains()[:n]
    for k, c in enumerate(ch):
        c["tag"] = k
    return ch


def _fake_runner(calls):
    """Stands in for the batch call: one output per chain, naming the chain and the device that ran it."""
    def run(sub, device):
        calls.append((device, [c["tag"] for c in sub]))
        return [{"tag": c["tag"], "device": device} for c in sub]
    return run


def test_fit_sharded_partitions_and_gathers_in_order():
    ch = _tagged()
    calls: list = []
    outs = shard.fit_sharded(ch, 100, 10, devices=[3, 5, 7], runner=_fake_runner(calls))
    assert [o["tag"] for o in outs] == list(range(len(ch)))
    for r, d in enumerate((3, 5, 7)):
        mine = shard.shard_chains(ch, r, 3)
        assert all(outs[i]["device"] == d for i in mine)
    assert sorted(d for d, _ in calls) == [3, 5, 7]


def test_fit_sharded_reports_a_failing_device():
    def bad(sub, device):
        if device == 1:
            raise ValueError("out of device memory")
        return [{} for _ in sub]
    import pytest
    with pytest.raises(RuntimeError, match="device 1: out of device memory"):
        shard.fit_sharded(_tagged(), 100, 10, devices=[0, 1], runner=bad)


def _dist_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        calls: list = []
        res = shard.fit_distributed(_tagged(), 100, 10, device=rank, runner=_fake_runner(calls))
        out[rank] = (res, calls)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_gather_chain_outputs():
    world = 2
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    tmp.start_processes(_dist_main, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    res0, calls0 = out[0]
    res1, calls1 = out[1]
    assert res1 is None
    assert [o["tag"] for o in res0] == list(range(13))
    ch = _tagged()
    for r, calls in ((0, calls0), (1, calls1)):
        assert calls == [(r, shard.shard_chains(ch, r, world))]
        assert all(res0[i]["device"] == r for i in shard.shard_chains(ch, r, world))


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.shard_chains(_chains(), rank, world)
        t = shard.max_over_ranks(10.0 + rank)
        out[rank] = (mine, t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_partition_and_max():
    world = 2
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    tmp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    parts = [out[r][0] for r in range(world)]
    assert sorted(parts[0] + parts[1]) == list(range(13)) and not set(parts[0]) & set(parts[1])
    assert [out[r][1] for r in range(world)] == [11.0, 11.0]
    assert shard.max_over_ranks(3.5) == 3.5   # no group: identity
