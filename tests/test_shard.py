"""Multi-GPU host logic on CPU: cost-balanced shards, and the two collectives
of a multi-rank run (max-over-ranks timing, end-of-run gather of per-filter
log-likelihood sums) on two gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _shard_mod():
    import __graft_entry__ as ge
    ge.load_package()
    import importlib
    return importlib.import_module("svpf_b200.shard")


def test_partition_covers_every_filter_once_and_balances():
    shard = _shard_mod()
    rng = np.random.default_rng(0)
    ns = rng.choice([256, 512, 1024, 2048, 4096], size=4096)
    for world in (1, 2, 3, 8):
        shares = shard.partition(ns, 8, world)
        allidx = np.concatenate(shares)
        assert np.array_equal(np.sort(allidx), np.arange(ns.shape[0]))
        assert shard.imbalance(ns, 8, shares) < 1.01
    # more ranks than filters: some shares are empty, none duplicated
    shares = shard.partition([4096, 256], 8, 4)
    assert sorted(np.concatenate(shares).tolist()) == [0, 1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, ns, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        shard = _shard_mod()
        shares = shard.partition(ns, 8, world)
        mine = shares[rank]
        values = mine.astype(np.float64) * 0.5 - 3.0       # stand-in per-filter log-likelihood sums
        full = shard.gather_by_filter(mine, values, len(ns))
        t = shard.max_over_ranks(1.0 + rank)
        q.put((rank, full.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_time():
    ns = np.array([4096, 256, 512, 2048, 1024, 256, 512, 4096, 300], dtype=np.int64)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, ns, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expected = np.arange(len(ns)) * 0.5 - 3.0
    for rank, full, t in results:
        assert np.allclose(full, expected)
        assert t == 2.0
