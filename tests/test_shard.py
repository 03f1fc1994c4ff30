"""Multi-GPU host logic on CPU: cost-balanced shards, and the two collectives
of a multi-rank run (max-over-ranks timing, end-of-run gather of per-filter
log-likelihood sums) on two gloo ranks -- with stand-in values, and with real
filters: each rank runs its share of a small workload through the FP64
oracle (noise keyed by the global filter index, as the engine keys it), and
the gathered sums must equal a one-process run of every filter."""
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


def _oracle_filter_loglik(f, n, params, ys):
    """FP64 oracle run of global filter f (Philox noise keyed by f): the FP64
    sum of its per-tick log-likelihoods."""
    import oracle
    cfg = oracle.default_config(4, 12.0)
    cfg.use_newton, cfg.use_full_newton, cfg.stein_min_steps, cfg.stein_max_steps = 1, 1, 2, 4
    o = oracle.OracleFilter(int(n), cfg, oracle.OracleParams(*params))
    o.initialize(seed=7, filter_id=int(f))
    yp = 0.0
    for t in range(ys.shape[0]):
        o.step(float(ys[t]), yp, seed=7, tick=t, filter_id=int(f))
        yp = float(ys[t])
    return float(o.ctl.loglik_sum)


def _workload(F):
    rng = np.random.default_rng(3)
    ns = rng.choice([16, 32, 48, 64], size=F)
    params = [(float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.1, 0.3)), float(rng.uniform(-2, 0)), 0.0)
              for _ in range(F)]
    ys = (0.3 * rng.standard_normal((F, 4))).astype(np.float32)
    return ns, params, ys


def _real_worker(rank, world, port, F, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        shard = _shard_mod()
        ns, params, ys = _workload(F)
        mine = shard.partition(ns, 4, world)[rank]
        sums = [_oracle_filter_loglik(f, ns[f], params[f], ys[f]) for f in mine]
        full = shard.gather_by_filter(mine, sums, F)
        q.put((rank, mine.tolist(), full.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_real_filters():
    F, world = 10, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_real_worker, args=(r, world, port, F, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ns, params, ys = _workload(F)
    want = np.array([_oracle_filter_loglik(f, ns[f], params[f], ys[f]) for f in range(F)])
    shares = sorted(r[1] for r in results)
    assert sorted(sum(shares, [])) == list(range(F)) and all(shares)   # both ranks worked, no filter twice
    for _, _, full in results:
        assert np.array_equal(np.array(full), want)
