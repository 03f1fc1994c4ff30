"""Parity of the batched engine's headline path with the FP64 oracle.

The benchmark ticks the persistent batch kernel through
svpf_batch_graph_launch (one captured launch per tick, replayed), with the
tile shape per particle count the autotuner picks.  Here that same call is
checked against the oracle (the per-filter tick of the reference,
src/svpf_optimized_graph.cu:915-1389):

* every compiled batch tile (rows per thread, column split) at particle
  counts 64 ... 4096, forced per filter in one batch;
* the first 16 filters of the benchmark's own workload (own theta, own nu,
  N drawn from {256, ..., 4096}) with the autotuner's tiles, over 12 ticks,
  which crosses t = 10 where the KSD-driven Stein budget and rejuvenation
  switch on.

Before every tick the oracle takes the engine's state (control record,
particles, previous particles, RMSProp moments); both sides draw the same
noise tape (captured once in the graph and replayed).  Tolerance 1e-4
relative (floor 1), as the other parity tests; KSD 1e-3.
"""
import concurrent.futures as cf
import os
import sys

import numpy as np
import pytest

import tape
from test_oracle import TOL, rel_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TILES = [(1, 4), (1, 2), (1, 1), (2, 1), (4, 1)]
SIZES = [64, 100, 256, 300, 1024, 2048, 4096]


def _twin(oracle_mod, batch, f, cfg, params, precision=0):
    ctl, h, hp, v, lw = batch.get_state(f)
    # particle count: the log-weights hold n values (h, h_prev, v hold 2n for two factors)
    o = oracle_mod.OracleFilter(lw.shape[0], oracle_mod.config_from_dict(cfg.to_dict()),
                                oracle_mod.OracleParams(*params), precision)
    # every field, the smoother's ring buffers and head included
    o.ctl = oracle_mod.ctl_from_dict({k: getattr(ctl, k) for k, _ in ctl._fields_})
    o.h, o.h_prev, o.v, o.log_w = (a.astype(np.float64) for a in (h, hp, v, lw))
    return o


def _run(pkg, oracle_mod, ns, cfgs, params, ys, ticks, tiles=None, tape_seed=31, slots=None, sensitivity=False):
    """Tick a batch through svpf_batch_graph_launch and the oracle side by side.
    sensitivity: also step the oracle's FP32 mirror from the same state, and
    from that state with the positions moved by about two FP32 ulps either way (three
    rounding paths), and widen each filter's tolerance to four times the
    largest deviation from the FP64 result where that is larger (ticks that
    are ill-conditioned in FP32)."""
    import torch

    F = len(ns)
    n_max = max(ns)
    b = pkg.Batch(ns, cfgs, [pkg.Params(*p) for p in params])
    two_factor = any(c.use_two_factor for c in cfgs)   # a two-factor initialisation draws 3 slots
    init = tape.init_normals(tape_seed, n_max, 3 if two_factor else 1)
    b.set_noise_tape(init if two_factor else init[None, :], np.ones((1, n_max), np.float32))
    b.initialize(seed=1)
    if tiles is not None:
        for f, (R, S) in enumerate(tiles):
            b.set_tile(f, R, S)
    used = [b.tile_of_filter(f) for f in range(F)]
    if slots is None:
        slots = 2 + max(c.stein_max_steps for c in cfgs) + 7
    nrm, uni = tape.tape(tape_seed + 1, 0, n_max, slots, 2)
    b.set_noise_tape(nrm, uni)   # one tape for every tick: the graph is captured once, then replayed
    d_yt = torch.empty(F, dtype=torch.float32, device="cuda")
    d_yp = torch.zeros(F, dtype=torch.float32, device="cuda")
    d_out = torch.zeros((F, 8), dtype=torch.float32, device="cuda")
    launches0 = b.kernel_launches
    pool = cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1))
    for t in range(ticks):
        twins = [_twin(oracle_mod, b, f, cfgs[f], params[f]) for f in range(F)]
        mirrors = []
        if sensitivity:
            for nudge in (0.0, 2.0 ** -22, -(2.0 ** -22)):
                m = [_twin(oracle_mod, b, f, cfgs[f], params[f], 1) for f in range(F)]
                for o in m:
                    o.h = o.h * (1.0 + nudge)
                mirrors.append(m)
        yp = ys[t - 1] if t > 0 else np.zeros(F, np.float32)
        d_yt.copy_(torch.from_numpy(np.ascontiguousarray(ys[t])))
        d_yp.copy_(torch.from_numpy(np.ascontiguousarray(yp)))
        torch.cuda.synchronize()
        b.graph_launch(d_yt.data_ptr(), d_yp.data_ptr(), d_out.data_ptr())
        b.sync()
        out = d_out.cpu().numpy()
        steps = out.view(np.int32)[:, 6]
        rejuv = out.view(np.int32)[:, 7]
        # the oracle's ticks run in threads: each is a ctypes call, which releases the GIL
        oo = list(pool.map(lambda f: twins[f].step(ys[t, f], yp[f], nrm[:, :ns[f]], uni[:, :ns[f]]), range(F)))
        outs32 = [list(pool.map(lambda f: m[f].step(ys[t, f], yp[f], nrm[:, :ns[f]], uni[:, :ns[f]]), range(F)))
                  for m in mirrors]
        ctl = b.ctl()
        for f in range(F):
            tag = (t, f, ns[f], used[f])
            assert ctl[f].status == 0, tag
            assert steps[f] == oo[f].steps_used, tag
            assert rejuv[f] == oo[f].rejuv_fired, tag
            h = b.get_particles(f)

            def tol(base, dev):
                return max(base, 4 * dev) if sensitivity else base

            def dev(name):   # largest deviation of the FP32 mirrors from the FP64 result
                want = getattr(oo[f], name)
                return max((abs(getattr(o[f], name) - want) / max(1.0, abs(want)) for o in outs32), default=0.0)

            th = tol(TOL, max((rel_err(m[f].h, twins[f].h) for m in mirrors), default=0.0))
            assert rel_err(h, twins[f].h) < th, (tag, rel_err(h, twins[f].h), th)
            for col, name in ((0, "loglik"), (1, "vol"), (2, "h_mean")):
                want = getattr(oo[f], name)
                assert abs(out[f, col] - want) < tol(TOL, dev(name)) * max(1.0, abs(want)), (tag, name, out[f, col],
                                                                                              want)
            want = oo[f].ksd
            assert abs(out[f, 5] - want) < tol(1e-3, dev("ksd")) * max(1.0, abs(want)), (tag, out[f, 5], want)
    pool.shutdown()
    # one captured graph per tick, replayed: one persistent launch per tick for
    # each kind of filter in the batch (single-factor, two-factor)
    kinds = int(any(not c.use_two_factor for c in cfgs)) + int(any(c.use_two_factor for c in cfgs))
    assert b.kernel_launches - launches0 == kinds * ticks
    b.close()
    return used


def test_every_batch_tile_matches_oracle(pkg, oracle_mod):
    """Each compiled tile at each size, forced per filter, 3 graph-replayed ticks."""
    ns, tiles, params, cfgs = [], [], [], []
    for i, n in enumerate(SIZES):
        for j, tl in enumerate(TILES):
            ns.append(n)
            tiles.append(tl)
            params.append((0.93 + 0.01 * j, 0.12 + 0.04 * (i % 4), -1.5 + 0.2 * j, -0.1 * (i % 2)))
            cfgs.append(pkg.production_config(5.0 + 4.0 * j, 8))
    F = len(ns)
    _, y = tape.sv_path(4, -1.0, 0.97, 0.2, seed=3)
    ys = np.tile(y[:, None], (1, F)).astype(np.float32) * np.linspace(0.6, 1.4, F, dtype=np.float32)[None, :]
    used = _run(pkg, oracle_mod, ns, cfgs, params, ys, ticks=3, tiles=tiles)
    assert used == tiles


def test_benchmark_workload_slice_matches_oracle(pkg, oracle_mod):
    """The first 16 filters of the benchmark's workload (own theta and nu, N up
    to 4096) with the autotuner's tiles, 12 graph-replayed ticks."""
    sys.path.insert(0, ROOT)
    import bench

    ns_all, rho, sz, mu, nu = bench.make_workload(4096, seed=0)
    Fs = 16
    ns = [int(n) for n in ns_all[:Fs]]
    assert max(ns) == 4096
    chosen = pkg.autotune(sorted(set(ns)), ticks=1)
    ys = bench.sv_paths(12, rho, sz, mu, nu, seed=0)[:, :Fs]
    params = [(float(rho[f]), float(sz[f]), float(mu[f]), 0.0) for f in range(Fs)]
    cfgs = [pkg.production_config(float(nu[f]), bench.MAX_STEPS) for f in range(Fs)]
    used = _run(pkg, oracle_mod, ns, cfgs, params, ys, ticks=12)
    for f, n in enumerate(ns):
        assert used[f] == tuple(chosen[n]), (n, used[f], chosen[n])


def test_tile_hook_rejects_unknown_shapes(pkg):
    b = pkg.Batch([256, 512], pkg.production_config(30.0, 8), pkg.Params(0.97, 0.15, -1.0, 0.0))
    for R, S in ((8, 1), (1, 8), (3, 1), (0, 0)):
        with pytest.raises(RuntimeError):
            b.set_tile(0, R, S)
    with pytest.raises(RuntimeError):
        b.set_tile(2, 1, 4)   # no such filter
    b.set_tile(1, 1, 2)
    assert b.tile_of_filter(1) == (1, 2)
    b.close()


def test_loop_counts_are_bounded(pkg):
    """Configurations whose Stein budget would keep a kernel running for long
    are refused before any launch (SVPF_MAX_STEIN_STEPS = 256 per tick)."""
    ok = pkg.production_config(30.0, 8)
    bad = pkg.production_config(30.0, 8)
    bad.stein_max_steps = 1 << 30
    with pytest.raises(RuntimeError):
        pkg.Batch([256, 256], [ok, bad], pkg.Params(0.97, 0.15, -1.0, 0.0))
    neg = pkg.production_config(30.0, 8)
    neg.stein_min_steps = -(1 << 30)
    with pytest.raises(RuntimeError):
        pkg.Batch([256], [neg], pkg.Params(0.97, 0.15, -1.0, 0.0))
    f = pkg.SVPF(256, 8, 30.0)
    f.initialize(0.97, 0.15, -1.0, 0.0, seed=1)
    f.configure(stein_max_steps=100000)
    rc, _ = f.step_raw(0.1, 0.0)
    assert rc == 1   # SVPF_ERR_INVALID_ARG, nothing launched
    f.configure(stein_max_steps=8)
    rc, _ = f.step_raw(0.1, 0.0)
    assert rc == 0
    f.close()


def test_maximum_particle_count_matches_oracle(pkg, oracle_mod):
    """N = SVPF_MAX_PARTICLES (8192), the largest filter the engine takes:
    the single-filter cluster kernel and the batch kernel (one CTA, ~190 KB
    of shared memory), 2 ticks each against the FP64 oracle."""
    import torch

    n = 8192
    cfg = pkg.production_config(30.0, 8)
    params = (0.97, 0.15, -1.0, 0.0)
    _, ys = tape.sv_path(3, -1.0, 0.97, 0.15, seed=8)
    init = tape.init_normals(41, n)
    slots = 2 + 8 + 7
    nrm, uni = tape.tape(42, 0, n, slots, 2)
    # single filter
    f = pkg.SVPF(n, 8, 30.0)
    f.configure(**cfg.to_dict())
    f.set_noise_tape(init[None, :], np.ones((1, n), np.float32))
    f.initialize(*params, seed=1)
    # batch of one
    b = pkg.Batch([n], cfg, pkg.Params(*params))
    b.set_noise_tape(init[None, :], np.ones((1, n), np.float32))
    b.initialize(seed=1)
    b.set_noise_tape(nrm, uni)
    f.set_noise_tape(nrm, uni)
    d_out = torch.zeros((1, 8), dtype=torch.float32, device="cuda")
    yp = 0.0
    for t in range(2):
        ctl, h, hp, v, lw = f.get_state()
        o1 = oracle_mod.OracleFilter(n, oracle_mod.config_from_dict(cfg.to_dict()), oracle_mod.OracleParams(*params))
        o1.ctl = oracle_mod.ctl_from_dict({k: getattr(ctl, k) for k, _ in ctl._fields_ if not k.startswith("smooth_")})
        o1.h, o1.h_prev, o1.v, o1.log_w = (a.astype(np.float64) for a in (h, hp, v, lw))
        o2 = _twin(oracle_mod, b, 0, cfg, params)
        rc, out = f.step_raw(ys[t], yp)
        assert rc == 0
        d_yt = torch.tensor([ys[t]], dtype=torch.float32, device="cuda")
        d_yp = torch.tensor([yp], dtype=torch.float32, device="cuda")
        b.step_device(d_yt.data_ptr(), d_yp.data_ptr(), d_out.data_ptr())
        b.sync()
        with cf.ThreadPoolExecutor(2) as ex:
            oo1, oo2 = ex.map(lambda o: o.step(ys[t], yp, nrm, uni), (o1, o2))
        yp = float(ys[t])
        assert rel_err(f.get_particles(), o1.h) < TOL and abs(out.loglik - oo1.loglik) < TOL * max(1, abs(oo1.loglik))
        assert rel_err(b.get_particles(0), o2.h) < TOL
        ob = d_out.cpu().numpy()
        assert abs(ob[0, 0] - oo2.loglik) < TOL * max(1, abs(oo2.loglik))
        assert out.steps_used == oo1.steps_used and int(ob.view(np.int32)[0, 6]) == oo2.steps_used
    f.close()
    b.close()
