"""Checkpoint and resume.

A filter's whole state is its control record (EKF, bandwidth and return
EMAs, KSD, smoother, adaptive mu, tick counter, FP64 log-likelihood sum) and
its particle arrays (positions, previous positions, RMSProp moments,
log-weights).  The noise is counter based, keyed by (seed, filter, particle,
draw, tick), so no RNG state exists beyond the tick counter.  A snapshot
taken with svpf_get_state / svpf_batch_get_state and restored into a fresh
filter (same configuration, same seed) therefore resumes the run exactly:
every later tick's outputs and state are the same bits.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

PARAMS = (0.97, 0.15, -1.0, 0.0)


def _ys(T, F, seed=2):
    return (0.02 * np.random.default_rng(seed).standard_t(5, size=(T, F))).astype(np.float32)


def test_single_filter_resumes_from_a_snapshot(pkg):
    n, T, k = 512, 20, 8
    cfg = pkg.production_config(6.0, 8)
    cfg.update(use_smoothing=1, smooth_lag=4, smooth_output_lag=1, use_adaptive_mu=1)
    ys = _ys(T, 1)[:, 0]

    def make():
        f = pkg.SVPF(n, 8, 6.0)
        f.configure(**cfg.to_dict())
        f.initialize(*PARAMS, seed=21)
        return f

    a = make()
    snap, ref = None, []
    yp = 0.0
    for t in range(T):
        if t == k:
            snap = a.get_state()
        rc, out = a.step_raw(float(ys[t]), yp)
        assert rc == 0
        if t >= k:
            ref.append((out.loglik, out.vol, out.h_mean, out.steps_used))
        yp = float(ys[t])
    end = a.get_state()
    b = make()
    b.step_raw(0.05, 0.0)                         # a fresh filter that has moved on elsewhere
    b.set_state(*snap)
    yp = float(ys[k - 1])
    for t in range(k, T):
        rc, out = b.step_raw(float(ys[t]), yp)
        assert rc == 0
        assert (out.loglik, out.vol, out.h_mean, out.steps_used) == ref[t - k], t
        yp = float(ys[t])
    got = b.get_state()
    assert bytes(got[0]) == bytes(end[0])
    for x, y in zip(got[1:], end[1:]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    a.close()
    b.close()


def test_batch_resumes_from_a_snapshot(pkg):
    """A mixed batch (single- and two-factor filters): snapshot every filter
    at tick k, restore into a new batch, replay: the same bits."""
    ns = [256, 512, 1024, 300, 384, 640]
    c1 = pkg.production_config(7.0, 8)
    c2 = pkg.default_config(4, 7.0)
    c2.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    cfgs = [c1, c1, c1, c1, c2, c2]
    F, T, k = len(ns), 14, 6
    ys = _ys(T, F, seed=4)

    def make():
        b = pkg.Batch(ns, cfgs, pkg.Params(*PARAMS))
        b.initialize(seed=8)
        return b

    a = make()
    snap, ref = None, []
    zeros = np.zeros(F, np.float32)
    for t in range(T):
        if t == k:
            snap = [a.get_state(f) for f in range(F)]
        out = a.step(ys[t], ys[t - 1] if t else zeros)
        if t >= k:
            ref.append([o.copy() for o in out])
    end = [a.get_state(f) for f in range(F)]
    b = make()
    for f in range(F):
        b.set_state(f, *snap[f])
    for t in range(k, T):
        out = b.step(ys[t], ys[t - 1])
        for got, want in zip(out, ref[t - k]):
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), t
    for f in range(F):
        got = b.get_state(f)
        assert bytes(got[0]) == bytes(end[f][0]), f
        for x, y in zip(got[1:], end[f][1:]):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f
    a.close()
    b.close()
