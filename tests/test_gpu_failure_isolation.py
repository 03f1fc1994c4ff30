"""A bad observation stays with its filter.

A feed glitch -- a NaN or infinite return -- must neither touch the other
filters of a batch nor destroy the filter that received it.  The engine
refuses a non-finite y_t: that filter's tick leaves its state exactly as it
was (particles, moments, control record, tick counter) and reports
SVPF_ERR_NONFINITE with NaN outputs; a non-finite y_prev is read as 0 (no
leverage) and flagged the same way while the tick runs.  The reference runs
such ticks: its clamps pin the particles to a bound and its EKF carries the
NaN, so its later ticks report finite nonsense.

No GPU fault is involved: the refusal is an ordinary branch of the tick.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

PARAMS = (0.97, 0.15, -1.0, 0.0)
NONFINITE = 5


def _state_bits(b, f):
    ctl, h, hp, v, lw = b.get_state(f)
    return bytes(ctl), tuple(a.view(np.uint32).tobytes() for a in (h, hp, v, lw))


def _state_bits_no_status(b, f):
    ctl, h, hp, v, lw = b.get_state(f)
    ctl.status = 0
    return bytes(ctl), tuple(a.view(np.uint32).tobytes() for a in (h, hp, v, lw))


def _batch(pkg):
    ns = [512, 256, 1024, 300, 384, 2048]
    c1 = pkg.production_config(7.0, 8)
    c2 = pkg.default_config(4, 7.0)
    c2.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    cfgs = [c1, c1, c1, c1, c2, c2]   # filters 4 and 5 are two-factor
    b = pkg.Batch(ns, cfgs, pkg.Params(*PARAMS))
    b.initialize(seed=3)
    return b, ns


def test_nonfinite_observation_is_refused_and_isolated(pkg):
    a, ns = _batch(pkg)
    b, _ = _batch(pkg)
    F = len(ns)
    rng = np.random.default_rng(0)
    ys = (0.02 * rng.standard_normal((8, F))).astype(np.float32)
    yp = np.zeros(F, np.float32)
    for t in range(3):   # a few ordinary ticks first
        for x in (a, b):
            x.step(ys[t], yp)
        yp = ys[t].copy()
    bad = {1: np.nan, 4: np.inf}   # a single-factor and a two-factor filter
    before = {f: _state_bits(a, f) for f in bad}
    y_bad = ys[3].copy()
    for f, v in bad.items():
        y_bad[f] = v
    ll_a, vol_a, hm_a = a.step(y_bad, yp)
    ll_b, vol_b, hm_b = b.step(ys[3], yp)
    ctl_a = a.ctl()
    for f in range(F):
        if f in bad:
            assert ctl_a[f].status == NONFINITE, f
            assert np.isnan(ll_a[f]) and np.isnan(vol_a[f]) and np.isnan(hm_a[f]), f
            ctl_bits, arrays = _state_bits(a, f)
            ctl_before, arrays_before = before[f]
            assert arrays == arrays_before, f            # particles, moments, log-weights untouched
            c0, c1 = pkg.Ctl.from_buffer_copy(ctl_before), pkg.Ctl.from_buffer_copy(ctl_bits)
            c0.status = c1.status = 0
            assert bytes(c0) == bytes(c1), f             # control record untouched but for the status
        else:
            assert ctl_a[f].status == 0, f
            assert _state_bits(a, f) == _state_bits(b, f), f   # the other filters: the same bits
            assert (ll_a[f], vol_a[f], hm_a[f]) == (ll_b[f], vol_b[f], hm_b[f]), f
    # next tick: finite y_t everywhere; filter 2 receives y_prev = NaN in batch
    # a and y_prev = 0 in batch b, which must give the same bits
    yp_a = ys[3].copy()
    for f in bad:
        yp_a[f] = yp[f]          # the caller keeps its last finite observation
    yp_a[2] = np.nan
    yp_b = ys[3].copy()
    yp_b[2] = 0.0
    ll_a, _, _ = a.step(ys[4], yp_a)
    b.step(ys[4], yp_b)
    ctl_a, ctl_b = a.ctl(), b.ctl()
    for f in bad:                # the refused filters step normally again
        assert ctl_a[f].status == 0, f
        assert np.isfinite(ll_a[f]) and np.isfinite(a.get_particles(f)).all(), f
    assert ctl_a[2].status == NONFINITE and ctl_b[2].status == 0
    assert _state_bits_no_status(a, 2) == _state_bits_no_status(b, 2)
    for f in (0, 3, 5):
        assert _state_bits(a, f) == _state_bits(b, f), f
    a.close()
    b.close()


def test_single_filter_refuses_nonfinite_observation(pkg):
    """svpf_step_graph on one filter: a NaN y_t leaves the state (and the
    tick counter, which keys the noise) unchanged, so the next tick equals the
    tick of a twin filter that never saw the NaN, bit for bit."""
    n = 512
    cfg = pkg.production_config(9.0, 8)
    fs = []
    for _ in range(2):
        f = pkg.SVPF(n, 8, 9.0)
        f.configure(**cfg.to_dict())
        f.initialize(*PARAMS, seed=11)
        fs.append(f)
    a, b = fs
    for y, yp in ((0.01, 0.0), (-0.03, 0.01)):
        for f in fs:
            assert f.step_raw(y, yp)[0] == 0
    before = a.get_state()
    rc, out = a.step_raw(float("nan"), -0.03)
    assert rc == NONFINITE and np.isnan(out.loglik)
    after = a.get_state()
    for x, y in zip(before[1:], after[1:]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert after[0].timestep == before[0].timestep
    ra, oa = a.step_raw(0.02, -0.03)
    rb, ob = b.step_raw(0.02, -0.03)
    assert ra == rb == 0
    assert (oa.loglik, oa.vol, oa.h_mean) == (ob.loglik, ob.vol, ob.h_mean)
    assert np.array_equal(a.get_particles().view(np.uint32), b.get_particles().view(np.uint32))
    for f in fs:
        f.close()


def test_request_loop_refuses_nonfinite_request(pkg):
    """The request loop keeps each instrument's previous observation on the
    device; a refused (NaN) request leaves it, and the instrument's state, as
    they were, so the instrument's next request equals the request of a twin
    loop that never received the NaN, bit for bit.  The two-factor
    instrument is refused the same way."""
    ns = [256, 512, 384]
    c1 = pkg.production_config(7.0, 8)
    c2 = pkg.default_config(4, 7.0)
    c2.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    cfgs = [c1, c1, c2]
    prm = pkg.Params(*PARAMS)
    loops = []
    for _ in range(2):
        s = pkg.Stream(4, 32 << 20, 512, seed=9)
        for f in range(3):
            assert s.admit(ns[f], cfgs[f], prm, seed=9) == f
        loops.append(s)
    a, b = loops
    slots = np.arange(3, dtype=np.int32)
    for y in (0.01, -0.02):
        for s in loops:
            s.process(slots, np.full(3, y, np.float32))
    before = [(bytes(a.ctl(f)), a.particles(f).tobytes()) for f in range(3)]
    out = a.process(np.array([0, 2], np.int32), np.array([np.nan, np.nan], np.float32))
    for r, f in enumerate((0, 2)):
        assert np.isnan(out[r].loglik), f
        c = a.ctl(f)
        assert c.status == NONFINITE, f
        c.status = pkg.Ctl.from_buffer_copy(before[f][0]).status
        assert bytes(c) == before[f][0], f              # y_prev, tick counter and the rest untouched
        assert a.particles(f).tobytes() == before[f][1], f
    ya = a.process(slots, np.full(3, 0.03, np.float32))
    yb = b.process(slots, np.full(3, 0.03, np.float32))
    for f in range(3):
        assert a.ctl(f).status == 0 and bytes(a.ctl(f)) == bytes(b.ctl(f)), f
        assert a.particles(f).tobytes() == b.particles(f).tobytes(), f
        assert (ya[f].loglik, ya[f].h_mean) == (yb[f].loglik, yb[f].h_mean), f
    for s in loops:
        s.close()


def test_multiscale_refuses_nonfinite_return(pkg):
    """The two-scale composition: a NaN return is refused by both scales of
    its instrument and leaves the composition's own state (surprise EMA,
    previous volatility and return) as it was, so the instrument's next step
    equals, bit for bit, the step of a twin that never received the NaN; the
    other instrument is untouched by it."""
    base = [pkg.Params(0.97, 0.15, -1.0, 0.0), pkg.Params(0.95, 0.2, -0.5, 0.0)]
    ms = []
    for _ in range(3):
        m = pkg.MultiScale(base)
        m.init(0.01, seed=5)
        ms.append(m)
    a, b, c = ms
    for y in ((0.01, -0.02), (-0.015, 0.03)):
        for m in ms:
            m.step(np.array(y, np.float32))
    oa = a.step(np.array([np.nan, 0.02], np.float32))
    ob = b.step(np.array([0.0, 0.02], np.float32))
    assert np.isnan(oa[0].h_combined) and np.isnan(oa[0].vol_combined)
    assert bytes(oa[1]) == bytes(ob[1])     # the other instrument: the same bits
    # c never sees the NaN step (instrument 1 of c then differs: not compared)
    oa = a.step(np.array([0.01, 0.01], np.float32))
    oc = c.step(np.array([0.01, 0.01], np.float32))
    assert np.isfinite(oa[0].h_combined) and bytes(oa[0]) == bytes(oc[0])
    for m in ms:
        m.close()
