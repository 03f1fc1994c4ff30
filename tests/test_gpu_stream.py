"""Request loop (svpf_stream_* through the C ABI): instruments admitted into a
fixed HBM budget, requests served in rounds.  Slot f with the same seeds is
the same filter as filter f of a batch, so every request must reproduce the
batch tick (same code, same noise): compared within the parity tolerance.
Also: repeated requests for one instrument in one call run in order, mixed
single/two-factor fleets, admission refusal at the budget and reuse after
eviction, and the device-array round."""
import numpy as np
import pytest

import cases
from test_oracle import TOL, rel_err

pytestmark = pytest.mark.gpu

SEED = 17


def fleet(pkg, F, two_factor_every=0):
    rng = np.random.default_rng(4)
    ns = rng.choice([64, 128, 256, 300, 512], size=F).astype(np.int32)
    cfgs, prms = [], []
    for f in range(F):
        c = pkg.default_config(4, float(rng.uniform(5, 20)))
        if two_factor_every and f % two_factor_every == 0:
            c.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2, nu=6.0, rho_fast=0.80, sigma_fast=0.30,
                            rho_slow=0.995, sigma_slow=0.05))
        else:
            c.update(**cases.PRODUCTION)
            c.update(stein_max_steps=4, stein_min_steps=2)
        cfgs.append(c)
        prms.append(pkg.Params(float(rng.uniform(0.9, 0.99)), float(rng.uniform(0.1, 0.3)),
                               float(rng.uniform(-2, 0)), 0.0))
    return ns, cfgs, prms


def observations(F, T, seed=0):
    return (0.02 * np.random.default_rng(seed).standard_t(6, size=(T, F))).astype(np.float32)


@pytest.mark.parametrize("two_factor_every", [0, 3], ids=["single_factor", "mixed"])
def test_requests_reproduce_batch_ticks(pkg, two_factor_every):
    F, T = 24, 4
    ns, cfgs, prms = fleet(pkg, F, two_factor_every)
    ys = observations(F, T)
    b = pkg.Batch(ns, cfgs, prms)
    b.initialize(seed=SEED)
    s = pkg.Stream(F, 64 << 20, int(ns.max()), seed=SEED)
    for f in range(F):
        assert s.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED) == f
    for f in range(F):
        assert rel_err(s.particles(f), b.get_particles(f)) == 0.0
    order = np.random.default_rng(1).permutation(F)
    for t in range(T):
        ll, vol, hm = b.step(ys[t], ys[t - 1] if t else np.zeros(F, np.float32))
        out = s.process(order, ys[t][order])
        for r, f in enumerate(order):
            assert abs(out[r].loglik - ll[f]) <= TOL * max(1, abs(ll[f])), (t, f)
            assert abs(out[r].h_mean - hm[f]) <= TOL * max(1, abs(hm[f])), (t, f)
    for f in range(F):
        assert rel_err(s.particles(f), b.get_particles(f)) < TOL, f
        assert s.ctl(f).status == 0
    b.close()
    s.close()


def test_repeated_requests_run_in_order(pkg):
    """Three requests for one instrument in one call equal three calls."""
    F = 6
    ns, cfgs, prms = fleet(pkg, F, 2)
    ys = observations(F, 3, seed=2)
    a = pkg.Stream(F, 32 << 20, int(ns.max()), seed=SEED)
    c = pkg.Stream(F, 32 << 20, int(ns.max()), seed=SEED)
    for f in range(F):
        a.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED)
        c.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED)
    slots = np.array([0, 0, 0, 1, 2, 1], np.int32)
    yv = np.array([ys[0, 0], ys[1, 0], ys[2, 0], ys[0, 1], ys[0, 2], ys[1, 1]], np.float32)
    launches0 = a.kernel_launches
    out_a = a.process(slots, yv)
    assert a.kernel_launches - launches0 >= 3      # three rounds
    out_c = []
    for k in range(len(slots)):
        out_c.append(c.process(slots[k:k + 1], yv[k:k + 1])[0])
    for k in range(len(slots)):
        assert abs(out_a[k].loglik - out_c[k].loglik) <= TOL * max(1, abs(out_c[k].loglik)), k
    for f in range(3):
        assert rel_err(a.particles(f), c.particles(f)) < TOL
    a.close()
    c.close()


def test_budget_admission_and_eviction(pkg):
    cfg = pkg.default_config(4, 10.0)
    cfg2 = pkg.default_config(4, 10.0)
    cfg2.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    p = pkg.Params(0.97, 0.15, -1.0, 0.0)
    budget = 2 << 20
    s = pkg.Stream(64, budget, 2048, seed=1)
    assert s.bytes_budget == budget
    base = s.bytes_in_use
    slots = []
    while True:
        k = s.admit(2048, cfg2, p, seed=len(slots))
        if k < 0:
            assert k == -7     # SVPF_ERR_BUDGET
            break
        slots.append(k)
        assert s.bytes_in_use == base + len(slots) * 16 * 4096
        assert s.bytes_in_use <= budget
    assert len(slots) >= 4
    # a smaller instrument may still fit; a full-size one fits again after an eviction
    s.evict(slots[1])
    assert s.admit(2048, cfg2, p, seed=99) == slots[1]
    assert s.admit(2048, cfg2, p, seed=100) == -7
    s.evict(slots[2])
    s.evict(slots[3])                      # neighbours merge: room for one 2F + one 1F of 2048
    assert s.admit(2048, cfg2, p, seed=101) >= 0
    assert s.admit(2048, cfg, p, seed=102) >= 0
    out = s.process([slots[0], slots[0]], [0.01, -0.02])
    assert out[1].steps_used > 0
    with pytest.raises(RuntimeError):
        s.process([63], [0.0])             # never admitted
    s.close()


def test_device_round_matches_host_round(pkg):
    torch = pytest.importorskip("torch")
    F = 10
    ns, cfgs, prms = fleet(pkg, F, 4)
    ys = observations(F, 2, seed=5)
    a = pkg.Stream(F, 32 << 20, int(ns.max()), seed=SEED)
    c = pkg.Stream(F, 32 << 20, int(ns.max()), seed=SEED)
    for f in range(F):
        a.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED)
        c.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED)
    one = [f for f in range(F) if not cfgs[f].use_two_factor]
    two = [f for f in range(F) if cfgs[f].use_two_factor]
    order = np.array(one + two, np.int32)
    d_slots = torch.tensor(order, device="cuda")
    d_y = torch.tensor(ys[0][order], device="cuda")
    d_out = torch.zeros((F, 8), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    a.process_device(len(one), len(two), d_slots.data_ptr(), d_y.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    out_c = c.process(order, ys[0][order])
    ll_dev = d_out[:, 0].cpu().numpy()
    for r in range(F):
        assert abs(ll_dev[r] - out_c[r].loglik) <= TOL * max(1, abs(out_c[r].loglik)), r
    a.close()
    c.close()


def test_large_two_factor_filters_on_clusters(pkg):
    """Two-factor instruments with N >= 1024 run on 4-CTA clusters in the
    request loop; their ticks must equal the batch's one-CTA ticks."""
    ns = np.array([2048, 1024, 300, 1500, 2048, 512, 1024, 1100], np.int32)
    F = len(ns)
    cfgs, prms = [], []
    for f in range(F):
        c = pkg.default_config(4, 6.0)
        c.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2, nu=6.0, rho_fast=0.80, sigma_fast=0.30,
                        rho_slow=0.995, sigma_slow=0.05))
        cfgs.append(c)
        prms.append(pkg.Params(0.995, 0.05, -3.5, 0.0))
    ys = observations(F, 3, seed=9)
    b = pkg.Batch(ns, cfgs, prms)
    b.initialize(seed=SEED)
    s = pkg.Stream(F, 64 << 20, int(ns.max()), seed=SEED)
    for f in range(F):
        assert s.admit(int(ns[f]), cfgs[f], prms[f], seed=SEED) == f
    for t in range(3):
        ll, _, hm = b.step(ys[t], ys[t - 1] if t else np.zeros(F, np.float32))
        out = s.process(np.arange(F), ys[t])
        for f in range(F):
            assert abs(out[f].loglik - ll[f]) <= TOL * max(1, abs(ll[f])), (t, f, out[f].loglik, ll[f])
            assert abs(out[f].h_mean - hm[f]) <= TOL * max(1, abs(hm[f])), (t, f)
    for f in range(F):
        assert rel_err(s.particles(f), b.get_particles(f)) < TOL, f
    b.close()
    s.close()
