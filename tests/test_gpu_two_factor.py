"""Two-factor tick (h = mu + h_fast + h_slow) of the CUDA engine through the C
ABI against the FP64 oracle, with state re-sync and a shared noise tape:
edge particle counts and cluster shapes, initialisation, the batch kernel
against the single-filter kernel, and batches mixing one- and two-factor
filters.  Tolerance: 1e-4 relative (floor 1 on the denominator)."""
import numpy as np
import pytest

import cases
import tape
from test_oracle import TOL, TWO_FACTOR_SCALARS, rel_err

pytestmark = pytest.mark.gpu

PARAMS = (0.99, 0.05, -3.5, 0.0)
PATH = ("2f", -3.5, 0.90, 0.15, 0.99, 0.05, 7.0)


def make_engine(pkg, n, cfg_over, cluster=0, n_stein=8, nu=7.0):
    f = pkg.SVPF(n, n_stein, nu)
    f.configure(**cfg_over)
    f.params = pkg.Params(*PARAMS)
    if cluster:
        f.set_cluster_size(cluster)
    f._initialized = True
    return f


def oracle_twin(oracle_mod, f):
    o = oracle_mod.OracleFilter(f.n_particles, oracle_mod.config_from_dict(f.config.to_dict()),
                                oracle_mod.OracleParams(*PARAMS))
    ctl, _, _, _, lw = f.get_state()
    h, hp, v = f.get_state_2f()
    o.ctl = oracle_mod.ctl_from_dict({k: getattr(ctl, k) for k, _ in ctl._fields_ if not k.startswith("smooth_")})
    o.h, o.h_prev, o.v, o.log_w = (a.astype(np.float64) for a in (h, hp, v, lw))
    return o


def init_tape(f, n, seed):
    z = tape.init_normals(seed, n, 3)
    f.set_noise_tape(z, np.ones((1, n), np.float32))


def check_tick(f, o, nrm, uni, y, yp, t):
    f.set_noise_tape(nrm, uni)
    rc, out = f.step_raw(y, yp)
    assert rc == 0, (t, rc)
    oo = o.step(y, yp, nrm, uni)
    h, hp, v = f.get_state_2f()
    ctl = f.get_state()[0]
    assert rel_err(h, o.h) < TOL, (t, rel_err(h, o.h))
    assert rel_err(hp, o.h_prev) < TOL, t
    assert rel_err(v, o.v, floor=1e-3) < 10 * TOL, (t, rel_err(v, o.v, floor=1e-3))
    assert abs(out.loglik - oo.loglik) < TOL * max(1, abs(oo.loglik)), (t, out.loglik, oo.loglik)
    assert abs(out.vol - oo.vol) < TOL * max(1, abs(oo.vol)), (t, out.vol, oo.vol)
    assert abs(out.h_mean - oo.h_mean) < TOL * max(1, abs(oo.h_mean)), (t, out.h_mean, oo.h_mean)
    assert out.steps_used == oo.steps_used
    for k in TWO_FACTOR_SCALARS:
        a, b = getattr(ctl, k), getattr(o.ctl, k)
        assert abs(a - b) <= TOL * max(1.0, abs(b)), (t, k, a, b)


@pytest.mark.parametrize("n,cluster", [(1, 1), (2, 1), (31, 1), (33, 2), (255, 4), (257, 8), (512, 0),
                                       (1000, 16), (2048, 0), (4096, 16), (4096, 8)])
def test_two_factor_matches_oracle_sizes(pkg, oracle_mod, n, cluster):
    """Edge sizes and cluster shapes, the reference's two-factor test knobs,
    3 ticks each from a re-synced state."""
    cfg = dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2)
    f = make_engine(pkg, n, cfg, cluster, n_stein=4)
    init_tape(f, n, 11)
    f.initialize(*PARAMS, seed=5)
    _, ys = tape.sv2_path(4, *PATH[1:6], seed=n, nu_obs=PATH[6])
    yp = 0.0
    slots = 2 + 2 * 2 * 4
    for t in range(3):
        o = oracle_twin(oracle_mod, f)
        nrm, uni = tape.tape(99, t, n, slots, 2)
        check_tick(f, o, nrm, uni, float(ys[t]), yp, t)
        yp = float(ys[t])
    f.close()


VARIANTS = {
    "reference_test": cases.TWO_FACTOR_TEST,
    "plain": dict(use_two_factor=1, use_svld=0, use_mim=0, use_guide=0, use_annealing=0,
                  use_exact_gradient=0, stein_repulsive_sign=1),
    "blend_guide": dict(use_two_factor=1, use_guide=1, use_guide_preserving=0, guide_strength=0.3,
                        n_anneal_steps=3, temperature=0.6),
    "no_guide_anneal4": dict(use_two_factor=1, use_guide=0, n_anneal_steps=4, use_mim=1,
                             mim_jump_prob=0.5, mim_jump_scale=4.0),
}


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_two_factor_variants_over_ticks(pkg, oracle_mod, name):
    """Each knob family over 10 ticks from its own initialisation (the guide's
    factor means come from the previous tick), state re-synced every tick."""
    n = 384
    f = make_engine(pkg, n, VARIANTS[name], n_stein=4, nu=9.0)
    init_tape(f, n, 3)
    f.initialize(*PARAMS, seed=1)
    _, ys = tape.sv2_path(11, *PATH[1:6], seed=17, nu_obs=PATH[6])
    yp = 0.0
    c = f.config
    slots = 2 + 2 * (c.n_anneal_steps if c.use_annealing else 1) * c.n_stein_steps
    for t in range(10):
        o = oracle_twin(oracle_mod, f)
        nrm, uni = tape.tape(5, t, n, slots, 2)
        check_tick(f, o, nrm, uni, float(ys[t]), yp, t)
        yp = float(ys[t])
    f.close()


def test_two_factor_initialize_matches_oracle(pkg, oracle_mod):
    """svpf_initialize with two factors: stationary draws of both factors from
    tape slots 1 and 2, EKF guide state reset."""
    n = 700
    f = make_engine(pkg, n, cases.TWO_FACTOR_TEST)
    z = tape.init_normals(8, n, 3)
    f.set_noise_tape(z, np.ones((1, n), np.float32))
    f.initialize(*PARAMS, seed=2)
    o = oracle_mod.OracleFilter(n, oracle_mod.config_from_dict(f.config.to_dict()), oracle_mod.OracleParams(*PARAMS))
    o.initialize(z)
    h, hp, v = f.get_state_2f()
    assert rel_err(h, o.h) < TOL and rel_err(hp, o.h_prev) < TOL
    assert np.all(v == 0)
    ctl = f.get_state()[0]
    for k in ("guide_mean_fast", "guide_mean_slow", "guide_var_fast", "guide_var_slow", "guide_2f_initialized"):
        assert abs(getattr(ctl, k) - getattr(o.ctl, k)) <= TOL * max(1.0, abs(getattr(o.ctl, k))), k
    f.close()


def test_two_factor_tape_too_short(pkg):
    n = 128
    f = make_engine(pkg, n, cases.TWO_FACTOR_TEST)
    init_tape(f, n, 1)
    f.initialize(*PARAMS, seed=1)
    f.set_noise_tape(np.zeros((2, n), np.float32), np.full((1, n), 0.5, np.float32))
    rc, _ = f.step_raw(0.01, 0.0)
    assert rc == 4   # SVPF_ERR_TAPE_SHORT
    f.set_noise_tape(None)
    rc, _ = f.step_raw(0.01, 0.0)
    assert rc == 0
    f.close()


def _batch_vs_singles(pkg, ns, cfgs, nrm_slots=2 + 2 * 2 * 4):
    params = pkg.Params(*PARAMS)
    b = pkg.Batch(ns, cfgs, params)
    n_max = max(ns)
    init = tape.init_normals(21, n_max, 3)
    b.set_noise_tape(init, np.ones((1, n_max), np.float32))
    b.initialize(seed=3)
    nrm, uni = tape.tape(8, 0, n_max, max(nrm_slots, 12), 2)
    ys = np.linspace(-0.03, 0.04, len(ns)).astype(np.float32)
    b.set_noise_tape(nrm, uni)
    ll, vol, hm = b.step(ys, np.zeros(len(ns), np.float32))
    for i, n in enumerate(ns):
        f = pkg.SVPF(n, cfgs[i].n_stein_steps, cfgs[i].nu)
        f.configure(**cfgs[i].to_dict())
        f.params = params
        f._initialized = True
        f.set_noise_tape(np.ascontiguousarray(init[:, :n]), np.ones((1, n), np.float32))
        f.initialize(*PARAMS, seed=3)
        f.set_noise_tape(np.ascontiguousarray(nrm[:, :n]), np.ascontiguousarray(uni[:, :n]))
        rc, out = f.step_raw(float(ys[i]), 0.0)
        assert rc == 0
        hb = b.get_particles(i)
        hs = f.get_state_2f()[0] if cfgs[i].use_two_factor else f.get_particles()
        assert hb.shape == hs.shape
        assert rel_err(hb, hs) < TOL, (i, n, rel_err(hb, hs))
        assert abs(ll[i] - out.loglik) < TOL * max(1, abs(out.loglik)), (i, ll[i], out.loglik)
        assert abs(hm[i] - out.h_mean) < TOL * max(1, abs(out.h_mean))
        f.close()
    ctl = b.ctl()
    assert all(c.status == 0 for c in ctl)
    b.close()


def test_two_factor_batch_matches_single_filters(pkg):
    ns = [256, 300, 512, 1024, 64, 2048]
    cfg = pkg.default_config(4, 7.0)
    cfg.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    _batch_vs_singles(pkg, ns, [cfg] * len(ns))


def test_mixed_batch_runs_both_kernels(pkg):
    """One batch of single-factor and two-factor filters: two persistent
    launches per tick, each filter equal to its single-filter tick."""
    ns = [512, 256, 1024, 300, 128, 2048]
    c1 = pkg.default_config(4, 7.0)
    c1.update(**cases.PRODUCTION)
    c1.update(stein_max_steps=4, stein_min_steps=4)
    c2 = pkg.default_config(4, 7.0)
    c2.update(**dict(cases.TWO_FACTOR_TEST, n_anneal_steps=2))
    cfgs = [c1 if i % 2 == 0 else c2 for i in range(len(ns))]
    _batch_vs_singles(pkg, ns, cfgs)
    b = pkg.Batch(ns, cfgs, pkg.Params(*PARAMS))
    b.initialize(seed=1)
    before = b.kernel_launches
    b.step(np.full(len(ns), 0.01, np.float32), np.zeros(len(ns), np.float32))
    assert b.kernel_launches - before == 2
    b.close()
