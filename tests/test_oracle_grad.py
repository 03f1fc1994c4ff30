"""The FP64 gradient oracle (forward-mode AD of a whole run) pinned two ways:
its primal equals the main oracle's run on the same Philox noise, and its
derivatives equal central finite differences of its own FP64 primal.  The
comparison step matters: the run is piecewise smooth in theta (clamps of the
score at +-10, of the Newton curvature and Hessian, of the bandwidth), so a
central difference is only exact when no clamp boundary lies within the step;
with N=64 particles over 12 ticks that holds at steps of 1e-7, and for the
vanilla transport already at 1e-5."""
import numpy as np
import pytest

import tape

THETA = np.array([-1.0, 0.97, 0.15, 12.0])


def grad_cfg(oracle_mod, **kw):
    cfg = oracle_mod.default_config(8, 12.0)
    base = dict(use_asymmetric_rho=0, use_rejuvenation=0, use_adaptive_beta=0, use_newton=1, use_full_newton=1,
                stein_min_steps=8, stein_max_steps=8, n_anneal_steps=3, use_exact_gradient=1)
    base.update(kw)
    for k, v in base.items():
        setattr(cfg, k, v)
    return cfg


CFGS = {
    "full_newton": {},
    "vanilla": dict(use_newton=0, use_full_newton=0),
    "plain_predict_no_guide": dict(use_mim=0, use_guide=0),
    "blend_guide_approx_grad": dict(use_guide_preserving=0, use_exact_gradient=0),
    "no_svld_no_annealing": dict(use_svld=0, use_annealing=0),
}


def test_unsupported_configurations_rejected(oracle_mod):
    assert oracle_mod.grad_supported(grad_cfg(oracle_mod))
    for bad in (dict(use_asymmetric_rho=1), dict(use_rejuvenation=1), dict(use_newton=1, use_full_newton=0),
                dict(use_two_factor=1), dict(use_adaptive_mu=1), dict(use_student_t_state=1), dict(use_guided=1),
                dict(use_adaptive_beta=1), dict(stein_min_steps=0)):
        assert not oracle_mod.grad_supported(grad_cfg(oracle_mod, **bad)), bad


@pytest.mark.parametrize("name", sorted(CFGS))
def test_primal_matches_main_oracle(oracle_mod, name):
    cfg = grad_cfg(oracle_mod, **CFGS[name])
    _, ys = tape.sv_path(12, -1.0, 0.97, 0.15, seed=3)
    ll, _, _ = oracle_mod.grad_run(cfg, 64, THETA, ys, seed=7)
    ref = oracle_mod.run_loglik(cfg, 64, THETA, ys, seed=7)
    # the main oracle stores the bandwidth in FP32 between stages; nothing else differs
    assert np.max(np.abs(ll - ref) / np.maximum(1, np.abs(ref))) < 1e-6


@pytest.mark.parametrize("objective", [0, 1], ids=["tick_loglik", "predictive"])
@pytest.mark.parametrize("name", sorted(CFGS))
def test_gradient_matches_central_differences(oracle_mod, name, objective):
    cfg = grad_cfg(oracle_mod, **CFGS[name])
    _, ys = tape.sv_path(12, -1.0, 0.97, 0.15, seed=3)
    _, g, _ = oracle_mod.grad_run(cfg, 64, THETA, ys, seed=7, objective=objective)
    for k in range(4):
        h = 1e-7 * max(1.0, abs(THETA[k]))
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (oracle_mod.grad_run(cfg, 64, tp, ys, seed=7, objective=objective)[0].sum() -
              oracle_mod.grad_run(cfg, 64, tm, ys, seed=7, objective=objective)[0].sum()) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(abs(g[k]), 1e-2), (name, k, fd, g[k])


def test_weights_are_linear(oracle_mod):
    cfg = grad_cfg(oracle_mod)
    _, ys = tape.sv_path(10, -1.0, 0.97, 0.15, seed=5)
    rng = np.random.default_rng(0)
    w1, w2 = rng.standard_normal(10), rng.standard_normal(10)
    g1 = oracle_mod.grad_run(cfg, 32, THETA, ys, w=w1, seed=2)[1]
    g2 = oracle_mod.grad_run(cfg, 32, THETA, ys, w=w2, seed=2)[1]
    g12 = oracle_mod.grad_run(cfg, 32, THETA, ys, w=w1 + w2, seed=2)[1]
    assert np.allclose(g1 + g2, g12, rtol=1e-12, atol=1e-12)
