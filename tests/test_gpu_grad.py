"""The CUDA adjoint (svpf_grad_* through the C ABI) against the FP64
forward-mode gradient oracle on the same Philox noise, checkpoint
invariance, tick weights, central finite differences of the FP64 oracle at
the step the benchmark quotes (1e-4), and the torch.autograd.Function.

Tolerances: per-tick log-likelihoods 1e-5 relative; gradients 2e-4 relative
(floor 1e-3) against the FP64 oracle, or four times the oracle's own
sensitivity where that is larger: the FP64 gradient's relative change when
theta moves by 1e-7 relative (FP32-sized input noise).  Most configurations
have a sensitivity ~1e-5 and the measured agreement is ~1e-5; without SVLD
noise and annealing the run is ill-conditioned (sensitivity 2e-3 .. 1e-2)."""
import os

import numpy as np
import pytest

import tape

pytestmark = pytest.mark.gpu

LL_TOL = 1e-5
G_TOL = 2e-4


def oracle_cfg(oracle_mod, cfg):
    return oracle_mod.config_from_dict(cfg.to_dict())


def thetas_for(F, seed=0):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(-2.0, 0.0, F), rng.uniform(0.90, 0.99, F), rng.uniform(0.08, 0.3, F),
                     rng.uniform(5.0, 25.0, F)], axis=1).astype(np.float32)


def paths_for(thetas, T, seed0=10):
    return np.stack([tape.sv_path(T, float(th[0]), float(th[1]), float(th[2]), seed=seed0 + f)[1]
                     for f, th in enumerate(thetas)])


def check_against_oracle(pkg, oracle_mod, cfg, ns, T, k=64, seed=7, w=None, gamma=None, objective=0, trunc=0):
    F = len(ns)
    th = thetas_for(F)
    ys = paths_for(th, T)
    g = pkg.Grad(ns, cfg, T_max=T, checkpoint_every=k)
    g.set_objective(objective)
    g.truncate_every = trunc
    ll, ls = g.forward(th, ys, gamma=gamma, seed=seed)
    grad = g.backward(w)
    g.close()
    for f in range(F):
        run = lambda t: oracle_mod.grad_run(oracle_cfg(oracle_mod, cfg), ns[f], t, ys[f],  # noqa: E731
                                            gamma=0.0 if gamma is None else float(gamma[f]),
                                            w=None if w is None else w[f].astype(np.float64), seed=seed,
                                            filter_id=f, objective=objective, truncate_every=trunc)
        base = th[f].astype(np.float64)
        oll, og, _ = run(base)
        assert np.max(np.abs(ll[f] - oll) / np.maximum(1, np.abs(oll))) < LL_TOL, f
        assert abs(ls[f] - oll.sum()) < LL_TOL * max(1, abs(oll.sum())) * T
        sens = 0.0
        for trial in range(3):
            pert = base * (1 + 1e-7 * np.random.default_rng(trial).standard_normal(4))
            sens = max(sens, np.max(np.abs(run(pert)[1] - og) / np.maximum(np.abs(og), 1e-3)))
        err = np.abs(grad[f] - og) / np.maximum(np.abs(og), 1e-3)
        assert np.all(err < max(G_TOL, 4 * sens)), (f, ns[f], grad[f], og, err, sens)
    return grad


CFGS = {
    "full_newton": dict(),
    "vanilla": dict(full_newton=False),
    "plain_predict_no_guide": dict(full_newton=False, use_mim=0, use_guide=0),
    "blend_guide_approx_grad": dict(use_guide_preserving=0, use_exact_gradient=0),
    "no_svld_no_annealing": dict(use_svld=0, use_annealing=0),
}


@pytest.mark.parametrize("name", sorted(CFGS))
def test_adjoint_matches_oracle_configs(pkg, oracle_mod, name):
    kw = dict(CFGS[name])
    full = kw.pop("full_newton", True)
    cfg = pkg.grad_config(6, 12.0, full_newton=full, **kw)
    check_against_oracle(pkg, oracle_mod, cfg, [64, 128, 200], T=12)


@pytest.mark.parametrize("ns", [[1, 2, 31], [257, 33], [512], [1000]])
def test_adjoint_matches_oracle_sizes(pkg, oracle_mod, ns):
    cfg = pkg.grad_config(4, 12.0)
    check_against_oracle(pkg, oracle_mod, cfg, ns, T=6)


@pytest.mark.parametrize("name", ["full_newton", "plain_predict_no_guide"])
def test_predictive_objective_matches_oracle(pkg, oracle_mod, name):
    """The predictive objective log p(y_t | y_1:t-1) at the predicted particles."""
    kw = dict(CFGS[name])
    full = kw.pop("full_newton", True)
    cfg = pkg.grad_config(6, 12.0, full_newton=full, **kw)
    check_against_oracle(pkg, oracle_mod, cfg, [64, 128, 200], T=12, objective=1)


@pytest.mark.parametrize("objective,trunc,k", [(0, 8, 64), (1, 5, 7)])
def test_truncated_adjoint_matches_oracle(pkg, oracle_mod, objective, trunc, k):
    """Truncated backpropagation every `trunc` ticks (cuts aligned and not
    aligned with the checkpoints) against the FP64 forward-mode oracle with
    the same cuts (the carried state's tangents zeroed at each cut)."""
    cfg = pkg.grad_config(6, 12.0)
    check_against_oracle(pkg, oracle_mod, cfg, [64, 128, 200], T=24, k=k, objective=objective, trunc=trunc)


def test_exploding_gradient_is_reported_and_truncation_bounds_it(pkg):
    """A filter of the benchmark's workload with narrow state noise (sigma_z
    0.056): its exact gradient grows exponentially with the run's length (the
    FP64 forward-mode oracle gives 5.8e5 for d/dmu after 200 ticks, 2.2e7 after
    250) and overflows FP32 within 1000 ticks -- reported as
    SVPF_ERR_NONFINITE; truncated backpropagation every 64 ticks keeps it
    finite."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    F = 256
    rng = np.random.default_rng(12)
    th = np.stack([rng.uniform(-2.0, 0.0, F), rng.uniform(0.90, 0.995, F), rng.uniform(0.05, 0.4, F),
                   rng.uniform(4.0, 30.0, F)], 1).astype(np.float32)
    ys = bench.sv_paths(1000, th[:, 1].astype(np.float64), th[:, 2].astype(np.float64), th[:, 0].astype(np.float64),
                        th[:, 3].astype(np.float64), seed=77).T.copy()
    f = 222
    g = pkg.Grad([512], pkg.grad_config(8, 12.0), T_max=1000, checkpoint_every=64)
    g.set_objective(g.PREDICTIVE)
    g.forward(th[f:f + 1], ys[f:f + 1], seed=1)
    assert not np.isfinite(g.backward()).all()
    assert g.status()[0] == 5   # SVPF_ERR_NONFINITE
    g.truncate_every = 64
    gt = g.backward()
    assert np.isfinite(gt).all() and np.abs(gt).max() < 1e5, gt
    assert g.status()[0] == 0
    g.close()


def test_leverage_and_weights(pkg, oracle_mod):
    cfg = pkg.grad_config(4, 9.0)
    rng = np.random.default_rng(3)
    w = rng.standard_normal((2, 10)).astype(np.float32)
    check_against_oracle(pkg, oracle_mod, cfg, [96, 160], T=10, w=w, gamma=np.array([-0.3, 0.2], np.float32))


def test_checkpoint_interval_does_not_change_the_gradient(pkg):
    """Recomputation from checkpoints is exact: every interval gives the
    same bits."""
    cfg = pkg.grad_config(4, 12.0)
    ns = [128, 64, 300]
    th = thetas_for(3, 1)
    ys = paths_for(th, 40)
    out = []
    for k in (1, 3, 16, 64):
        g = pkg.Grad(ns, cfg, T_max=40, checkpoint_every=k)
        ll, _ = g.forward(th, ys, seed=11)
        out.append((ll, g.backward()))
        g.close()
    for ll, gr in out[1:]:
        assert np.array_equal(ll, out[0][0])
        assert np.array_equal(gr, out[0][1])


@pytest.mark.parametrize("objective", [0, 1])
def test_record_modes_give_the_same_bits(pkg, objective):
    """The forward keeping every tick's record (no recomputation), recording a
    whole checkpoint segment in one forward, and re-recording each tick before
    its adjoint are the same computation."""
    cfg = pkg.grad_config(8 if objective else 4, 12.0)
    ns = [128, 300, 64, 512]
    th = thetas_for(4, 6)
    ys = paths_for(th, 20)
    out = []
    for run, seg in ((True, False), (False, True), (False, False)):
        g = pkg.Grad(ns, cfg, T_max=20, checkpoint_every=7)
        g.set_objective(objective)
        g.run_records = run
        g.segment_records = seg
        assert g.run_records == run and g.segment_records == seg
        ll, _ = g.forward(th, ys, seed=2)
        out.append((ll, g.backward()))
        g.close()
    for ll, gr in out[1:]:
        assert np.array_equal(out[0][0], ll)
        assert np.array_equal(out[0][1], gr)


def test_weights_select_ticks(pkg):
    """A one-hot weight on tick t gives the gradient of loglik_t alone, and
    weights combine linearly."""
    cfg = pkg.grad_config(4, 12.0)
    ns = [128, 128]
    th = thetas_for(2, 2)
    T = 16
    ys = paths_for(th, T)
    g = pkg.Grad(ns, cfg, T_max=T, checkpoint_every=5)
    g.forward(th, ys, seed=3)
    full = g.backward()
    parts = np.zeros_like(full)
    for t0 in range(0, T, 4):
        w = np.zeros((2, T), np.float32)
        w[:, t0:t0 + 4] = 1.0
        parts += g.backward(w)
    g.close()
    assert np.allclose(parts, full, rtol=1e-5, atol=1e-5)


def test_adjoint_matches_fp64_central_differences(pkg, oracle_mod):
    """Central finite differences of the FP64 oracle at step 1e-4 (vanilla
    transport; 64 particles, 10 ticks) against the CUDA adjoint: 1e-3."""
    cfg = pkg.grad_config(4, 12.0, full_newton=False)
    th = thetas_for(1, 4)
    ys = paths_for(th, 10)
    g = pkg.Grad([64], cfg, T_max=10)
    g.forward(th, ys, seed=5)
    grad = g.backward()[0]
    g.close()
    oc = oracle_cfg(oracle_mod, cfg)
    base = th[0].astype(np.float64)
    for k in range(4):
        h = 1e-4
        tp, tm = base.copy(), base.copy()
        tp[k] += h
        tm[k] -= h
        fd = (oracle_mod.grad_run(oc, 64, tp, ys[0], seed=5)[0].sum() -
              oracle_mod.grad_run(oc, 64, tm, ys[0], seed=5)[0].sum()) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-3 * max(abs(grad[k]), 1e-2), (k, fd, grad[k])


def test_production_adjoint_matches_fp64_fd_and_forward_mode(pkg):
    """The benchmark's differentiation check settled in FP64: its first four
    filters (production gradient configuration: full Newton, 8 Stein
    iterations over 3 stages, SVLD, MIM, EKF guide, nu free; N = 512, 200
    ticks, the predictive objective) with the FP64 oracle's forward-mode
    gradient and its central differences at step 1e-4 max(1, |theta|)
    recorded by tests/golden/make_grad_fd.py.

    * CUDA adjoint vs the FP64 forward-mode gradient: 2e-4 relative (floor
      1e-3) or four times the run's sensitivity to a 1e-7 change of theta.
    * CUDA adjoint vs the FP64 central differences: 1e-3 wherever the FP64
      differences agree with the FP64 forward-mode gradient to 1e-3
      (kink-free: no clamp switches inside the step).  The recorded kinks:
      filter 1's differences are biased by 2.8e-3 (mu), 3.4e-2 (rho) and
      4.2e-2 (sigma_z) against the exact FP64 derivative, which the adjoint
      matches instead."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "grad_fd_production.npz"))
    th, ys, n, seed = z["theta"], z["ys"], int(z["n"]), int(z["seed"])
    F, T = ys.shape
    g = pkg.Grad([n] * F, pkg.grad_config(8, 12.0), T_max=T, checkpoint_every=64)
    g.set_objective(g.PREDICTIVE)
    _, ls = g.forward(th, ys, seed=seed)
    grad = g.backward()
    g.close()
    assert np.allclose(ls, z["loglik_sum"], rtol=1e-5, atol=1e-3), (ls, z["loglik_sum"])
    fm, fd = z["grad"], z["fd"]
    rel_fm = np.abs(grad - fm) / np.maximum(np.abs(fm), 1e-3)
    assert np.all(rel_fm < np.maximum(G_TOL, 4 * z["sens"][:, None])), rel_fm
    kink_free = np.abs(fd - fm) / np.maximum(np.abs(fm), 1e-3) < 1e-3
    assert kink_free.sum() >= 12 and not kink_free[1, 1:3].any()
    rel_fd = np.abs(grad - fd) / np.maximum(np.abs(fd), 1e-3)
    assert np.all(rel_fd[kink_free] < 1e-3), rel_fd


def test_unsupported_configuration_is_rejected(pkg):
    cfg = pkg.grad_config(4, 12.0)
    assert pkg.Grad.supported(cfg)
    bad = pkg.default_config(4, 12.0)   # asymmetric rho and rejuvenation are on by default
    assert not pkg.Grad.supported(bad)
    with pytest.raises(RuntimeError):
        pkg.Grad([64], bad, T_max=4)


def test_torch_autograd_function(pkg):
    torch = pytest.importorskip("torch")
    from importlib import import_module
    ag = import_module(pkg.__name__ + ".autograd")
    cfg = pkg.grad_config(4, 12.0)
    ns = [96, 128, 64]
    th = thetas_for(3, 5)
    T = 12
    ys = paths_for(th, T)
    eng = ag.GradEngine(ns, cfg, T_max=T, checkpoint_every=4)
    theta = torch.tensor(th, device="cuda", requires_grad=True)
    y = torch.tensor(ys, device="cuda")
    ll = ag.svpf_loglik(theta, y, eng, seed=9)
    w = torch.linspace(0.5, 1.5, T, device="cuda")
    loss = (ll * w).sum()
    loss.backward()
    ref = pkg.Grad(ns, cfg, T_max=T, checkpoint_every=4)
    ll2, _ = ref.forward(th, ys, seed=9)
    g2 = ref.backward(np.broadcast_to(w.cpu().numpy(), (3, T)).copy())
    ref.close()
    assert np.array_equal(ll.detach().cpu().numpy(), ll2)
    assert np.allclose(theta.grad.cpu().numpy(), g2, rtol=1e-6, atol=1e-6)
    eng.close()
