"""The CUDA forward and adjoint of the reference's differentiable torch model
(svpf_estimator_* through the C ABI, and the torch module mirroring
SVPFParamEstimator) against golden fixtures of that model run unmodified by
torch autograd in FP64, and against the FP64 oracle restatement at other
sizes.

Tolerances (FP32 engine against FP64): log-likelihoods and volatility
estimates 1e-4 relative (floor 1), gradients 2e-4 relative (floor 1e-3), or
four times the FP64 oracle's own sensitivity where that is larger (the
largest relative change of its output when theta moves by 1e-7 relative,
FP32-sized input noise).  The reference's train() configuration is
ill-conditioned in this sense (gradient sensitivity 2e-3); the others are
not (<= 3e-5)."""
import glob
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "estimator_*.npz")))
LL_TOL = 1e-4
G_TOL = 2e-4


def load(path):
    d = np.load(path)
    T = d["y"].shape[0]
    b = int(d["burn_in"])
    w = np.zeros(T)
    w[b:] = -1.0 / (T - b)
    return d, w


def sensitivity(n, S, lr, theta, ys, ti, tt, trunc, w):
    """Largest relative change of the oracle's (loglik, vol, grad) for 1e-7
    relative moves of theta."""
    ll0, v0, g0 = oracle.estimator_run(n, S, lr, theta, ys, ti, tt, trunc, w)
    sl = sv = sg = 0.0
    for trial in range(3):
        th = np.asarray(theta, np.float64) * (1 + 1e-7 * np.random.default_rng(trial).standard_normal(4))
        ll, v, g = oracle.estimator_run(n, S, lr, th, ys, ti, tt, trunc, w)
        sl = max(sl, float(np.max(np.abs(ll - ll0) / np.maximum(1.0, np.abs(ll0)))))
        sv = max(sv, float(np.max(np.abs(v - v0) / v0)))
        sg = max(sg, float(np.max(np.abs(g - g0) / np.maximum(np.abs(g0), 1e-3))))
    return sl, sv, sg


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_engine_matches_reference_torch_autograd(pkg, path):
    d, w = load(path)
    n, S, lr, trunc = int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]), int(d["truncate_every"])
    T = d["y"].shape[0]
    sl, sv, sg = sensitivity(n, S, lr, d["theta"], d["y"], d["tape_init"], d["tape_ticks"], trunc, w)
    e = pkg.Estimator(1, n, S, lr, T_max=T, checkpoint_every=16, truncate_every=trunc)
    tape = pkg.Estimator.make_tape(d["tape_init"], d["tape_ticks"])[None]
    ll, vol, ls = e.forward(d["theta"][None], d["y"][None], tape=tape)
    g = e.backward(w[None].astype(np.float32))[0]
    e.close()
    lt = max(LL_TOL, 4 * sl)
    assert np.max(np.abs(ll[0] - d["loglik"]) / np.maximum(1.0, np.abs(d["loglik"]))) < lt
    assert np.max(np.abs(vol[0] - d["vol"]) / np.abs(d["vol"])) < max(LL_TOL, 4 * sv)
    assert abs(ls[0] - ll[0].astype(np.float64).sum()) < 1e-3
    err = np.abs(g[:3] - d["grad"]) / np.maximum(np.abs(d["grad"]), 1e-3)
    assert np.all(err < max(G_TOL, 4 * sg)), (g[:3], d["grad"], err, sg)


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_torch_module_matches_reference_module(pkg, path):
    """The drop-in module: same constructor, transforms and loss; gradients
    reach the unconstrained parameters through torch."""
    import torch
    from importlib import import_module
    est = import_module(pkg.__name__ + ".estimator")
    d, w = load(path)
    kw = _module_kwargs(d)
    model = est.SVPFParamEstimator(**kw).double().cuda()
    y = torch.tensor(d["y"].astype(np.float64), device="cuda")
    tape = torch.tensor(pkg.Estimator.make_tape(d["tape_init"], d["tape_ticks"]), device="cuda")
    nll, vols = model(y, truncate_every=int(d["truncate_every"]), burn_in=int(d["burn_in"]), noise_tape=tape)
    nll.backward()
    s_rho = torch.sigmoid(model._rho_logit.detach())
    s_sig = torch.sigmoid(model._log_sigma.detach())
    g = np.array([float(model._mu.grad), float(model._rho_logit.grad / (0.499 * s_rho * (1 - s_rho))),
                  float(model._log_sigma.grad / s_sig)])
    sl, _, sg = sensitivity(int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]), d["theta"], d["y"],
                            d["tape_init"], d["tape_ticks"], int(d["truncate_every"]), w)
    assert abs(float(nll.detach()) - float(d["nll"])) < max(LL_TOL, 4 * sl) * max(1.0, abs(float(d["nll"])))
    assert vols.shape == (d["y"].shape[0],)
    err = np.abs(g - d["grad"]) / np.maximum(np.abs(d["grad"]), 1e-3)
    assert np.all(err < max(G_TOL, 4 * sg)), (g, d["grad"], err)


def _module_kwargs(d):
    """Constructor arguments reproducing the fixture's natural parameters."""
    mu, rho, sz, nu = (float(v) for v in d["theta"])
    # invert the module's transforms (rho = 0.5 + 0.499 s, sigma = softplus + 0.001)
    s = (rho - 0.5) / 0.499
    return dict(n_particles=int(d["n"]), n_stein_steps=int(d["n_stein"]), stein_lr=float(d["stein_lr"]), nu=nu,
                init_rho=s, init_sigma_z=float(np.expm1(sz - 0.001)), init_mu=mu)


def _random_case(n, T, seed):
    rng = np.random.default_rng(seed)
    ti = rng.standard_normal(n).astype(np.float32)
    tt = rng.standard_normal((T, n // 2)).astype(np.float32)
    h = -3.0
    ys = []
    for _ in range(T):
        h = -3.0 + 0.95 * (h + 3.0) + 0.2 * rng.standard_normal()
        ys.append(np.exp(h / 2) * rng.standard_t(8))
    return np.array(ys, np.float32), ti, tt


@pytest.mark.parametrize("n,S,trunc", [(2, 1, 0), (4, 0, 0), (30, 3, 0), (256, 2, 7), (1000, 1, 0), (2048, 2, 5)])
def test_engine_matches_oracle_sizes(pkg, n, S, trunc):
    T, F, lr = 20, 3, 0.12
    rng = np.random.default_rng(n)
    thetas = np.stack([rng.uniform(-4, -2, F), rng.uniform(0.85, 0.98, F), rng.uniform(0.1, 0.3, F),
                       rng.uniform(5, 20, F)], 1)
    cases = [_random_case(n, T, 100 * n + f) for f in range(F)]
    w = rng.uniform(-1, 1, (F, T))
    e = pkg.Estimator(F, n, S, lr, T_max=T, checkpoint_every=6, truncate_every=trunc)
    tape = np.stack([pkg.Estimator.make_tape(c[1], c[2]) for c in cases])
    ll, vol, _ = e.forward(thetas, np.stack([c[0] for c in cases]), tape=tape)
    g = e.backward(w.astype(np.float32))
    e.close()
    for f in range(F):
        ys, ti, tt = cases[f]
        oll, ovol, og = oracle.estimator_run(n, S, lr, thetas[f], ys, ti, tt, trunc, w[f])
        sl, sv, sg = sensitivity(n, S, lr, thetas[f], ys, ti, tt, trunc, w[f])
        assert np.max(np.abs(ll[f] - oll) / np.maximum(1.0, np.abs(oll))) < max(LL_TOL, 4 * sl), f
        assert np.max(np.abs(vol[f] - ovol) / ovol) < max(LL_TOL, 4 * sv), (f, sv)
        err = np.abs(g[f] - og) / np.maximum(np.abs(og), 1e-3)
        assert np.all(err < max(G_TOL, 4 * sg)), (n, f, g[f], og, err, sg)


def test_checkpoint_interval_does_not_change_the_result(pkg):
    n, S, T = 128, 2, 30
    ys, ti, tt = _random_case(n, T, 5)
    th = np.array([[-3.0, 0.95, 0.2, 8.0]])
    tape = pkg.Estimator.make_tape(ti, tt)[None]
    out = []
    for k in (1, 4, 64):
        e = pkg.Estimator(1, n, S, 0.15, T_max=T, checkpoint_every=k, truncate_every=10)
        ll, _, _ = e.forward(th, ys[None], tape=tape)
        out.append((ll, e.backward()))
        e.close()
    for ll, g in out[1:]:
        assert np.array_equal(ll, out[0][0]) and np.array_equal(g, out[0][1])


def test_counter_based_noise_is_repeatable(pkg):
    n, T, F = 64, 40, 4
    ys = np.stack([_random_case(n, T, f)[0] for f in range(F)])
    th = np.tile([-3.0, 0.95, 0.2, 8.0], (F, 1))
    e = pkg.Estimator(F, n, 2, 0.15, T_max=T)
    a = e.forward(th, ys, seed=7)[0]
    ga = e.backward()
    b = e.forward(th, ys, seed=7)[0]
    gb = e.backward()
    c = e.forward(th, ys, seed=8)[0]
    e.close()
    assert np.array_equal(a, b) and np.array_equal(ga, gb)
    assert not np.array_equal(a, c)
    # same theta and y on every path, different keys per path: different draws
    assert not np.array_equal(a[0], a[1])
    assert np.all(np.isfinite(ga))


def test_invalid_sizes_are_rejected(pkg):
    with pytest.raises(RuntimeError):
        pkg.Estimator(1, 63, 2, 0.1, T_max=10)
    with pytest.raises(RuntimeError):
        pkg.Estimator(1, 64, 2, 0.1, T_max=0)
