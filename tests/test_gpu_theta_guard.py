"""Parameters outside the model's domain never reach a kernel's loops.

theta comes from the caller (and, through the torch binding, from an
optimiser step that may diverge).  The host entry points reject it before any
launch; with device theta, each filter is checked on the device and a filter
outside the domain (non-finite component, nu <= 0, sigma_z <= 0, |rho| >= 1)
is left out with SVPF_ERR_INVALID_ARG, NaN outputs and a NaN gradient, while
every other filter's result is bit-identical to a run without it (its noise
is keyed by its own index).  The digamma these values used to reach is
bounded by construction (tests/test_math_host.py checks it on the CPU).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BAD = {1: (3, -math.inf), 3: (3, -1e30), 4: (2, math.nan)}   # filter: (theta column, value)


def _theta(F):
    rng = np.random.default_rng(4)
    return np.stack([rng.uniform(-2, 0, F), rng.uniform(0.9, 0.99, F), rng.uniform(0.1, 0.3, F),
                     rng.uniform(5, 20, F)], 1).astype(np.float32)


def _ys(F, T):
    rng = np.random.default_rng(5)
    return (0.4 * rng.standard_normal((F, T))).astype(np.float32)


def test_grad_engine_leaves_out_bad_theta(pkg):
    import torch

    F, N, T = 6, 128, 24
    good = _theta(F)
    bad = good.copy()
    for f, (q, v) in BAD.items():
        bad[f, q] = v
    ys = _ys(F, T)
    cfg = pkg.grad_config(4, 12.0)

    # host theta: refused before any launch
    g = pkg.Grad([N] * F, cfg, T_max=T, checkpoint_every=8)
    with pytest.raises(RuntimeError, match="error 1"):
        g.forward(bad, ys, seed=3)

    def run(theta):
        d_th = torch.from_numpy(theta).cuda()
        d_y = torch.from_numpy(ys).cuda()
        d_ll = torch.empty((F, T), dtype=torch.float32, device="cuda")
        d_g = torch.empty((F, 4), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.forward_device(d_th.data_ptr(), None, d_y.data_ptr(), T, 3, d_ll.data_ptr())
        st_fwd = g.status()
        g.backward_device(None, d_g.data_ptr())
        st = g.status()   # waits for the engine's own stream before the copies below
        return d_ll.cpu().numpy(), d_g.cpu().numpy(), st_fwd, st

    ll_ref, g_ref, st0, st1 = run(good)
    assert not st0.any() and not st1.any()
    ll_bad, g_bad, st_fwd, st = run(bad)
    for f in range(F):
        if f in BAD:
            assert st_fwd[f] == 1 and st[f] == 1, (f, st_fwd, st)
            assert np.isnan(ll_bad[f]).all() and np.isnan(g_bad[f]).all()
        else:
            assert st[f] == 0
            assert np.array_equal(ll_bad[f], ll_ref[f]), f
            assert np.array_equal(g_bad[f], g_ref[f]), (f, g_bad[f], g_ref[f])
    g.close()


def test_estimator_leaves_out_bad_theta(pkg):
    import torch

    F, N, T = 5, 64, 20
    good = _theta(F)
    good[:, 0] -= 2.0
    bad = good.copy()
    bad[1, 3] = -math.inf
    bad[3, 1] = 1.5
    ys = _ys(F, T)
    e = pkg.Estimator(F, N, 2, 0.15, T_max=T, checkpoint_every=8, truncate_every=0)
    with pytest.raises(RuntimeError, match="error 1"):
        e.forward(bad, ys, seed=2)

    def run(theta):
        d_th = torch.from_numpy(theta).cuda()
        d_y = torch.from_numpy(ys).cuda()
        d_ll = torch.empty((F, T), dtype=torch.float32, device="cuda")
        d_v = torch.empty((F, T), dtype=torch.float32, device="cuda")
        d_g = torch.empty((F, 4), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        e.forward_device(d_th.data_ptr(), d_y.data_ptr(), T, 2, None, d_ll.data_ptr(), d_v.data_ptr())
        e.backward_device(None, d_g.data_ptr())
        st = e.status()   # waits for the engine's own stream before the copies below
        return d_ll.cpu().numpy(), d_g.cpu().numpy(), st

    ll_ref, g_ref, st0 = run(good)
    assert not st0.any()
    ll_bad, g_bad, st = run(bad)
    for f in range(F):
        if f in (1, 3):
            assert st[f] == 1 and np.isnan(ll_bad[f]).all() and np.isnan(g_bad[f]).all()
        else:
            assert st[f] == 0
            assert np.array_equal(ll_bad[f], ll_ref[f]) and np.array_equal(g_bad[f], g_ref[f]), f
    e.close()


def test_autograd_path_reports_bad_theta(pkg):
    """Through torch.autograd: a diverged nu gives that filter NaN values and
    gradient and leaves the others as they were."""
    import torch
    import importlib

    ag = importlib.import_module("svpf_b200.autograd")
    F, N, T = 4, 128, 16
    th = torch.from_numpy(_theta(F)).cuda()
    y = torch.from_numpy(_ys(F, T)).cuda()
    eng = ag.GradEngine([N] * F, pkg.grad_config(4, 12.0), T_max=T, checkpoint_every=8)
    t1 = th.clone().requires_grad_(True)
    ag.svpf_loglik(t1, y, eng, seed=1).sum().backward()
    t2 = th.clone()
    t2[2, 3] = -1e30
    t2.requires_grad_(True)
    ll2 = ag.svpf_loglik(t2, y, eng, seed=1)
    ll2.sum().backward()
    assert torch.isnan(ll2[2]).all() and torch.isnan(t2.grad[2]).all()
    keep = [0, 1, 3]
    assert torch.equal(t1.grad[keep], t2.grad[keep])
    assert list(eng.status()) == [0, 0, 1, 0]
    eng.close()
