"""The FP64 restatement of the reference's differentiable torch model
(SVPFParamEstimator, py-torch/diff_svpf_torch.py:147-217) against golden
fixtures of that model run unmodified in FP64 by torch autograd
(tests/golden/make_estimator_golden.py): same data, same noise (the model's
torch.randn draws as a tape), same truncation and burn-in.

Tolerances: gradients 1e-9 relative; per-tick log-likelihoods 1e-7 absolute
(the model keeps its Student-t constant as a float32 buffer, :75-80, so each
of its log-likelihoods carries that constant's float32 rounding, 2.4e-8);
volatility estimates 1e-10 relative.  The whole tangent, d/d nu included (nu
is fixed in the torch model), is also checked against central differences of
the oracle itself with the model's two cuts held as its autograd holds them:
the bandwidth frozen at the run's values, no truncation."""
import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "estimator_*.npz")))


def load(path):
    d = np.load(path)
    T = d["y"].shape[0]
    b = int(d["burn_in"])
    w = np.zeros(T)
    w[b:] = -1.0 / (T - b)     # NLL = -mean(loglik[burn_in:])  (:214-215)
    return d, w


def run(d, w, theta=None):
    return oracle.estimator_run(int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]),
                                d["theta"] if theta is None else theta, d["y"], d["tape_init"], d["tape_ticks"],
                                int(d["truncate_every"]), w)


def test_fixtures_present():
    assert len(FIXTURES) == 4


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_torch_autograd(path):
    d, w = load(path)
    ll, vol, g = run(d, w)
    assert np.max(np.abs(ll - d["loglik"])) < 1e-7
    assert np.max(np.abs(vol - d["vol"]) / np.abs(d["vol"])) < 1e-10
    nll = float(np.dot(w, ll))
    assert abs(nll - float(d["nll"])) < 1e-7 * max(1.0, abs(float(d["nll"])))
    rel = np.abs(g[:3] - d["grad"]) / np.maximum(np.abs(d["grad"]), 1e-6)
    assert np.all(rel < 1e-9), (g[:3], d["grad"], rel)


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_tangents_match_central_differences(path):
    d, w = load(path)
    args = (int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]))
    data = (d["y"], d["tape_init"], d["tape_ticks"], 0, w)
    _, _, g, bw = oracle.estimator_run(*args, d["theta"], *data, return_bw=True)
    for k in range(4):
        h = 1e-7 * max(1.0, abs(float(d["theta"][k])))   # clamp kinks lie within 1e-5
        tp, tm = d["theta"].copy(), d["theta"].copy()
        tp[k] += h
        tm[k] -= h
        fd = (np.dot(w, oracle.estimator_run(*args, tp, *data, bw_fixed=bw)[0]) -
              np.dot(w, oracle.estimator_run(*args, tm, *data, bw_fixed=bw)[0])) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1e-2, abs(g[k])), (k, fd, g[k])


def test_truncation_cuts_the_particle_path():
    """With truncation every tick, the gradient of a late tick's likelihood
    only sees theta through that tick and the one before it."""
    d, _ = load(FIXTURES[0])
    T = d["y"].shape[0]
    w = np.zeros(T)
    w[-1] = 1.0
    one = oracle.estimator_run(int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]), d["theta"], d["y"],
                               d["tape_init"], d["tape_ticks"], 1, w)[2]
    full = oracle.estimator_run(int(d["n"]), int(d["n_stein"]), float(d["stein_lr"]), d["theta"], d["y"],
                                d["tape_init"], d["tape_ticks"], 0, w)[2]
    assert np.all(np.isfinite(one)) and not np.allclose(one, full)


def test_odd_particle_count_is_rejected():
    d, w = load(FIXTURES[0])
    with pytest.raises(RuntimeError):
        oracle.estimator_run(63, 2, 0.1, d["theta"], d["y"][:3], d["tape_init"][:63],
                             np.zeros((3, 31), np.float32), 0, None)
