"""Golden fixtures of the reference's differentiable torch model.

Runs ``SVPFParamEstimator.forward`` of the reference
(py-torch/diff_svpf_torch.py:147-217) in FP64 on CPU, unmodified, and records
what its autograd returns: the predictive NLL, the per-tick predictive
log-likelihoods, the per-tick volatility estimates and d NLL / d(mu, rho,
sigma_z) (the model learns unconstrained parameters, :82-105; the gradients
are carried to the natural parameters by the chain rule of its transforms).
The model's Student-t constant is a float32 buffer (:75-80): it shifts every
log-likelihood by its float32 rounding and does not enter the gradients.

The model draws its noise with torch.randn (the initial particles, then N/2
antithetic normals per tick, :170, :184-185); the script records that
sequence from the same seed and stores it as the noise tape the engine and
the oracle replay.  matplotlib (imported by the reference module for its
plots) is not installed here and is replaced by an empty module.

    python tests/golden/make_estimator_golden.py [reference_dir [out_dir]]

Writes tests/golden/estimator_*.npz.
"""
from __future__ import annotations

import contextlib
import importlib.util
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, model kwargs, data kwargs of the reference's generate_sv_data, T,
#  truncate_every, burn_in, torch seed)
CASES = [
    # train() settings (:224-232) at its initial parameters, the __main__ data (:302-305)
    ("estimator_train_n64", dict(n_particles=64, n_stein_steps=2, stein_lr=0.15, nu=8.0, init_rho=0.85,
                                 init_sigma_z=0.10, init_mu=-4.5),
     dict(rho=0.95, sigma_z=0.20, mu=-3.0, nu=8.0, seed=42), 120, 50, 20, 1),
    # the same data at the true parameters
    ("estimator_true_n64", dict(n_particles=64, n_stein_steps=2, stein_lr=0.15, nu=8.0, init_rho=0.95,
                                init_sigma_z=0.20, init_mu=-3.0),
     dict(rho=0.95, sigma_z=0.20, mu=-3.0, nu=8.0, seed=42), 120, 50, 20, 2),
    # the class defaults (:62-70) with more particles and Stein steps, no truncation
    ("estimator_n256_s4", dict(n_particles=256, n_stein_steps=4, stein_lr=0.1, nu=5.0, init_rho=0.9,
                               init_sigma_z=0.15, init_mu=-3.5),
     dict(rho=0.97, sigma_z=0.15, mu=-3.5, nu=5.0, seed=7), 60, 0, 0, 3),
    # short truncation windows
    ("estimator_n128_trunc10", dict(n_particles=128, n_stein_steps=3, stein_lr=0.2, nu=12.0, init_rho=0.92,
                                    init_sigma_z=0.25, init_mu=-2.5),
     dict(rho=0.9, sigma_z=0.3, mu=-2.0, nu=12.0, seed=11), 45, 10, 5, 4),
]


def load_reference(ref_dir: str):
    for name in ("matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    path = os.path.join(ref_dir, "py-torch", "diff_svpf_torch.py")
    spec = importlib.util.spec_from_file_location("diff_svpf_torch", path)
    mod = importlib.util.module_from_spec(spec)
    with contextlib.redirect_stdout(open(os.devnull, "w")):
        spec.loader.exec_module(mod)
    return mod


@contextlib.contextmanager
def instrumented(torch, out: list):
    """Record every torch.logsumexp result (the model's log_lik_t + log N,
    :197), and hand the model its float32 torch.randn draws as float64: a
    0-dim double parameter does not promote a float32 vector, so without this
    the particles would stay float32 after .double()."""
    orig_lse, orig_randn = torch.logsumexp, torch.randn

    def lse(*a, **k):
        r = orig_lse(*a, **k)
        out.append(float(r.detach()))
        return r

    def randn(*a, **k):
        return orig_randn(*a, **k).double()

    torch.logsumexp, torch.randn = lse, randn
    try:
        yield
    finally:
        torch.logsumexp, torch.randn = orig_lse, orig_randn


def run_case(mod, torch, case):
    name, mk, dk, T, trunc, burn, seed = case
    y, h = mod.generate_sv_data(T, **dk)
    model = mod.SVPFParamEstimator(**mk).double()
    n = mk["n_particles"]
    torch.manual_seed(seed)
    tape_init = torch.randn(n).numpy().astype(np.float32)
    tape_ticks = np.stack([torch.randn(n // 2).numpy() for _ in range(T)]).astype(np.float32)
    torch.manual_seed(seed)
    yt = torch.tensor(y.astype(np.float64))
    lse = []
    with instrumented(torch, lse):
        nll, vols = model(yt, truncate_every=trunc, burn_in=burn)
    nll.backward()
    # replay check: the recorded draws are the ones the model used
    torch.manual_seed(seed)
    assert np.array_equal(torch.randn(n).numpy(), tape_init)
    s_rho = torch.sigmoid(model._rho_logit.detach())
    s_sig = torch.sigmoid(model._log_sigma.detach())
    g_mu = float(model._mu.grad)
    g_rho = float(model._rho_logit.grad / (0.499 * s_rho * (1 - s_rho)))
    g_sz = float(model._log_sigma.grad / s_sig)
    with torch.no_grad():
        theta = np.array([float(model.mu), float(model.rho), float(model.sigma_z), mk["nu"]], np.float64)
    ll = np.array(lse, np.float64) - math.log(n)
    assert ll.shape == (T,)
    assert vols.dtype == torch.float64
    return name, dict(y=y.astype(np.float32), tape_init=tape_init, tape_ticks=tape_ticks, theta=theta,
                      n=n, n_stein=mk["n_stein_steps"], stein_lr=mk["stein_lr"], truncate_every=trunc,
                      burn_in=burn, nll=float(nll), loglik=ll, vol=vols.detach().numpy().astype(np.float64),
                      grad=np.array([g_mu, g_rho, g_sz], np.float64),
                      student_t_const=float(model.student_t_const))


def main():
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    import oracle
    ref = sys.argv[1] if len(sys.argv) > 1 else oracle.reference_dir()
    out = sys.argv[2] if len(sys.argv) > 2 else HERE
    mod = load_reference(ref)
    import torch
    torch.set_num_threads(1)
    for case in CASES:
        name, d = run_case(mod, torch, case)
        np.savez_compressed(os.path.join(out, name + ".npz"), **d)
        print(name, "nll", d["nll"], "grad", d["grad"])


if __name__ == "__main__":
    main()
