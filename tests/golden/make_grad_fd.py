"""FP64 reference gradients for the benchmark's differentiation check.

The benchmark's gradient workload differentiates the predictive
log-likelihood sum_t log p(y_t | y_1:t-1) of filters in the production
gradient configuration (full Newton, <= 8 Stein iterations over 3 stages,
SVLD, MIM, EKF guide, nu free) with respect to (mu, rho, sigma_z, nu), and
checks its first four filters over the first 200 ticks against central
differences at step 1e-4 max(1, |theta|).  This script computes, with the
FP64 oracle (oracle/svpf_oracle.cpp) on the same filters, paths and Philox
noise (seed 1, filter ids 0..3):

* the forward-mode (dual-number) gradient -- the exact derivative of the
  FP64 run, clamps contributing their one-sided derivative;
* central differences of the FP64 run at the benchmark's step;
* the forward-mode gradient at three thetas perturbed by 1e-7 relative (the
  run's sensitivity to FP32-sized input noise).

    python tests/golden/make_grad_fd.py          # about 2 minutes on 8 cores

Output: tests/golden/grad_fd_production.npz
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402

FILTERS, TICKS, N, SEED = 4, 200, 512, 1


def config():
    """The production gradient configuration (the engine's grad_config(8, 12.0);
    filling it needs no GPU) on the oracle's configuration record."""
    import __graft_entry__ as ge
    return oracle.config_from_dict(ge.load_package().grad_config(8, 12.0).to_dict())


def workload():
    """theta [4] and paths [4, 200] of the benchmark's gradient workload
    (bench.gradient_workload: rng seed 12 over 256 filters, paths seed 77)."""
    import bench
    F = 256
    rng = np.random.default_rng(12)
    th = np.stack([rng.uniform(-2.0, 0.0, F), rng.uniform(0.90, 0.995, F), rng.uniform(0.05, 0.4, F),
                   rng.uniform(4.0, 30.0, F)], 1).astype(np.float32)
    ys = bench.sv_paths(1000, th[:, 1].astype(np.float64), th[:, 2].astype(np.float64), th[:, 0].astype(np.float64),
                        th[:, 3].astype(np.float64), seed=77).T.copy()
    return th[:FILTERS], ys[:FILTERS, :TICKS]


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "grad_fd_production.npz")
    cfg = config()
    th, ys = workload()
    th64 = th.astype(np.float64)
    steps = 1e-4 * np.maximum(1.0, np.abs(th64))

    def run(f, theta):
        ll, g, _ = oracle.grad_run(cfg, N, theta, ys[f], seed=SEED, filter_id=f, objective=1)
        return ll.sum(), g

    jobs = {}
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        for f in range(FILTERS):
            jobs[(f, "base")] = ex.submit(run, f, th64[f])
            for q in range(4):
                for sgn in (1, -1):
                    t = th64[f].copy()
                    t[q] += sgn * steps[f, q]
                    jobs[(f, q, sgn)] = ex.submit(run, f, t)
            for trial in range(3):
                t = th64[f] * (1 + 1e-7 * np.random.default_rng(trial).standard_normal(4))
                jobs[(f, "sens", trial)] = ex.submit(run, f, t)
        res = {k: v.result() for k, v in jobs.items()}
    grad = np.array([res[(f, "base")][1] for f in range(FILTERS)])
    fd = np.array([[(res[(f, q, 1)][0] - res[(f, q, -1)][0]) / (2 * steps[f, q]) for q in range(4)]
                   for f in range(FILTERS)])
    sens = np.array([max(np.max(np.abs(res[(f, "sens", k)][1] - grad[f]) / np.maximum(np.abs(grad[f]), 1e-3))
                         for k in range(3)) for f in range(FILTERS)])
    np.savez_compressed(out, theta=th, ys=ys, n=np.int32(N), seed=np.int64(SEED), steps=steps, grad=grad, fd=fd,
                        sens=sens, loglik_sum=np.array([res[(f, "base")][0] for f in range(FILTERS)]))
    rel = np.abs(fd - grad) / np.maximum(np.abs(grad), 1e-3)
    print("forward-mode vs FD relative difference per filter x (mu, rho, sigma_z, nu):\n", rel)
    print("sensitivity:", sens)


if __name__ == "__main__":
    main()
