"""The reference's differentiable SVPF estimator on the CUDA engine.

``SVPFParamEstimator`` keeps the interface of the reference's torch module
(py-torch/diff_svpf_torch.py:49-217): the same constructor arguments,
learnable unconstrained parameters (_rho_logit, _log_sigma, _mu) with the
same transforms (rho = 0.5 + 0.499 sigmoid, sigma_z = softplus + 0.001,
:88-105), ``get_params`` and ``forward(y, truncate_every, burn_in) ->
(neg_log_lik, vol_estimates)``.  The particle filter and its gradient run in
the svpf_estimator_* kernels (forward and hand-written adjoint) instead of
being traced by torch autograd; the transforms stay in torch, so gradients
reach the unconstrained parameters as before.

    model = SVPFParamEstimator(n_particles=64, n_stein_steps=2, stein_lr=0.15, nu=8.0).cuda()
    nll, vols = model(y_cuda, truncate_every=50, burn_in=20)
    nll.backward()

The noise is the engine's counter-based stream keyed by a seed drawn from
torch's default generator (so torch.manual_seed makes runs repeatable), or a
given tape (``noise_tape``: the n initial normals followed by n/2 per tick, the
order in which the reference's forward calls torch.randn).
"""
from __future__ import annotations

import math

import torch
import torch.nn as nn
import torch.nn.functional as F

from .autograd import torch_stream_handle
from .svpf import Estimator


class EstimatorRun(torch.autograd.Function):
    """Per-tick predictive log-likelihoods [P,T] and volatility estimates
    [P,T] of P paths; differentiable in theta [P,4]."""

    @staticmethod
    def forward(ctx, theta, y, engine: Estimator, seed: int, tape):
        if not theta.is_cuda or not y.is_cuda:
            raise ValueError("theta and y must be CUDA tensors (the engine has no CPU path)")
        P, T = y.shape
        th = theta.detach().to(torch.float32).contiguous()
        yy = y.detach().to(torch.float32).contiguous()
        tp = None if tape is None else tape.detach().to(device=y.device, dtype=torch.float32).contiguous()
        ll = torch.empty((P, T), dtype=torch.float32, device=y.device)
        vol = torch.empty((P, T), dtype=torch.float32, device=y.device)
        engine.forward_device(th.data_ptr(), yy.data_ptr(), T, int(seed), None if tp is None else tp.data_ptr(),
                              ll.data_ptr(), vol.data_ptr())
        ctx.keep = (th, yy, tp)     # the backward reads them again
        ctx.engine = engine
        ctx.forward_id = engine.forward_id
        ctx.theta_dtype = theta.dtype
        ctx.mark_non_differentiable(vol)
        return ll, vol

    @staticmethod
    def backward(ctx, grad_ll, grad_vol):
        engine = ctx.engine
        if engine.forward_id != ctx.forward_id:
            raise RuntimeError("the estimator engine ran another forward since this graph was built")
        w = grad_ll.detach().to(torch.float32).contiguous()
        g = torch.empty((engine.F, 4), dtype=torch.float64, device=w.device)
        engine.backward_device(w.data_ptr(), g.data_ptr())
        return g.to(ctx.theta_dtype), None, None, None, None


class SVPFParamEstimator(nn.Module):
    """Learns (rho, sigma_z, mu) with nu fixed, loss = predictive NLL."""

    def __init__(self, n_particles: int = 64, n_stein_steps: int = 2, stein_lr: float = 0.1, nu: float = 8.0,
                 init_rho: float = 0.9, init_sigma_z: float = 0.15, init_mu: float = -3.5,
                 checkpoint_every: int = 64):
        super().__init__()
        if n_particles < 2 or n_particles % 2:
            raise ValueError("n_particles must be even (antithetic pairs)")
        self.n_particles = n_particles
        self.n_stein_steps = n_stein_steps
        self.stein_lr = stein_lr
        self.nu = nu
        self.checkpoint_every = checkpoint_every
        self.register_buffer("student_t_const", torch.tensor(
            math.lgamma((nu + 1) / 2) - math.lgamma(nu / 2) - 0.5 * math.log(nu * math.pi)))
        self._rho_logit = nn.Parameter(torch.tensor(self._logit(init_rho)))
        self._log_sigma = nn.Parameter(torch.tensor(math.log(init_sigma_z)))
        self._mu = nn.Parameter(torch.tensor(init_mu))
        self._engines = {}

    @staticmethod
    def _logit(x):
        return math.log(x / (1 - x + 1e-8) + 1e-8)

    @property
    def rho(self):
        return 0.5 + 0.499 * torch.sigmoid(self._rho_logit)

    @property
    def sigma_z(self):
        return F.softplus(self._log_sigma) + 0.001

    @property
    def mu(self):
        return self._mu

    def get_params(self):
        return {"rho": self.rho.item(), "sigma_z": self.sigma_z.item(), "mu": self.mu.item(), "nu": self.nu}

    def _engine(self, paths: int, T: int, truncate_every: int, device) -> Estimator:
        stream = torch_stream_handle(device)
        key = (paths, truncate_every, device.index, stream)
        e = self._engines.get(key)
        if e is None or e.T_max < T:
            if e is not None:
                e.close()
            with torch.cuda.device(device):
                e = Estimator(paths, self.n_particles, self.n_stein_steps, self.stein_lr, T_max=T,
                              checkpoint_every=self.checkpoint_every, truncate_every=max(int(truncate_every), 0),
                              stream=stream)
            self._engines[key] = e
        return e

    def forward(self, y, truncate_every: int = 50, burn_in: int = 20, noise_tape=None, seed=None):
        """y [T] (or [P,T]: P paths sharing the parameters).  Returns
        (neg_log_lik = -mean of the per-tick predictive log-likelihoods after
        the burn-in, vol_estimates [T] or [P,T])."""
        single = y.dim() == 1
        yy = y[None] if single else y
        P, T = yy.shape
        if T <= burn_in:
            raise ValueError("need more ticks than the burn-in")
        nu = torch.tensor(float(self.nu), dtype=self._mu.dtype, device=self._mu.device)
        theta = torch.stack([self.mu, self.rho, self.sigma_z, nu]).to(yy.device)
        theta = theta[None].expand(P, 4)
        if seed is None:
            seed = int(torch.randint(0, 2 ** 62, (1,)).item())
        tape = None
        if noise_tape is not None:
            tape = torch.as_tensor(noise_tape).reshape(P, -1)
        engine = self._engine(P, T, truncate_every, yy.device)
        ll, vol = EstimatorRun.apply(theta, yy, engine, seed, tape)
        nll = -ll[:, burn_in:].mean()
        return nll.to(self._mu.dtype), (vol[0] if single else vol)


__all__ = ["SVPFParamEstimator", "EstimatorRun", "Estimator"]
