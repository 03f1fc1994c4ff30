"""torch.autograd.Function over the gradient engine (svpf_grad_* C ABI).

    engine = GradEngine(ns, cfg, T_max)              # bound to torch's current CUDA stream
    ll = svpf_loglik(theta, y, engine, seed=0)       # theta [F,4] (mu, rho, sigma_z, nu), y [F,T]
    ll.sum().backward()                              # theta.grad: d loss / d theta

The forward runs the whole filter (initialisation included) on the engine's
stream and returns the per-tick log-likelihoods [F,T]; the backward feeds the
incoming gradient [F,T] as the tick weights of the adjoint and returns
d loss / d theta [F,4].  The noise is the engine's counter-based stream keyed
by `seed`, so forward and backward see the same draws.
"""
from __future__ import annotations

import torch

from .svpf import Config, Grad


def torch_stream_handle(device=None) -> int:
    """Handle of torch's current CUDA stream for an engine to launch on.  The
    legacy default stream has handle 0, which the engines read as "make a
    private stream"; cudaStreamLegacy (handle 1) names it explicitly."""
    return torch.cuda.current_stream(device).cuda_stream or 1


class GradEngine(Grad):
    """A Grad bound to torch's current CUDA stream, so its launches are
    ordered with the surrounding torch work."""

    def __init__(self, ns, configs, T_max: int, checkpoint_every: int = 64):
        super().__init__(ns, configs, T_max, checkpoint_every, stream=torch_stream_handle())


class SVPFLogLik(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, y, engine: GradEngine, seed: int = 0, gamma=None):
        if not theta.is_cuda or not y.is_cuda:
            raise ValueError("theta and y must be CUDA tensors (the engine has no CPU path)")
        F, T = y.shape
        if theta.shape != (F, 4) or engine.F != F:
            raise ValueError("theta must be [F, 4] and y [F, T] with F the engine's filter count")
        th = theta.detach().to(torch.float32).contiguous()
        yy = y.detach().to(torch.float32).contiguous()
        gm = None if gamma is None else gamma.detach().to(torch.float32).contiguous()
        ll = torch.empty((F, T), dtype=torch.float32, device=y.device)
        engine.forward_device(th.data_ptr(), None if gm is None else gm.data_ptr(), yy.data_ptr(), T,
                              int(seed), ll.data_ptr())
        # the engine reads theta / y / gamma again in the backward
        ctx.keep = (th, yy, gm)
        ctx.engine = engine
        ctx.forward_id = engine.forward_id
        ctx.theta_dtype = theta.dtype
        return ll

    @staticmethod
    def backward(ctx, grad_ll):
        engine = ctx.engine
        if engine.forward_id != ctx.forward_id:
            raise RuntimeError("the gradient engine ran another forward since this graph was built")
        w = grad_ll.detach().to(torch.float32).contiguous()
        g = torch.empty((engine.F, 4), dtype=torch.float64, device=w.device)
        engine.backward_device(w.data_ptr(), g.data_ptr())
        return g.to(ctx.theta_dtype), None, None, None, None


def svpf_loglik(theta, y, engine: GradEngine, seed: int = 0, gamma=None):
    """Per-tick log-likelihoods [F,T] of the filters, differentiable in theta."""
    return SVPFLogLik.apply(theta, y, engine, seed, gamma)


__all__ = ["GradEngine", "SVPFLogLik", "svpf_loglik", "Config"]
