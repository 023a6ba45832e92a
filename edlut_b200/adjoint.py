"""Differentiable membrane traces of batched LIF networks.

:class:`TraceModel` holds a batch of LIF networks (explicit connectivity, e.g.
:func:`edlut_b200.configs.adjoint_networks`) on the GPU; calling it with a
parameter tensor ``[networks, 4]`` (g_leak, e_leak, tau_exc, tau_inh) and a
weight tensor (every synapse, networks in order, each in its spec order) runs the
unchanged time-driven forward and returns the membrane traces of the observed
neurons, ``[networks, steps, m]``, as a tensor that autograd differentiates
through :class:`LIFTraces` -- a ``torch.autograd.Function`` whose backward is the
hand-written adjoint kernel (``eb_sweep_adjoint``: checkpoints every K steps,
one recomputation per segment, exact reset jump at every spike).

>>> model = TraceModel(specs, n_steps=5000, observed=obs, checkpoint_every=100)
>>> params = model.initial_params().requires_grad_()
>>> weights = model.initial_weights().requires_grad_()
>>> loss = ((model(params, weights) - target) ** 2).mean()
>>> loss.backward()
"""
from __future__ import annotations

import numpy as np
import torch

from .configs import ADJOINT_PARAMS
from .sweep import Sweep


class TraceModel:
    def __init__(self, specs, n_steps: int, observed, integrator: str = "RK2", dt: float = 1e-4,
                 delay: float = 1e-3, checkpoint_every: int = 100, device: int = 0,
                 max_rate_hz: float = 500.0, block: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("TraceModel needs a CUDA device (there is no CPU path)")
        self.device = torch.device("cuda", device)
        self.sweep = Sweep.from_specs(specs, n_steps_max=n_steps, integrator=integrator, dt=dt, delay=delay,
                                      device=device, max_rate_hz=max_rate_hz)
        if block:
            self.sweep.configure(block=block, steps_per_launch=checkpoint_every)
        obs = np.asarray(observed, np.int32)
        if obs.ndim == 1:
            obs = np.broadcast_to(obs, (len(specs), len(obs)))
        self.sweep.set_observed(obs)
        self.sweep.set_checkpoints(checkpoint_every)
        self.n_steps = n_steps
        self.n_networks = len(specs)
        self.n_obs = obs.shape[1]
        self.specs = specs
        self.n_weights = self.sweep.info()["synapses"]

    def initial_params(self, dtype=torch.float64) -> torch.Tensor:
        return torch.tensor([[s["params"][k] for k in ADJOINT_PARAMS] for s in self.specs], dtype=dtype)

    def initial_weights(self) -> torch.Tensor:
        return torch.from_numpy(np.concatenate([s["w"] for s in self.specs]).astype(np.float32)).to(self.device)

    def __call__(self, params: torch.Tensor, weights: torch.Tensor) -> torch.Tensor:
        return LIFTraces.apply(params, weights, self)


class LIFTraces(torch.autograd.Function):
    """Observed membrane traces of a :class:`TraceModel` as a function of its
    parameters and weights.  Forward: the method's own time stepping; backward: the
    discrete adjoint of that forward (eb_sweep_adjoint)."""

    @staticmethod
    def forward(ctx, params, weights, model):
        sw = model.sweep
        p = params.detach().to("cpu", torch.float64).numpy()
        for i in range(model.n_networks):
            sw.set_params(i, {k: float(p[i, j]) for j, k in enumerate(ADJOINT_PARAMS)})
        w = weights.detach().to(model.device, torch.float32).contiguous()
        if w.numel() != model.n_weights:
            raise ValueError("expected %d weights, got %d" % (model.n_weights, w.numel()))
        torch.cuda.current_stream(model.device).synchronize()
        sw.set_weights(w)
        sw.reset()
        sw.run(model.n_steps)
        out = torch.empty(model.n_networks, model.n_steps, model.n_obs, device=model.device, dtype=torch.float32)
        sw.trace(model.n_steps, out=out)
        ctx.model = model
        ctx.p_meta = (params.dtype, params.device)
        ctx.w_meta = (weights.dtype, weights.device)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        model = ctx.model
        g = grad_out.to(model.device, torch.float32).contiguous()
        gw = torch.empty(model.n_weights, device=model.device, dtype=torch.float32)
        torch.cuda.current_stream(model.device).synchronize()
        gp, _ = model.sweep.adjoint(g, grad_w=gw)
        return (torch.from_numpy(gp).to(ctx.p_meta[1], ctx.p_meta[0]), gw.to(ctx.w_meta[1], ctx.w_meta[0]), None)
