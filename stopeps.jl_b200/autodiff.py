"""lognorm as a differentiable function of the site tensors.

``LognormFunction`` is a ``torch.autograd.Function`` (the Python counterpart
of a ChainRulesCore ``rrule``): its forward uploads the site tensors and runs
the row method's ``lognorm`` (``src/contraction/boundary_mps.jl:180-186``) on
the device, keeping the derivative that the same reverse pass produces
(``sps_lognorm_gradient``); its backward scales that derivative by the
incoming cotangent.  The site tensors are host (or device) float64 torch
tensors in x + y*Lx order; the device computation goes through the engine's
C ABI in both directions.  The reference has no derivatives.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import lognorm_gradient


class LognormFunction(torch.autograd.Function):
    """lnZ(sites) with its reverse-mode derivative; ``apply(engine, leg_dims,
    is_pepo, contraction, checkpoint_rows, beta, log_amplitude, *sites)``."""

    @staticmethod
    def forward(ctx, engine, leg_dims, is_pepo, contraction, checkpoint_rows, beta, log_amplitude, *sites):
        host = [s.detach().to("cpu", torch.float64).numpy() for s in sites]
        state = engine.upload_state(host, leg_dims, is_pepo, beta=beta, log_amplitude=log_amplitude)
        value, grads = lognorm_gradient(state, contraction, checkpoint_rows=checkpoint_rows)
        ctx.save_for_backward(*[torch.from_numpy(np.ascontiguousarray(g)).to(s.device)
                                for g, s in zip(grads, sites)])
        return torch.tensor(value, dtype=torch.float64, device=sites[0].device)

    @staticmethod
    def backward(ctx, grad_output):
        grads = ctx.saved_tensors
        return (None,) * 7 + tuple(grad_output * g for g in grads)


def lognorm_differentiable(engine, sites, leg_dims, contraction, is_pepo=True, beta=0.0, log_amplitude=0.0,
                           checkpoint_rows=False):
    """lnZ of the state with site tensors ``sites`` (torch float64, x + y*Lx
    order, legs (w, n, p, a, e, s) with per-leg parity multiplicities
    ``leg_dims``), differentiable with respect to every site tensor."""
    if len(sites) != engine.Lx * engine.Ly:
        raise ValueError("one site tensor per lattice site")
    for s in sites:
        if s.dtype != torch.float64:
            raise TypeError("site tensors are float64")
    return LognormFunction.apply(engine, leg_dims, is_pepo, contraction, checkpoint_rows, beta, log_amplitude,
                                 *sites)
