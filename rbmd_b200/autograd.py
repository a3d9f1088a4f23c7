"""torch.autograd binding of the RBL + RBE force and its adjoint.

A thin layer over the C ABI for force-field fitting and for tests: the forward
pass sets the engine's parameters and positions and evaluates the force with
the engine's fixed k-samples and batch epoch; the backward pass is
rbx_engine_force_vjp.  The engine itself does not use torch.  One forward and
its backward must run before the engine is used for anything else.
"""
from __future__ import annotations

import numpy as np
import torch

from . import rbx


class RBLRBEForce(torch.autograd.Function):
    """F(eps[ntypes], sigma[ntypes], charge[n], alpha, pos[n, 3]) -> [n, 3] (FP64, CPU)."""

    @staticmethod
    def forward(ctx, eps, sigma, charge, alpha, pos, engine: rbx.Engine, epoch: int):
        engine.set_lj_params(sigma.detach().cpu().numpy(), eps.detach().cpu().numpy())
        engine.set_charges(charge.detach().cpu().numpy())
        engine.set_alpha(float(alpha))
        engine.set_positions(pos.detach().cpu().numpy())
        engine.compute_forces(epoch)
        ctx.engine = engine
        return torch.from_numpy(engine.get_state()["force"])

    @staticmethod
    def backward(ctx, grad_f):
        out = ctx.engine.force_vjp(grad_f.detach().cpu().numpy().astype(np.float64))
        t = torch.from_numpy
        return (t(out["eps"]), t(out["sigma"]), t(out["charge"]),
                torch.tensor(out["alpha"], dtype=torch.float64), t(out["pos"]), None, None)


def force(engine, eps, sigma, charge, alpha, pos, epoch=0):
    """Differentiable force of `engine` at the given parameters and positions."""
    return RBLRBEForce.apply(eps, sigma, charge, alpha, pos, engine, epoch)
