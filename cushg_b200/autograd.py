"""torch.autograd binding of the adjoint march, for gradient checks.

``SHGPower.apply(waist, focus, temp, poling, params)`` returns the SH output power of a
plain run as a 0-d tensor; its backward multiplies the incoming gradient by dJ/dwaist,
dJ/dfocus, dJ/dtemp and dJ/dpoling from ``shg_grad``.  Both directions run through the C
ABI of libshg_b200.so; torch only carries the scalars.
"""
from __future__ import annotations

import numpy as np
import torch

from . import shg
from .params import ShgParams


def _with(p: ShgParams, waist, focus, temp) -> ShgParams:
    return p.replace(waist=float(waist), focus=float(focus), temp=float(temp), t_peltier=float(temp))


class SHGPower(torch.autograd.Function):
    """J(waist, focus, temp, poling) = SH output power [W] of the plain run ``params``."""

    @staticmethod
    def forward(ctx, waist, focus, temp, poling, params: ShgParams):
        p = _with(params, waist.item(), focus.item(), temp.item())
        pol = poling.detach().cpu().numpy().astype(np.float64)
        ctx.save_for_backward(waist, focus, temp, poling)
        ctx.params = params
        return torch.tensor(shg.sh_power(p, pol), dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        waist, focus, temp, poling = ctx.saved_tensors
        p = _with(ctx.params, waist.item(), focus.item(), temp.item())
        g = shg.grad(p, poling.detach().cpu().numpy().astype(np.float64))
        go = grad_out.to(torch.float64)
        return (go * g["d_waist"], go * g["d_focus"], go * g["d_temp"],
                go * torch.as_tensor(g["d_poling"], dtype=torch.float64), None)


def sh_power(waist, focus, temp, poling, params: ShgParams):
    return SHGPower.apply(waist, focus, temp, poling, params)
