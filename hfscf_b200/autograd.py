"""torch.autograd.Function over the engine's forward/backward pair.

forward:  E2(R) = sum_ij D_ij (2 J[D] - K[D])_ij at coordinates R (hfgpu_energy_forward);
backward: dE2/dR at fixed D from the adjoint derivative-ERI kernel
          (hfgpu_grad2e_backward), scaled by the incoming gradient.
The density is treated as a constant, as in the two-electron term of the SCF
gradient (src/gradient/hfscf_grad_rhf.cpp:121-141).
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine as eng


class TwoElectronEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, D, engine, precision=eng.FP64):
        engine.set_geometry(coords.detach().cpu().numpy().astype(np.float64))
        Dn = D.detach().cpu().numpy().astype(np.float64)
        e2 = engine.energy2e(Dn, precision)
        ctx.engine, ctx.D, ctx.precision = engine, Dn, precision
        return torch.tensor(e2, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        g = ctx.engine.grad2e(ctx.D, scale=float(grad_out), precision=ctx.precision)
        return torch.from_numpy(g), None, None, None


def two_electron_energy(coords, D, engine, precision=eng.FP64):
    return TwoElectronEnergy.apply(coords, D, engine, precision)
