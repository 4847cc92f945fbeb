"""torch.autograd.Function over the CUDA kernels.

``thole_dipole(charges, polarizabilities, tholes, dipoles, kernel, system)``
returns (energy, forces) as torch tensors and differentiates both with respect
to the per-particle charges, isotropic polarizabilities, Thole factors and
molecular-frame dipoles.  The backward is the hand-written adjoint of
tdp_adjoint (one adjoint solve of the same symmetric (alpha^-1 - T) system for
Mutual polarization, pair damping recomputed).  Positions, axis frames and
covalent maps are fixed inputs.

The kernel object keeps the state of its last forward evaluation, so each
forward must be followed by its backward before the same kernel evaluates
again (the usual single forward/backward per step of a training loop).
"""
from __future__ import annotations

import numpy as np
import torch

from .kernel import CudaCalcTholeDipoleForceKernel
from .systems import TholeSystem


class TholeDipoleFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, charges, polarizabilities, tholes, dipoles, kernel: CudaCalcTholeDipoleForceKernel,
                system: TholeSystem):
        s = system.copy(charges=charges.detach().cpu().double().numpy().copy(),
                        polarizabilities=polarizabilities.detach().cpu().double().numpy().copy(),
                        tholes=tholes.detach().cpu().double().numpy().copy(),
                        dipoles=dipoles.detach().cpu().double().numpy().reshape(-1, 3).copy())
        kernel.copyParametersToContext(s)
        energy, forces = kernel.execute(s.positions)
        ctx.kernel = kernel
        ctx.device = charges.device
        return (torch.tensor(energy, dtype=torch.float64, device=charges.device),
                torch.tensor(forces, dtype=torch.float64, device=charges.device))

    @staticmethod
    def backward(ctx, grad_energy, grad_forces):
        gE = 0.0 if grad_energy is None else float(grad_energy)
        gF = None if grad_forces is None else grad_forces.detach().cpu().double().numpy()
        g = ctx.kernel.adjoint(gF, gE)
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=ctx.device)
        return t(g[:, 0]), t(g[:, 1]), t(g[:, 2]), t(g[:, 3:6]), None, None


def thole_dipole(charges, polarizabilities, tholes, dipoles, kernel, system):
    return TholeDipoleFunction.apply(charges, polarizabilities, tholes, dipoles, kernel, system)
