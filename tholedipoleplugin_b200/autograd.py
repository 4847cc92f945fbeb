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


class ClusterGradients:
    """Gradients over a batch of isolated clusters (the cluster workload of the
    batched kernels, tdp_batch_*): one CudaCalcTholeDipoleForceKernel per
    cluster evaluates it and runs its adjoint, so a loss over every cluster's
    energy and forces differentiates with respect to every particle's charge,
    polarizability, Thole factor and molecular dipole.  Parameters are
    concatenated in cluster order (cluster c owns particles offsets[c]:offsets[c+1])."""

    def __init__(self, clusters, precision="double"):
        from .systems import concat_clusters

        self.clusters = [c.copy() for c in clusters]
        self.system, self.offsets = concat_clusters(self.clusters)
        self.kernels = [CudaCalcTholeDipoleForceKernel(c, precision=precision) for c in self.clusters]

    def close(self):
        for k in self.kernels:
            k.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def slices(self):
        return [slice(int(self.offsets[c]), int(self.offsets[c + 1])) for c in range(len(self.clusters))]


class ClusterBatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, charges, polarizabilities, tholes, dipoles, batch: ClusterGradients):
        q = charges.detach().cpu().double().numpy()
        a = polarizabilities.detach().cpu().double().numpy()
        t = tholes.detach().cpu().double().numpy()
        d = dipoles.detach().cpu().double().numpy().reshape(-1, 3)
        energies = np.zeros(len(batch.clusters))
        forces = np.zeros((batch.system.n, 3))
        for c, (sl, k, cl) in enumerate(zip(batch.slices(), batch.kernels, batch.clusters)):
            s = cl.copy(charges=q[sl].copy(), polarizabilities=a[sl].copy(), tholes=t[sl].copy(),
                        dipoles=d[sl].copy())
            k.copyParametersToContext(s)
            energies[c], forces[sl] = k.execute(s.positions)
        ctx.batch = batch
        ctx.device = charges.device
        return (torch.tensor(energies, dtype=torch.float64, device=charges.device),
                torch.tensor(forces, dtype=torch.float64, device=charges.device))

    @staticmethod
    def backward(ctx, grad_energies, grad_forces):
        batch = ctx.batch
        gE = None if grad_energies is None else grad_energies.detach().cpu().double().numpy()
        gF = None if grad_forces is None else grad_forces.detach().cpu().double().numpy()
        out = np.zeros((batch.system.n, 6))
        for c, (sl, k) in enumerate(zip(batch.slices(), batch.kernels)):
            out[sl] = k.adjoint(None if gF is None else gF[sl], 0.0 if gE is None else float(gE[c]))
        t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device=ctx.device)
        return t(out[:, 0]), t(out[:, 1]), t(out[:, 2]), t(out[:, 3:6]), None


def thole_dipole_clusters(charges, polarizabilities, tholes, dipoles, batch: ClusterGradients):
    """(energies per cluster, forces) of every cluster, differentiable like thole_dipole."""
    return ClusterBatchFunction.apply(charges, polarizabilities, tholes, dipoles, batch)
