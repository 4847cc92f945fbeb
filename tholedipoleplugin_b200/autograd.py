"""torch.autograd.Function over the CUDA kernels.

``thole_dipole(charges, polarizabilities, tholes, dipoles, kernel, system)``
returns (energy, forces) as torch tensors and differentiates both with respect
to the per-particle charges, isotropic polarizabilities, Thole factors and
molecular-frame dipoles.  The backward is the hand-written adjoint of
tdp_adjoint (one adjoint solve of the same symmetric (alpha^-1 - T) system for
Mutual polarization, pair damping recomputed).  Positions, axis frames and
covalent maps are fixed inputs.

With CUDA tensors (float64) everything stays on the device: the parameters
go to the library by pointer (tdp_update_particle_params), the forces are
written into a device tensor, and the backward's cotangent and gradients are
device tensors too (tdp_adjoint_device); only the energy and the energy
cotangent cross as host scalars.  CPU tensors take the host path of the same
entry points.  Work runs on torch's current CUDA stream.

``thole_dipole_clusters`` does the same for a batch of isolated clusters with
one persistent launch forward (tdp_batch_compute) and one backward
(tdp_batch_adjoint).

A kernel (or batch) keeps the state of its last forward evaluation, so each
forward must be followed by its backward before the same object evaluates
again (the usual single forward/backward per step of a training loop).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi as A
from .batch import ClusterBatch
from .kernel import CudaCalcTholeDipoleForceKernel
from .systems import TholeSystem


def _dev(t: torch.Tensor) -> torch.Tensor:
    return t.detach().to(torch.float64).contiguous()


class TholeDipoleFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, charges, polarizabilities, tholes, dipoles, kernel: CudaCalcTholeDipoleForceKernel,
                system: TholeSystem, positions=None):
        n = kernel.n
        ctx.kernel = kernel
        ctx.device = charges.device
        ctx.cuda = charges.is_cuda
        if ctx.cuda:
            kernel.setStream(torch.cuda.current_stream(charges.device).cuda_stream)
            kernel.updateParticleParams(_dev(charges), _dev(dipoles).reshape(n, 3), _dev(polarizabilities),
                                        _dev(tholes))
            if positions is None:
                positions = torch.as_tensor(system.positions, dtype=torch.float64, device=charges.device)
            pos = _dev(positions).reshape(n, 3)
            forces = torch.zeros((n, 3), dtype=torch.float64, device=charges.device)
            energy = kernel.execute_device(pos.data_ptr(), A.F64, forces.data_ptr(), A.F64)
            return torch.tensor(energy, dtype=torch.float64, device=charges.device), forces
        kernel.updateParticleParams(charges.detach().double().numpy(), dipoles.detach().double().numpy().reshape(n, 3),
                                    polarizabilities.detach().double().numpy(), tholes.detach().double().numpy())
        pos = system.positions if positions is None else positions.detach().double().numpy().reshape(n, 3)
        energy, forces = kernel.execute(pos)
        return torch.tensor(energy, dtype=torch.float64), torch.from_numpy(forces)

    @staticmethod
    def backward(ctx, grad_energy, grad_forces):
        kernel = ctx.kernel
        gE = 0.0 if grad_energy is None else float(grad_energy)
        if ctx.cuda:
            kernel.setStream(torch.cuda.current_stream(ctx.device).cuda_stream)
            gF = None if grad_forces is None else _dev(grad_forces)
            g = torch.empty((kernel.n, 6), dtype=torch.float64, device=ctx.device)
            kernel.adjoint_device(0 if gF is None else gF.data_ptr(), gE, g.data_ptr())
        else:
            gF = None if grad_forces is None else grad_forces.detach().double().numpy()
            g = torch.from_numpy(kernel.adjoint(gF, gE))
        return g[:, 0], g[:, 1], g[:, 2], g[:, 3:6], None, None, None


def thole_dipole(charges, polarizabilities, tholes, dipoles, kernel, system, positions=None):
    return TholeDipoleFunction.apply(charges, polarizabilities, tholes, dipoles, kernel, system, positions)


class ClusterGradients:
    """A batch of isolated clusters (the cluster workload of the batched
    kernels, tdp_batch_*) for differentiation: one ClusterBatch evaluates every
    cluster in one persistent launch and runs every cluster's adjoint in one
    more.  A loss over the clusters' energies and forces differentiates with
    respect to every particle's charge, polarizability, Thole factor and
    molecular dipole.  Parameters are concatenated in cluster order (cluster c
    owns particles offsets[c]:offsets[c+1])."""

    def __init__(self, clusters, precision="double"):
        self.batch = ClusterBatch(clusters, precision=precision)
        self.system = self.batch.system
        self.offsets = self.batch.offsets
        self.num_clusters = self.batch.num_clusters
        self.n = self.batch.n
        self._pos = {}

    def positions(self, device) -> torch.Tensor:
        key = str(device)
        if key not in self._pos:
            self._pos[key] = torch.as_tensor(self.batch.positions, dtype=torch.float64, device=device).contiguous()
        return self._pos[key]

    def close(self):
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def slices(self):
        return [slice(int(self.offsets[c]), int(self.offsets[c + 1])) for c in range(self.num_clusters)]


class ClusterBatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, charges, polarizabilities, tholes, dipoles, cg: ClusterGradients):
        b = cg.batch
        ctx.cg = cg
        ctx.device = charges.device
        ctx.cuda = charges.is_cuda
        if ctx.cuda:
            b.setStream(torch.cuda.current_stream(charges.device).cuda_stream)
            b.updateParams(_dev(charges), _dev(dipoles).reshape(b.n, 3), _dev(polarizabilities), _dev(tholes))
            forces = torch.empty((b.n, 3), dtype=torch.float64, device=charges.device)
            energies = torch.empty(b.num_clusters, dtype=torch.float64, device=charges.device)
            b.compute_device(cg.positions(charges.device).data_ptr(), forces.data_ptr(), energies.data_ptr())
            return energies, forces
        b.updateParams(charges.detach().double().numpy(), dipoles.detach().double().numpy().reshape(b.n, 3),
                       polarizabilities.detach().double().numpy(), tholes.detach().double().numpy())
        energies, forces = b.compute()
        return torch.from_numpy(energies), torch.from_numpy(forces)

    @staticmethod
    def backward(ctx, grad_energies, grad_forces):
        b = ctx.cg.batch
        if ctx.cuda:
            b.setStream(torch.cuda.current_stream(ctx.device).cuda_stream)
            gE = None if grad_energies is None else _dev(grad_energies)
            gF = None if grad_forces is None else _dev(grad_forces)
            g = torch.empty((b.n, 6), dtype=torch.float64, device=ctx.device)
            b.adjoint_device(0 if gF is None else gF.data_ptr(), 0 if gE is None else gE.data_ptr(), g.data_ptr())
        else:
            gE = None if grad_energies is None else grad_energies.detach().double().numpy()
            gF = None if grad_forces is None else grad_forces.detach().double().numpy()
            g = torch.from_numpy(b.adjoint(gF, gE))
        return g[:, 0], g[:, 1], g[:, 2], g[:, 3:6], None


def thole_dipole_clusters(charges, polarizabilities, tholes, dipoles, batch: ClusterGradients):
    """(energies per cluster, forces) of every cluster, differentiable like thole_dipole."""
    return ClusterBatchFunction.apply(charges, polarizabilities, tholes, dipoles, batch)
